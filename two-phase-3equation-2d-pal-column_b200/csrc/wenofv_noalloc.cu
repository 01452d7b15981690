// wenofv_noalloc.cu -- one SSP-RK step without any device allocation.
//
// For callers that must not allocate device memory: code that owns the GPU's memory
// through its own pool or a framework allocator (where a stray cudaMalloc would bypass its
// accounting or fail its limit), programs that reserve all free device memory at start-up,
// and latency-bound loops that cannot afford the device synchronisation of cudaMalloc/cudaFree.
// They pass their own device input and output states; everything else the fused stage
// kernel needs -- the intermediate RK stage state, the grid metric, the instance
// descriptor, the loop/status block, the work list and the last-CTA counter -- lives in
// one file-scope device array of fixed size that every GPU loading the library keeps until
// the process exits.
//
// Limits (checked before any GPU work, WENOFV_EINVAL otherwise):
//   nvar x ny x pitch doubles <= WENOFV_NOALLOC_STATE_DOUBLES (4 MiB of state: e.g. 256 x 256
//   with 4 variables and pitch 256, or 362 x 362), 2 nx + ny <= 8192, work items <= 8192.
//
// The first call on a device looks up the array's device address with cudaGetSymbolAddress
// (with that device current); make that first call before any stream capture.  All calls
// share the one array, which keeps the last call's contents: every call rewrites what it
// reads (descriptor, metric, loop state, work list, counter), so nothing depends on the old
// contents, but two calls whose work overlaps on the GPU race on it and corrupt each other.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "wenofv_engine.h"

namespace wenofv {
namespace {

constexpr size_t NOALLOC_STATE_DOUBLES = (size_t)4 << 17; // 4 MiB of FP64 state
constexpr int NOALLOC_METRIC_DOUBLES = 8192;
constexpr int NOALLOC_MAX_WORK = 8192;
constexpr int NOALLOC_ROWS = 16; // rows per work item
constexpr int NOALLOC_NT = 128;  // CTA width of its stage kernels (the grids it takes are narrow)

// layout of the scratch array (each part 256-byte aligned)
constexpr size_t OFF_DESC = 0;
constexpr size_t OFF_STATE = 256;
constexpr size_t OFF_FIN = 512;
constexpr size_t OFF_COUNTER = 768;
constexpr size_t OFF_WORK = 1024;
constexpr size_t OFF_METRIC = OFF_WORK + NOALLOC_MAX_WORK * sizeof(WorkItem);
constexpr size_t OFF_STAGE = OFF_METRIC + NOALLOC_METRIC_DOUBLES * sizeof(double);
constexpr size_t SCRATCH_BYTES = OFF_STAGE + NOALLOC_STATE_DOUBLES * sizeof(double);
static_assert(sizeof(InstDesc) <= 256 && sizeof(InstState) <= 256, "scratch header layout");
static_assert(OFF_METRIC % 256 == 0 && OFF_STAGE % 256 == 0, "scratch alignment");

// In host code this name is only a stand-in: the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
unsigned char *g_addr[MAX_DEVICES] = {};

// puts the caller's current device back on every return path: the step makes cfg->device
// current for its copies and launches, and a framework caller's own device must not change
struct DeviceGuard {
    int saved = -1;
    DeviceGuard() { if (cudaGetDevice(&saved) != cudaSuccess) { saved = -1; (void)cudaGetLastError(); } }
    ~DeviceGuard() { if (saved >= 0) cudaSetDevice(saved); }
};

int scratch_address(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_addr[device] = (unsigned char *)p;
    }
    *out = g_addr[device];
    return WENOFV_OK;
}

} // namespace
} // namespace wenofv

using namespace wenofv;

extern "C" int wenofv_step_noalloc(const wenofv_config *cfg, const wenofv_eq_params *eq, const double *d_U,
                                   double *d_U_next, int pitch, double dt, void *stream, uint32_t *flags)
{
    int rc = validate(cfg, eq);
    if (rc) return rc;
    if (cfg->bc == WENOFV_BC_NEUMANN2) { set_error("NEUMANN2 needs a ghost frame: use a context (wenofv_set_frame)"); return WENOFV_ENOTSUP; }
    if (!d_U || !d_U_next || d_U == d_U_next) { set_error("need distinct device input and output states"); return WENOFV_EINVAL; }
    if (!std::isfinite(dt) || dt < 0.0) { set_error("dt must be a finite non-negative number"); return WENOFV_EINVAL; }
    if (pitch < cfg->nx) { set_error("pitch (%d) must be at least nx (%d)", pitch, cfg->nx); return WENOFV_EINVAL; }
    const int nv = nvar_of(eq->eq_kind);
    const int recon = eq->eq_kind == WENOFV_EQ_LINEAR_ADV ? 0 : cfg->reconstruction;
    const int sch = recon == 4 ? 2 : cfg->scheme; // PRIMITIVE3: the 7-point geometry
    const int strictf = cfg->precision == WENOFV_FP64_STRICT, fp32 = cfg->precision == WENOFV_FP32_BULK;
    const size_t state = (size_t)nv * cfg->ny * pitch;
    if (state > NOALLOC_STATE_DOUBLES) {
        set_error("the no-allocation step holds at most %zu state doubles (nvar*ny*pitch = %zu)", NOALLOC_STATE_DOUBLES, state);
        return WENOFV_EINVAL;
    }
    if (2 * (size_t)cfg->nx + cfg->ny > (size_t)NOALLOC_METRIC_DOUBLES) {
        set_error("the no-allocation step needs 2*nx + ny <= %d", NOALLOC_METRIC_DOUBLES);
        return WENOFV_EINVAL;
    }
    const int tx = strictf ? strict::stage_tx(eq->eq_kind, recon, 0, sch, NOALLOC_NT) : fast::stage_tx(eq->eq_kind, recon, fp32, sch, NOALLOC_NT);
    const long nwork = (long)((cfg->nx + tx - 1) / tx) * ((cfg->ny + NOALLOC_ROWS - 1) / NOALLOC_ROWS);
    if (nwork > NOALLOC_MAX_WORK) { set_error("the no-allocation step takes at most %d work items", NOALLOC_MAX_WORK); return WENOFV_EINVAL; }

    if (cfg->device < 0 || cfg->device >= MAX_DEVICES) { set_error("device ordinal out of range"); return WENOFV_EINVAL; }
    const DeviceGuard device_guard;
    WENOFV_CUDA(cudaSetDevice(cfg->device));
    unsigned char *base = nullptr;
    rc = scratch_address(cfg->device, &base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;

    // buffer roles of the step's stages: the input is buffer 0, the caller's output is the
    // buffer the last stage writes, the scratch state is the remaining one
    const int out_buf = stage_roles(cfg->rk_method, 0, stage_count(cfg->rk_method) - 1).bout;
    double *scratch_state = (double *)(base + OFF_STAGE);
    double *metric = (double *)(base + OFF_METRIC);

    InstDesc d;
    std::memset(&d, 0, sizeof d);
    d.buf[0] = const_cast<double *>(d_U); // only ever read: no stage writes buffer 0 of a parity-0 step
    d.buf[out_buf] = d_U_next;
    d.buf[3 - out_buf] = scratch_state;
    d.dxc = metric;
    d.dxl = metric + cfg->nx;
    d.dy = metric + 2 * cfg->nx;
    d.nx = cfg->nx; d.ny = cfg->ny; d.pitch = pitch; d.bc = cfg->bc;
    d.scheme = cfg->scheme; d.flux = cfg->riemann_flux; d.limiter = cfg->pp_limiter; d.recon = recon;
    d.eq_kind = eq->eq_kind;
    d.cfl = cfg->cfl;
    d.dX = (cfg->xr - cfg->xl) / cfg->nx;
    d.dx4 = std::pow(d.dX, 4); // the reference's pow(m_deltaX, 4), include/Utility.hpp:313
    d.dY = (cfg->yr - cfg->yl) / cfg->ny;
    d.eq = eq_params_of(*eq);

    InstState st;
    std::memset(&st, 0, sizeof st);
    const double one = 1.0;
    std::memcpy(&st.accum, &one, sizeof one);
    st.bad_cell = -1;
    st.dt = dt;
    st.mode = MODE_MANUAL;

    // host staging on the stack; the stream is synchronised after the copies from it, so the
    // buffers can go out of scope (or be refilled) safely
    double met[NOALLOC_METRIC_DOUBLES];
    grid_metric(*cfg, met, met + cfg->nx, met + 2 * cfg->nx);
    WorkItem work[NOALLOC_MAX_WORK / 8];
    const int fin = 0;
    WENOFV_CUDA(cudaMemcpyAsync(base + OFF_DESC, &d, sizeof d, cudaMemcpyHostToDevice, s));
    WENOFV_CUDA(cudaMemcpyAsync(base + OFF_STATE, &st, sizeof st, cudaMemcpyHostToDevice, s));
    WENOFV_CUDA(cudaMemcpyAsync(base + OFF_FIN, &fin, sizeof fin, cudaMemcpyHostToDevice, s));
    WENOFV_CUDA(cudaMemsetAsync(base + OFF_COUNTER, 0, sizeof(unsigned int), s)); // must start at zero
    WENOFV_CUDA(cudaMemcpyAsync(metric, met, (2 * (size_t)cfg->nx + cfg->ny) * sizeof(double), cudaMemcpyHostToDevice, s));
    int k = 0, chunk0 = 0;
    for (int j0 = 0; j0 < cfg->ny; j0 += NOALLOC_ROWS)
        for (int i0 = 0; i0 < cfg->nx; i0 += tx) {
            work[k++ - chunk0] = WorkItem{0, i0, j0, j0 + NOALLOC_ROWS < cfg->ny ? j0 + NOALLOC_ROWS : cfg->ny};
            if (k - chunk0 == NOALLOC_MAX_WORK / 8) {
                WENOFV_CUDA(cudaMemcpyAsync(base + OFF_WORK + chunk0 * sizeof(WorkItem), work,
                                            (k - chunk0) * sizeof(WorkItem), cudaMemcpyHostToDevice, s));
                WENOFV_CUDA(cudaStreamSynchronize(s));
                chunk0 = k;
            }
        }
    if (k > chunk0)
        WENOFV_CUDA(cudaMemcpyAsync(base + OFF_WORK + chunk0 * sizeof(WorkItem), work, (k - chunk0) * sizeof(WorkItem),
                                    cudaMemcpyHostToDevice, s));
    WENOFV_CUDA(cudaStreamSynchronize(s));

    int sms = 0;
    WENOFV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device));
    const int flx = eq->eq_kind == WENOFV_EQ_LINEAR_ADV ? 0 : cfg->riemann_flux;
    const int bps = strictf ? strict::stage_blocks_per_sm(eq->eq_kind, recon, fp32, sch, flx, NOALLOC_NT)
                            : fast::stage_blocks_per_sm(eq->eq_kind, recon, fp32, sch, flx, NOALLOC_NT);
    const int grid = (int)(k < (long)sms * (bps > 0 ? bps : 1) ? k : (long)sms * (bps > 0 ? bps : 1));
    for (int stage = 0; stage < stage_count(cfg->rk_method); stage++) {
        const Roles ro = stage_roles(cfg->rk_method, 0, stage);
        StageLaunch L;
        std::memset(&L, 0, sizeof L);
        L.inst = (const InstDesc *)(base + OFF_DESC);
        L.state = (InstState *)(base + OFF_STATE);
        L.work = (const WorkItem *)(base + OFF_WORK);
        L.nwork = k;
        L.fin_ids = (const int *)(base + OFF_FIN);
        L.nfin = 1;
        L.counter = (unsigned int *)(base + OFF_COUNTER);
        L.bin = ro.bin; L.bun = ro.bun; L.bout = ro.bout;
        L.first_stage = stage == 0;
        L.final_stage = stage == stage_count(cfg->rk_method) - 1;
        L.rk1 = cfg->rk_method == 0;
        stage_coeffs(cfg->rk_method, stage, L.A, L.B, L.C);
        const int lrc = strictf ? strict::launch_stage(eq->eq_kind, recon, 0, sch, flx, NOALLOC_NT, L, grid, stream)
                                : fast::launch_stage(eq->eq_kind, recon, fp32, sch, flx, NOALLOC_NT, L, grid, stream);
        if (lrc) return cuda_fail((cudaError_t)lrc, "stage kernel launch");
    }
    if (flags) {
        InstState out;
        WENOFV_CUDA(cudaMemcpyAsync(&out, base + OFF_STATE, sizeof out, cudaMemcpyDeviceToHost, s));
        WENOFV_CUDA(cudaStreamSynchronize(s));
        *flags = out.flags;
    }
    return WENOFV_OK;
}
