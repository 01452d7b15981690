// wenofv_engine.cu -- host side of the C ABI: instances, work lists, buffer rotation and
// the device-resident time loop in captured CUDA graphs.
#include <nvtx3/nvToolsExt.h> // header-only NVTX ranges: the host phases show up in nsys/ncu timelines

#include "wenofv_engine.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

namespace wenofv {

static thread_local char g_err[512];

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
const char *last_error_text() { return g_err; }

int cuda_fail(cudaError_t e, const char *what)
{
    set_error("%s: %s", what, cudaGetErrorString(e));
    (void)cudaGetLastError(); // a failed allocation is not sticky: do not let a later check see it
    return e == cudaErrorMemoryAllocation ? WENOFV_ENOMEM : WENOFV_ECUDA;
}

int nvar_of(int k) { return k == WENOFV_EQ_LINEAR_ADV ? 1 : 4; }

EqParams eq_params_of(const wenofv_eq_params &e)
{
    EqParams P{e.eq_kind, e.rho10, e.rho20, e.sound1, e.sound2, e.preb, e.gamma, e.adv_u, e.adv_v,
               e.gamma1, e.pinf1, e.gamma2, e.pinf2, e.gravity};
    if (e.eq_kind == WENOFV_EQ_TWO_PHASE_SG) { // the linearised sound speeds: the first guess of the equilibrium
        P.sound1 = std::sqrt(e.gamma1 * (e.preb + e.pinf1) / e.rho10);
        P.sound2 = std::sqrt(e.gamma2 * (e.preb + e.pinf2) / e.rho20);
    }
    return P;
}

int validate(const wenofv_config *c, const wenofv_eq_params *e)
{
    if (!c || !e) { set_error("null config or equation"); return WENOFV_EINVAL; }
    if (c->nx < 1 || c->ny < 1) { set_error("nx, ny must be positive (got %d, %d)", c->nx, c->ny); return WENOFV_EINVAL; }
    if (!(c->xr > c->xl) || !(c->yr > c->yl)) { set_error("empty domain"); return WENOFV_EINVAL; }
    if (c->rk_method < 0 || c->rk_method > 2) { set_error("RKMETH must be 0, 1 or 2"); return WENOFV_EINVAL; }
    if (!(c->cfl > 0)) { set_error("CFL must be positive"); return WENOFV_EINVAL; }
    if (c->scheme < 0 || c->scheme > 2) { set_error("SCHEME must be 0, 1 or 2"); return WENOFV_EINVAL; }
    if (c->scheme == 2 && c->precision == WENOFV_FP32_BULK) {
        // lambda^2 h^2 is a ratio of 5th to 3rd differences, which FP32 rounds to noise on smooth data
        set_error("SCHEME 2 (WENOEXP) runs in FP64 only");
        return WENOFV_ENOTSUP;
    }
    if (c->reconstruction == 5) {
        // ThincOnlyForZ1: the reference's dispatch has no branch for it (src/WENOFV.cpp:593-598)
        set_error("RECONSTRUCTIONTYPE 5 is not supported");
        return WENOFV_ENOTSUP;
    }
    if (c->reconstruction < 0 || c->reconstruction > 4) { set_error("RECONSTRUCTIONTYPE must be 0 .. 4"); return WENOFV_EINVAL; }
    if (c->reconstruction == 4 && c->precision == WENOFV_FP32_BULK) {
        set_error("RECONSTRUCTIONTYPE 4 (PRIMITIVE3) runs in FP64 only");
        return WENOFV_ENOTSUP;
    }
    if (c->reconstruction >= 2 && e && e->eq_kind != WENOFV_EQ_TWO_PHASE) {
        set_error("RECONSTRUCTIONTYPE %d (primitive variables) is defined for the two-phase model only", c->reconstruction);
        return WENOFV_ENOTSUP;
    }
    if (c->riemann_flux < 0 || c->riemann_flux > 1) { set_error("RIEMANNFLUX must be 0 or 1"); return WENOFV_EINVAL; }
    if (c->pp_limiter < 0 || c->pp_limiter > 1) { set_error("PPlimiter must be 0 or 1"); return WENOFV_EINVAL; }
    if (c->bc < 0 || c->bc > 5) { set_error("boundary kind %d is not supported", c->bc); return WENOFV_ENOTSUP; }
    if (c->precision < 0 || c->precision > 2) { set_error("unknown precision %d", c->precision); return WENOFV_EINVAL; }
    if (c->ref_slabs < 0 || (c->ref_slabs > 0 && c->nx % c->ref_slabs != 0)) {
        set_error("ELEMNUMX (%d) must be divisible by the slab count (%d)", c->nx, c->ref_slabs);
        return WENOFV_EINVAL;
    }
    if (e->eq_kind < 0 || e->eq_kind > 3) { set_error("unknown equation kind %d", e->eq_kind); return WENOFV_EINVAL; }
    if (!(e->gravity == e->gravity) || (e->gravity != 0.0 && e->eq_kind != WENOFV_EQ_TWO_PHASE && e->eq_kind != WENOFV_EQ_TWO_PHASE_SG)) {
        set_error("gravity is a finite source of the two-phase kinds");
        return WENOFV_EINVAL;
    }
    if (e->eq_kind == WENOFV_EQ_TWO_PHASE_SG) {
        if (!(e->gamma1 > 1.0 && e->gamma2 > 1.0 && e->pinf1 >= 0.0 && e->pinf2 >= 0.0 && e->rho10 > 0.0 && e->rho20 > 0.0 &&
              e->preb + e->pinf1 > 0.0 && e->preb + e->pinf2 > 0.0)) {
            set_error("stiffened gas needs gamma_k > 1, pinf_k >= 0, rho_k0 > 0 and preb + pinf_k > 0");
            return WENOFV_EINVAL;
        }
        if (c->reconstruction > 1) {
            set_error("the stiffened-gas model has RECONSTRUCTIONTYPE 0 and 1 only");
            return WENOFV_ENOTSUP;
        }
        if (c->precision == WENOFV_FP32_BULK) { set_error("the stiffened-gas model runs in FP64 only"); return WENOFV_ENOTSUP; }
    }
    if (e->eq_kind == WENOFV_EQ_TWO_PHASE && !(e->sound1 > 0 && e->sound2 > 0)) { set_error("sound speeds must be positive"); return WENOFV_EINVAL; }
    if (e->eq_kind == WENOFV_EQ_EULER && !(e->gamma > 1.0)) { set_error("gamma must exceed 1"); return WENOFV_EINVAL; }
    if ((size_t)c->nx * c->ny > (size_t)1 << 31) { set_error("grid too large"); return WENOFV_EINVAL; }
    return WENOFV_OK;
}

// Cell sizes exactly as the reference's grid generator rounds them (src/WENOFV.cpp:89-123):
// rank p of a P-slab decomposition builds its cells from its own ghost origin.
void grid_metric(const wenofv_config &c, double *dxc, double *dxl, double *dy)
{
    const double dX = (c.xr - c.xl) / c.nx, dY = (c.yr - c.yl) / c.ny;
    const int G = 3;
    if (c.ref_slabs <= 0) {
        for (int i = 0; i < c.nx; i++) dxc[i] = dxl[i] = dX;
        for (int j = 0; j < c.ny; j++) dy[j] = dY;
        return;
    }
    const int m = c.nx / c.ref_slabs;
    for (int g = 0; g < c.nx; g++) {
        const int rank = g / m, ei = g - rank * m + G;
        const double procXLeft = c.xl + rank * m * dX;
        const double ghostLeft = procXLeft - dX * G;
        dxc[g] = (ghostLeft + (ei + 1) * dX) - (ghostLeft + ei * dX);
        dxl[g] = (ghostLeft + ei * dX) - (ghostLeft + (ei - 1) * dX);
    }
    const double procYLeft = c.yl + 0 * c.ny * dY;
    const double ghostBottom = procYLeft - dY * G;
    for (int j = 0; j < c.ny; j++) dy[j] = (ghostBottom + (j + G + 1) * dY) - (ghostBottom + (j + G) * dY);
}

int stage_count(int rk) { return rk + 1; }

Roles stage_roles(int rk, int parity, int stage)
{
    static const Roles r3[2][3] = {{{0, 0, 1}, {1, 0, 2}, {2, 0, 1}}, {{1, 1, 0}, {0, 1, 2}, {2, 1, 0}}};
    static const Roles r2[2][2] = {{{0, 0, 1}, {1, 0, 2}}, {{2, 2, 1}, {1, 2, 0}}};
    static const Roles r1[2][1] = {{{0, 0, 1}}, {{1, 1, 0}}};
    if (rk == 2) return r3[parity][stage];
    if (rk == 1) return r2[parity][stage];
    return r1[parity][stage];
}
static int end_buffer(int rk, int parity) { return stage_roles(rk, parity, stage_count(rk) - 1).bout; }

// SSP-RK stage coefficients of RunRK2/RunRK3, src/WENOFV.cpp:402-418, :443-465
void stage_coeffs(int rk, int stage, double &A, double &B, double &C)
{
    if (rk == 2) {
        static const double a[3] = {1.0, 3.0 / 4.0, 1.0 / 3.0}, b[3] = {0.0, 1.0 / 4.0, 2.0 / 3.0}, c[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
        A = a[stage]; B = b[stage]; C = c[stage];
    } else if (rk == 1) {
        static const double a[2] = {1.0, 0.5}, b[2] = {0.0, 0.5}, c[2] = {1.0, 0.5};
        A = a[stage]; B = b[stage]; C = c[stage];
    } else {
        A = 0.0; B = 1.0; C = 1.0;
    }
}

static InstState fresh_state(int cur)
{
    InstState s;
    std::memset(&s, 0, sizeof s);
    const double one = 1.0;
    std::memcpy(&s.accum, &one, sizeof one);
    s.bad_cell = -1;
    s.cur_buf = cur;
    s.mode = MODE_MANUAL;
    return s;
}

Engine::~Engine()
{
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (copy_stream_) cudaStreamSynchronize(copy_stream_);
    drop_graphs();
    free_work();
    for (int i = 0; i < cap_; i++) free_instance(i);
    cudaFree(d_desc_);
    cudaFree(d_state_);
    cudaFree(d_rhs_);
    if (h_state_) cudaFreeHost(h_state_);
    if (h_stage_) cudaFreeHost(h_stage_);
    cudaFree(d_snap_);
    if (h_snap_) cudaFreeHost(h_snap_);
    if (snap_ready_) cudaEventDestroy(snap_ready_);
    if (snap_done_) cudaEventDestroy(snap_done_);
    if (fork_) cudaEventDestroy(fork_);
    cudaFree(arena_);
    if (copy_stream_) cudaStreamDestroy(copy_stream_);
    if (stream) cudaStreamDestroy(stream);
}

size_t Engine::bytes_needed(const wenofv_config &c, const wenofv_eq_params &e)
{
    const size_t pitch = (size_t)(c.nx + 15) / 16 * 16;
    return 3 * (size_t)nvar_of(e.eq_kind) * c.ny * pitch * sizeof(double) + (2 * (size_t)c.nx + c.ny) * sizeof(double);
}

int Engine::init_slots(int capacity, int dev, int rk_method, size_t arena_bytes)
{
    if (capacity < 1) { set_error("capacity must be positive"); return WENOFV_EINVAL; }
    device = dev;
    rk = rk_method;
    int ndev = 0;
    WENOFV_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) { set_error("no CUDA device %d", device); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    WENOFV_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device));
    WENOFV_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    cap_ = capacity;
    cfg_.assign(cap_, wenofv_config{});
    eq_.assign(cap_, wenofv_eq_params{});
    desc_.assign(cap_, InstDesc{});
    dmem_.assign(cap_, nullptr);
    dmetric_.assign(cap_, nullptr);
    dframe_.assign(cap_, nullptr);
    dtheta_.assign(cap_, nullptr);
    frame_set_.assign(cap_, 0);
    live_.assign(cap_, 0);
    WENOFV_CUDA(cudaMalloc(&d_desc_, cap_ * sizeof(InstDesc)));
    WENOFV_CUDA(cudaMemset(d_desc_, 0, cap_ * sizeof(InstDesc)));
    WENOFV_CUDA(cudaMalloc(&d_state_, cap_ * sizeof(InstState)));
    WENOFV_CUDA(cudaMallocHost(&h_state_, cap_ * sizeof(InstState)));
    for (int i = 0; i < cap_; i++) {
        h_state_[i] = fresh_state(0);
        h_state_[i].done = 1; // an empty slot is never stepped
    }
    slot_off_.assign(cap_, 0);
    if (arena_bytes > 0) {
        arena_bytes = arena_bytes / 256 * 256;
        WENOFV_CUDA(cudaMalloc((void **)&arena_, arena_bytes));
        arena_bytes_ = arena_bytes;
        arena_freelist_.clear();
        arena_freelist_[0] = arena_bytes;
        arena_used_.clear();
    }
    return push_state();
}

// first fit over the free blocks; neighbouring free blocks are merged on release
int Engine::arena_alloc(size_t bytes, size_t *off)
{
    bytes = (bytes + 255) / 256 * 256;
    for (auto it = arena_freelist_.begin(); it != arena_freelist_.end(); ++it) {
        if (it->second < bytes) continue;
        const size_t o = it->first, rest = it->second - bytes;
        arena_freelist_.erase(it);
        if (rest) arena_freelist_[o + bytes] = rest;
        arena_used_[o] = bytes;
        *off = o;
        return WENOFV_OK;
    }
    set_error("the slot arena has no free block of %zu bytes", bytes);
    return WENOFV_ENOMEM;
}

void Engine::arena_free(size_t off)
{
    auto u = arena_used_.find(off);
    if (u == arena_used_.end()) return;
    size_t o = off, sz = u->second;
    arena_used_.erase(u);
    auto nx = arena_freelist_.lower_bound(o);
    if (nx != arena_freelist_.end() && nx->first == o + sz) { // merge with the block after
        sz += nx->second;
        nx = arena_freelist_.erase(nx);
    }
    if (nx != arena_freelist_.begin()) { // merge with the block before
        auto pv = std::prev(nx);
        if (pv->first + pv->second == o) {
            o = pv->first;
            sz += pv->second;
            arena_freelist_.erase(pv);
        }
    }
    arena_freelist_[o] = sz;
}

size_t Engine::arena_free_bytes() const
{
    size_t f = 0;
    for (const auto &kv : arena_freelist_) f += kv.second;
    return f;
}

// NEUMANN2's fixed ghost frame: every variable on the grid widened by 4 cells on each side
// (the widest halo, WENOEXP's), SoA [v][ny+8][nx+8]; the interior entries are never read
static size_t frame_bytes(const wenofv_config &c, const wenofv_eq_params &e)
{
    return (size_t)nvar_of(e.eq_kind) * ((size_t)c.ny + 8) * ((size_t)c.nx + 8) * sizeof(double);
}

int Engine::set_frame(int i, const double *frame)
{
    if (!live(i)) { set_error("instance %d is not live", i); return WENOFV_EINVAL; }
    if (cfg_[i].bc != WENOFV_BC_NEUMANN2) { set_error("a ghost frame belongs to the NEUMANN2 boundary only"); return WENOFV_EINVAL; }
    if (!frame) { set_error("null frame"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    // synchronous: the caller may reuse its array on return, and later stages read the copy
    WENOFV_CUDA(cudaMemcpyAsync(dframe_[i], frame, frame_bytes(cfg_[i], eq_[i]), cudaMemcpyHostToDevice, stream));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    frame_set_[i] = 1;
    return WENOFV_OK;
}

int Engine::check_frames() const
{
    for (int i = 0; i < n; i++)
        if (live_[i] && cfg_[i].bc == WENOFV_BC_NEUMANN2 && !frame_set_[i]) {
            set_error("instance %d has the NEUMANN2 boundary but no ghost frame (wenofv_set_frame)", i);
            return WENOFV_EINVAL;
        }
    return WENOFV_OK;
}

int Engine::alloc_instance(int i, const wenofv_config &c, const wenofv_eq_params &e)
{
    const int nv = nvar_of(e.eq_kind);
    const int pitch = (c.nx + 15) / 16 * 16;
    const size_t per = (size_t)nv * c.ny * pitch;
    std::vector<double> met(2 * (size_t)c.nx + c.ny);
    grid_metric(c, met.data(), met.data() + c.nx, met.data() + 2 * c.nx);
    if (arena_) { // one arena block: three state buffers, then the metric
        size_t off = 0;
        const int rc = arena_alloc(bytes_needed(c, e), &off);
        if (rc) return rc;
        slot_off_[i] = off;
        dmem_[i] = (double *)(arena_ + off);
        dmetric_[i] = dmem_[i] + 3 * per;
    } else {
        WENOFV_CUDA(cudaMalloc(&dmem_[i], 3 * per * sizeof(double)));
        WENOFV_CUDA(cudaMalloc(&dmetric_[i], met.size() * sizeof(double)));
    }
    WENOFV_CUDA(cudaMemsetAsync(dmem_[i], 0, 3 * per * sizeof(double), stream));
    WENOFV_CUDA(cudaMemcpyAsync(dmetric_[i], met.data(), met.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
    InstDesc &d = desc_[i];
    std::memset(&d, 0, sizeof d);
    for (int b = 0; b < 3; b++) d.buf[b] = dmem_[i] + b * per;
    d.dxc = dmetric_[i];
    d.dxl = dmetric_[i] + c.nx;
    d.dy = dmetric_[i] + 2 * c.nx;
    d.nx = c.nx; d.ny = c.ny; d.pitch = pitch; d.bc = c.bc;
    d.scheme = c.scheme; d.flux = c.riemann_flux; d.limiter = c.pp_limiter;
    d.recon = e.eq_kind == WENOFV_EQ_LINEAR_ADV ? 0 : c.reconstruction;
    d.eq_kind = e.eq_kind;
    d.cfl = c.cfl;
    d.dX = (c.xr - c.xl) / c.nx;
    d.dx4 = std::pow(d.dX, 4); // the reference's pow(m_deltaX, 4), include/Utility.hpp:313
    d.dY = (c.yr - c.yl) / c.ny;
    d.eq = eq_params_of(e);
    frame_set_[i] = 0;
    if (c.bc == WENOFV_BC_NEUMANN2) {
        WENOFV_CUDA(cudaMalloc(&dframe_[i], frame_bytes(c, e)));
        d.frame = dframe_[i];
    }
    if (theta_record && c.pp_limiter && e.eq_kind != WENOFV_EQ_LINEAR_ADV) { // the limiter's per-cell record
        WENOFV_CUDA(cudaMalloc(&dtheta_[i], (size_t)c.nx * c.ny));
        WENOFV_CUDA(cudaMemsetAsync(dtheta_[i], 0, (size_t)c.nx * c.ny, stream));
        d.theta_flag = dtheta_[i];
    }
    // from pageable host memory: both copies have read their sources when they return
    WENOFV_CUDA(cudaMemcpyAsync(d_desc_ + i, &d, sizeof(InstDesc), cudaMemcpyHostToDevice, stream));
    if (!arena_) WENOFV_CUDA(cudaStreamSynchronize(stream));
    cfg_[i] = c;
    eq_[i] = e;
    live_[i] = 1;
    h_state_[i] = fresh_state(0);
    work_dirty_ = true;
    return WENOFV_OK;
}

void Engine::free_instance(int i)
{
    if (i < 0 || i >= cap_) return;
    if (arena_) {
        if (dmem_[i]) arena_free(slot_off_[i]);
    } else {
        if (dmem_[i]) cudaFree(dmem_[i]);
        if (dmetric_[i]) cudaFree(dmetric_[i]);
    }
    if (dframe_[i]) cudaFree(dframe_[i]);
    if (dtheta_[i]) cudaFree(dtheta_[i]);
    dmem_[i] = nullptr;
    dmetric_[i] = nullptr;
    dframe_[i] = nullptr;
    dtheta_[i] = nullptr;
    frame_set_[i] = 0;
    if (live_[i]) work_dirty_ = true;
    live_[i] = 0;
    if (h_state_) {
        h_state_[i] = fresh_state(0);
        h_state_[i].done = 1;
    }
}

int Engine::init(int count, const wenofv_config *cfgs, const wenofv_eq_params *eqs)
{
    if (count < 1) { set_error("instance count must be positive"); return WENOFV_EINVAL; }
    for (int i = 0; i < count; i++) {
        const int rc = validate(&cfgs[i], &eqs[i]);
        if (rc) return rc;
        if (cfgs[i].device != cfgs[0].device || cfgs[i].rk_method != cfgs[0].rk_method) {
            set_error("all instances of a batch share the device and RKMETH");
            return WENOFV_EINVAL;
        }
    }
    int rc = init_slots(count, cfgs[0].device, cfgs[0].rk_method);
    if (rc) return rc;
    n = count;
    for (int i = 0; i < n && !rc; i++) rc = alloc_instance(i, cfgs[i], eqs[i]);
    if (!rc) rc = push_state();
    if (!rc) rc = ensure_work();
    return rc;
}

int Engine::ensure_work()
{
    if (!work_dirty_) return WENOFV_OK;
    WENOFV_CUDA(cudaStreamSynchronize(stream)); // the lists may be in use by queued launches
    const int rc = build_work();                // drops the graphs when a buffer moved
    if (!rc) work_dirty_ = false;
    return rc;
}

int Engine::add(const wenofv_config &c, const wenofv_eq_params &e, int *slot)
{
    int rc = validate(&c, &e);
    if (rc) return rc;
    if (c.rk_method != rk || c.device != device) { set_error("slot RKMETH/device differ from the server's"); return WENOFV_ENOTSUP; }
    int k = -1;
    for (int i = 0; i < cap_; i++)
        if (!live_[i]) { k = i; break; }
    if (k < 0) { set_error("no free slot"); return WENOFV_EBUSY; }
    WENOFV_CUDA(cudaSetDevice(device));
    rc = alloc_instance(k, c, e);
    if (rc) { free_instance(k); return rc; }
    n = std::max(n, k + 1);
    *slot = k;
    return WENOFV_OK;
}

int Engine::remove(int slot)
{
    if (!live(slot)) { set_error("slot %d is not live", slot); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    free_instance(slot);
    WENOFV_CUDA(cudaMemcpyAsync(d_state_ + slot, &h_state_[slot], sizeof(InstState), cudaMemcpyHostToDevice, stream));
    return WENOFV_OK;
}

int Engine::start(int slot, double t_end, int64_t max_steps)
{
    return start_many(std::vector<int>{slot}, std::vector<double>{t_end}, std::vector<int64_t>{max_steps});
}

int Engine::run_pairs(int K)
{
    WENOFV_CUDA(cudaSetDevice(device));
    int rc = ensure_work();
    for (int k = 0; k < K && !rc; k++)
        for (int p = 0; p < 2 && !rc; p++)
            for (int s = 0; s < stage_count(rk) && !rc; s++) rc = launch_stage_all(p, s, nullptr);
    return rc;
}

int Engine::run_graph_pairs(int K)
{
    WENOFV_CUDA(cudaSetDevice(device));
    const int rc = ensure_work();
    if (rc) return rc;
    return run_graph(K);
}

int Engine::refresh() { return pull_state(); }

void Engine::free_work()
{
    for (Group &g : groups_) {
        cudaFree(g.d_work);
        cudaFree(g.d_fin);
        cudaFree(g.d_counts);
        cudaFree(g.d_init_work);
        cudaFree(g.d_init_fin);
        cudaFree(g.d_counter);
        if (g.gstream) cudaStreamDestroy(g.gstream);
        if (g.joined) cudaEventDestroy(g.joined);
    }
    groups_.clear();
}

// rows per work item of a launch group whose instances `inst` have strips of tx columns and
// `slots` resident CTAs (the tiling override when set)
int Engine::item_rows(const std::vector<int> &inst, int tx, int slots) const
{
    if (rows_per_item_ > 0) return rows_per_item_;
    long strips_rows = 0;
    for (int i : inst) strips_rows += (long)((cfg_[i].nx + tx - 1) / tx) * cfg_[i].ny;
    int seg = 32;
    if (slots > 2 * sms_) {
        // many resident CTAs per SM (the 128-thread kernels): long enough to amortise the 2
        // halo rows, short enough to fill the GPU (measured best on the 1024^2 column)
        while (seg > 8 && strips_rows / seg < 2L * slots) seg /= 2;
        // a grid that leaves SMs idle even at 8 rows: shorter items, since each CTA's time
        // is its rows in sequence (latency-bound), not the work
        while (seg > 2 && strips_rows / seg < sms_) seg /= 2;
        return seg;
    }
    // 1-2 resident CTAs per SM: the CTAs take items in waves, and an item of s rows costs
    // about s + 2 halo rows + 3 rows' worth of start-up (its first 2H+1 rows load before the
    // loop; measured: 8 % of a 32-row item); pick the s of the shortest waves x (s + 5).  On
    // the 1024^2 column it picks 64 rows: 0.897 ms per stage against 0.972 for 16 and 0.924 for
    // 32 (measured).
    double best = 1e300;
    for (int s : {2, 4, 8, 16, 24, 32, 48, 64}) {
        const double cost = waves_of(inst, tx, slots, s) * (s + 5);
        if (cost < best - 1e-9) { best = cost; seg = s; }
    }
    return seg;
}

// waves of work items of s rows over `slots` resident CTAs
double Engine::waves_of(const std::vector<int> &inst, int tx, int slots, int s) const
{
    long items = 0;
    for (int i : inst) items += (long)((cfg_[i].nx + tx - 1) / tx) * ((cfg_[i].ny + s - 1) / s);
    return std::ceil((double)items / std::max(1, slots));
}

// the CTA width of an instance's stage kernel: 256 (strips of 58 columns) or 128 (26 columns)
// where both exist.  The override (wenofv_batch_set_threads, the autotuner) forces one width
// where it exists.
//
// Among many instances (batches, servers) the GPU is full, so the throughput decides: the
// wide kernel costs about 0.85 (FP64) or 0.93 (FP32-bulk) of the narrow one per column-row it
// computes (measured on a 1024-wide grid), but rounds the grid's width up to whole strips of
// 58; the width of the smaller cost x padded width.
//
// A context's single instance is alone on the GPU, and a small grid does not fill it: its
// stage takes the waves of work items of its own tiling (item_rows) x (rows + 5) row
// iterations, and a row iteration of the wide kernel takes about 1.3 (FP64) or 1.1 (FP32-bulk)
// of the narrow one's (measured on the 1024^2 and 256^2 columns: 0.725 against 0.896 ms per
// FP64 stage at 1024^2, 0.119 against 0.098 ms at 256^2, where the narrow kernel's 10 strips
// spread over more SMs than the wide kernel's 5).
int Engine::instance_nt(int i) const
{
    const int eqk = desc_[i].eq_kind, recon = desc_[i].recon;
    const int strict = cfg_[i].precision == WENOFV_FP64_STRICT, fp32 = cfg_[i].precision == WENOFV_FP32_BULK;
    const int wide = strict ? strict::stage_wide(eqk, recon) : fast::stage_wide(eqk, recon);
    if (!wide) return 128;
    if (nt_override_ == 128 || nt_override_ == 256) return nt_override_;
    const int sch = recon == 4 ? 2 : desc_[i].scheme;
    const int tn = strict ? strict::stage_tx(eqk, recon, fp32, sch, 128) : fast::stage_tx(eqk, recon, fp32, sch, 128);
    const int tw = strict ? strict::stage_tx(eqk, recon, fp32, sch, 256) : fast::stage_tx(eqk, recon, fp32, sch, 256);
    if (solo) {
        const std::vector<int> one{i};
        const int flx = eqk == WENOFV_EQ_LINEAR_ADV ? 0 : desc_[i].flux;
        double rows_t[2];
        const int nts[2] = {128, 256};
        for (int k = 0; k < 2; k++) {
            const int tx = k ? tw : tn;
            const int bps = std::max(1, strict ? strict::stage_blocks_per_sm(eqk, recon, fp32, sch, flx, nts[k])
                                               : fast::stage_blocks_per_sm(eqk, recon, fp32, sch, flx, nts[k]));
            const int slots = sms_ * (ctas_per_sm_ > 0 ? std::min(ctas_per_sm_, bps) : bps);
            const int seg = item_rows(one, tx, slots);
            rows_t[k] = waves_of(one, tx, slots, seg) * (seg + 5);
        }
        return (fp32 ? 1.1 : 1.3) * rows_t[1] < rows_t[0] ? 256 : 128;
    }
    const int nx = cfg_[i].nx;
    const double narrow = (double)((nx + tn - 1) / tn) * tn;
    const double wide_cost = (fp32 ? 0.93 : 0.85) * (double)((nx + tw - 1) / tw) * tw;
    return wide_cost < narrow ? 256 : 128;
}

// the template key of an instance's launch group: form, equation, reconstruction, scheme
// (PRIMITIVE3 always on WENOEXP's 7-point geometry), flux and CTA width
long Engine::group_key(int i) const
{
    const int strict = cfg_[i].precision == WENOFV_FP64_STRICT;
    const int fp32 = cfg_[i].precision == WENOFV_FP32_BULK;
    const int sch = desc_[i].recon == 4 ? 2 : desc_[i].scheme;
    const int flx = desc_[i].eq_kind == WENOFV_EQ_LINEAR_ADV ? 0 : desc_[i].flux;
    const int wide = instance_nt(i) == 256;
    return ((long)wide << 40) | ((long)strict << 32) | ((long)fp32 << 24) | (desc_[i].eq_kind << 16) | (desc_[i].recon << 8) |
           (sch << 4) | flx;
}

namespace {
// grows a device array to at least n elements (capacity doubles); reports whether it moved
template <class T> int grow(T **p, int *cap, int n, bool *moved)
{
    if (n <= *cap) return WENOFV_OK;
    int c = std::max(64, *cap);
    while (c < n) c *= 2;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    WENOFV_CUDA(cudaMalloc(p, (size_t)c * sizeof(T)));
    *cap = c;
    *moved = true;
    return WENOFV_OK;
}
} // namespace

// One launch group per template key; work items are strips of TX columns by `seg` rows.  The
// grid is persistent (at most the resident CTA count; in slot mode always that count, so that
// a captured graph fits any later work list).  Work lists are rewritten in place; a new group
// or a buffer that had to grow drops the captured graphs.
int Engine::build_work()
{
    std::map<long, std::vector<int>> members;
    for (int i = 0; i < cap_; i++)
        if (live_[i]) members[group_key(i)].push_back(i);
    bool moved = false;
    if (!slot_mode) { // contexts and batches: the groups of the current instances only
        free_work();
        moved = true;
    }
    for (auto &kv : members) {
        bool found = false;
        for (Group &g : groups_) found = found || g.key == kv.first;
        if (found) continue;
        Group g;
        const int i = kv.second[0];
        g.key = kv.first;
        g.ns_strict = cfg_[i].precision == WENOFV_FP64_STRICT;
        g.fp32 = cfg_[i].precision == WENOFV_FP32_BULK;
        g.eq = desc_[i].eq_kind;
        g.recon = desc_[i].recon;
        g.scheme = desc_[i].recon == 4 ? 2 : desc_[i].scheme;
        g.flux = desc_[i].eq_kind == WENOFV_EQ_LINEAR_ADV ? 0 : desc_[i].flux;
        g.nt = instance_nt(i);
        WENOFV_CUDA(cudaMalloc(&g.d_counts, 4 * sizeof(int)));
        WENOFV_CUDA(cudaMalloc(&g.d_counter, sizeof(unsigned int)));
        WENOFV_CUDA(cudaMemsetAsync(g.d_counter, 0, sizeof(unsigned int), stream));
        WENOFV_CUDA(cudaStreamCreateWithFlags(&g.gstream, cudaStreamNonBlocking));
        WENOFV_CUDA(cudaEventCreateWithFlags(&g.joined, cudaEventDisableTiming));
        groups_.push_back(g);
        moved = true;
    }
    for (Group &g : groups_) {
        auto m = members.find(g.key);
        g.inst = m == members.end() ? std::vector<int>() : m->second;
        const int tx = g.ns_strict ? strict::stage_tx(g.eq, g.recon, g.fp32, g.scheme, g.nt) : fast::stage_tx(g.eq, g.recon, g.fp32, g.scheme, g.nt);
        const int bps = std::max(1, g.ns_strict ? strict::stage_blocks_per_sm(g.eq, g.recon, g.fp32, g.scheme, g.flux, g.nt)
                                                : fast::stage_blocks_per_sm(g.eq, g.recon, g.fp32, g.scheme, g.flux, g.nt));
        const int slots = sms_ * (ctas_per_sm_ > 0 ? std::min(ctas_per_sm_, bps) : bps);
        const int seg = item_rows(g.inst, tx, slots);
        std::vector<WorkItem> work;
        for (int i : g.inst)
            for (int j0 = 0; j0 < cfg_[i].ny; j0 += seg)
                for (int i0 = 0; i0 < cfg_[i].nx; i0 += tx)
                    work.push_back(WorkItem{i, i0, j0, std::min(cfg_[i].ny, j0 + seg)});
        g.nwork = (int)work.size();
        const int grid = slot_mode ? slots : std::max(1, std::min(g.nwork, slots));
        if (grid != g.grid) moved = true;
        g.grid = grid;
        int rc = grow(&g.d_work, &g.cap_work, std::max(1, g.nwork), &moved);
        if (!rc) rc = grow(&g.d_fin, &g.cap_fin, std::max(1, (int)g.inst.size()), &moved);
        if (rc) return rc;
        // pageable sources: each copy has read its source when it returns
        if (g.nwork) WENOFV_CUDA(cudaMemcpyAsync(g.d_work, work.data(), work.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, stream));
        if (!g.inst.empty())
            WENOFV_CUDA(cudaMemcpyAsync(g.d_fin, g.inst.data(), g.inst.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
        const int counts[2] = {g.nwork, (int)g.inst.size()};
        WENOFV_CUDA(cudaMemcpyAsync(g.d_counts, counts, sizeof counts, cudaMemcpyHostToDevice, stream));
    }
    if (moved) drop_graphs();
    return WENOFV_OK;
}

int Engine::push_state()
{
    WENOFV_CUDA(cudaMemcpyAsync(d_state_, h_state_, cap_ * sizeof(InstState), cudaMemcpyHostToDevice, stream));
    return WENOFV_OK;
}
int Engine::pull_state()
{
    WENOFV_CUDA(cudaMemcpyAsync(h_state_, d_state_, cap_ * sizeof(InstState), cudaMemcpyDeviceToHost, stream));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    return WENOFV_OK;
}

// the launch arguments every stage and CFL launch of a group shares
int Engine::group_launch(const Group &g, StageLaunch &L) const
{
    std::memset(&L, 0, sizeof L);
    L.inst = d_desc_;
    L.state = d_state_;
    L.work = g.d_work;
    L.nwork = g.nwork;
    L.fin_ids = g.d_fin;
    L.nfin = (int)g.inst.size();
    L.counts = g.d_counts;
    L.counter = g.d_counter;
    return WENOFV_OK;
}

// one stage of every group; inside a graph capture each group launches on its own branch
int Engine::launch_stage_all(int parity, int stage, double *rhs_out)
{
    const Roles ro = stage_roles(rk, parity, stage);
    for (Group &g : groups_) {
        StageLaunch L;
        group_launch(g, L);
        if (rhs_out) {
            L.bin = L.bun = L.bout = cur_;
            L.first_stage = 1;
            L.final_stage = 0;
            L.rhs_out = rhs_out;
        } else {
            L.bin = ro.bin; L.bun = ro.bun; L.bout = ro.bout;
            L.first_stage = stage == 0;
            L.final_stage = stage == stage_count(rk) - 1;
            L.rk1 = rk == 0;
            stage_coeffs(rk, stage, L.A, L.B, L.C);
        }
        cudaStream_t s = capturing_ ? g.gstream : stream;
        const int rc = g.ns_strict ? strict::launch_stage(g.eq, g.recon, g.fp32, g.scheme, g.flux, g.nt, L, g.grid, s)
                                   : fast::launch_stage(g.eq, g.recon, g.fp32, g.scheme, g.flux, g.nt, L, g.grid, s);
        if (rc) return cuda_fail((cudaError_t)rc, "stage kernel launch");
    }
    return WENOFV_OK;
}

int Engine::launch_cfl_all()
{
    for (Group &g : groups_) {
        StageLaunch L;
        group_launch(g, L);
        const int rc = g.ns_strict ? strict::launch_cfl(g.eq, g.recon, g.fp32, g.scheme, g.nt, L, g.grid, stream)
                                   : fast::launch_cfl(g.eq, g.recon, g.fp32, g.scheme, g.nt, L, g.grid, stream);
        if (rc) return cuda_fail((cudaError_t)rc, "cfl kernel launch");
    }
    return WENOFV_OK;
}

// the CFL pass and loop set-up (FIN_INIT) of the given slots only: per group, a work list
// of just their strips in the group's second pair of buffers
int Engine::start_many(const std::vector<int> &slots, const std::vector<double> &t_end, const std::vector<int64_t> &max_steps)
{
    WENOFV_CUDA(cudaSetDevice(device));
    int rc = ensure_work();
    if (rc) return rc;
    for (size_t k = 0; k < slots.size(); k++) {
        const int sl = slots[k];
        if (!live(sl)) { set_error("slot %d is not live", sl); return WENOFV_EINVAL; }
        h_state_[sl] = fresh_state(0);
        h_state_[sl].mode = MODE_ADVANCE;
        h_state_[sl].t_end = t_end[k];
        h_state_[sl].max_steps = max_steps[k] > 0 ? max_steps[k] : 0;
        WENOFV_CUDA(cudaMemcpyAsync(d_state_ + sl, &h_state_[sl], sizeof(InstState), cudaMemcpyHostToDevice, stream));
    }
    for (Group &g : groups_) {
        std::vector<int> fin;
        std::vector<WorkItem> work;
        const int tx = g.ns_strict ? strict::stage_tx(g.eq, g.recon, g.fp32, g.scheme, g.nt) : fast::stage_tx(g.eq, g.recon, g.fp32, g.scheme, g.nt);
        for (int sl : slots) {
            if (group_key(sl) != g.key) continue;
            fin.push_back(sl);
            for (int j0 = 0; j0 < cfg_[sl].ny; j0 += 32)
                for (int i0 = 0; i0 < cfg_[sl].nx; i0 += tx) work.push_back(WorkItem{sl, i0, j0, std::min(cfg_[sl].ny, j0 + 32)});
        }
        if (fin.empty()) continue;
        bool moved = false;
        rc = grow(&g.d_init_work, &g.cap_init_work, (int)work.size(), &moved);
        if (!rc) rc = grow(&g.d_init_fin, &g.cap_init_fin, (int)fin.size(), &moved);
        if (rc) return rc;
        WENOFV_CUDA(cudaMemcpyAsync(g.d_init_work, work.data(), work.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, stream));
        WENOFV_CUDA(cudaMemcpyAsync(g.d_init_fin, fin.data(), fin.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
        StageLaunch L;
        group_launch(g, L);
        L.work = g.d_init_work;
        L.nwork = (int)work.size();
        L.fin_ids = g.d_init_fin;
        L.nfin = (int)fin.size();
        L.counts = nullptr;
        const int grid = std::max(1, std::min(L.nwork, g.grid));
        const int lrc = g.ns_strict ? strict::launch_cfl(g.eq, g.recon, g.fp32, g.scheme, g.nt, L, grid, stream)
                                    : fast::launch_cfl(g.eq, g.recon, g.fp32, g.scheme, g.nt, L, grid, stream);
        if (lrc) return cuda_fail((cudaError_t)lrc, "cfl kernel launch");
    }
    return WENOFV_OK;
}

static void to_pitch(const double *U, int layout, int nv, int nx, int ny, int pitch, double *dst)
{
    for (int v = 0; v < nv; v++)
        for (int j = 0; j < ny; j++) {
            double *row = dst + ((size_t)v * ny + j) * pitch;
            if (layout == WENOFV_LAYOUT_SOA) {
                std::memcpy(row, U + ((size_t)v * ny + j) * nx, nx * sizeof(double));
            } else {
                for (int i = 0; i < nx; i++) row[i] = U[((size_t)i * ny + j) * nv + v];
            }
            for (int i = nx; i < pitch; i++) row[i] = 0.0;
        }
}
static void from_pitch(const double *src, int layout, int nv, int nx, int ny, int pitch, double *U)
{
    for (int v = 0; v < nv; v++)
        for (int j = 0; j < ny; j++) {
            const double *row = src + ((size_t)v * ny + j) * pitch;
            if (layout == WENOFV_LAYOUT_SOA) std::memcpy(U + ((size_t)v * ny + j) * nx, row, nx * sizeof(double));
            else
                for (int i = 0; i < nx; i++) U[((size_t)i * ny + j) * nv + v] = row[i];
        }
}

// pinned staging for the layouts that need a host-side repack, allocated on first use
int Engine::ensure_stage(size_t bytes)
{
    if (bytes <= h_stage_bytes_) return WENOFV_OK;
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    if (h_stage_) cudaFreeHost(h_stage_);
    h_stage_ = nullptr;
    h_stage_bytes_ = 0;
    WENOFV_CUDA(cudaMallocHost(&h_stage_, bytes));
    h_stage_bytes_ = bytes;
    return WENOFV_OK;
}

int Engine::upload(int i, const double *U, int layout)
{
    if (!live(i) || !U) { set_error("bad instance index or null array"); return WENOFV_EINVAL; }
    if (layout != WENOFV_LAYOUT_SOA && layout != WENOFV_LAYOUT_REF_AOS) { set_error("unknown layout"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    const InstDesc &d = desc_[i];
    const int nv = nvar_of(d.eq_kind);
    const int b = slot_mode ? 0 : cur_;
    if (layout == WENOFV_LAYOUT_SOA) {
        // one strided copy straight from the caller's array (the pitch padding is never read);
        // from pinned memory this is a single DMA without a host-side repack
        WENOFV_CUDA(cudaMemcpy2DAsync(d.buf[b], (size_t)d.pitch * sizeof(double), U, (size_t)d.nx * sizeof(double),
                                      (size_t)d.nx * sizeof(double), (size_t)nv * d.ny, cudaMemcpyHostToDevice, stream));
        WENOFV_CUDA(cudaStreamSynchronize(stream));
        return WENOFV_OK;
    }
    const int src = ensure_stage((size_t)nv * d.ny * d.pitch * sizeof(double));
    if (src) return src;
    WENOFV_CUDA(cudaStreamSynchronize(stream)); // the staging buffer may still feed a copy
    to_pitch(U, layout, nv, d.nx, d.ny, d.pitch, h_stage_);
    WENOFV_CUDA(cudaMemcpyAsync(d.buf[b], h_stage_, (size_t)nv * d.ny * d.pitch * sizeof(double), cudaMemcpyHostToDevice, stream));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    return WENOFV_OK;
}

int Engine::download(int i, double *U, int layout)
{
    if (!live(i) || !U) { set_error("bad instance index or null array"); return WENOFV_EINVAL; }
    if (layout != WENOFV_LAYOUT_SOA && layout != WENOFV_LAYOUT_REF_AOS) { set_error("unknown layout"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    const InstDesc &d = desc_[i];
    const int nv = nvar_of(d.eq_kind);
    const int b = slot_mode ? h_state_[i].cur_buf : cur_;
    if (layout == WENOFV_LAYOUT_SOA) {
        WENOFV_CUDA(cudaMemcpy2DAsync(U, (size_t)d.nx * sizeof(double), d.buf[b], (size_t)d.pitch * sizeof(double),
                                      (size_t)d.nx * sizeof(double), (size_t)nv * d.ny, cudaMemcpyDeviceToHost, stream));
        WENOFV_CUDA(cudaStreamSynchronize(stream));
        return WENOFV_OK;
    }
    const int src = ensure_stage((size_t)nv * d.ny * d.pitch * sizeof(double));
    if (src) return src;
    WENOFV_CUDA(cudaMemcpyAsync(h_stage_, d.buf[b], (size_t)nv * d.ny * d.pitch * sizeof(double), cudaMemcpyDeviceToHost, stream));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    from_pitch(h_stage_, layout, nv, d.nx, d.ny, d.pitch, U);
    return WENOFV_OK;
}

int Engine::theta_flags(int i, unsigned char *out, int layout)
{
    if (!live(i) || !out) { set_error("bad instance index or null array"); return WENOFV_EINVAL; }
    if (layout != WENOFV_LAYOUT_SOA && layout != WENOFV_LAYOUT_REF_AOS) { set_error("unknown layout"); return WENOFV_EINVAL; }
    const int nx = cfg_[i].nx, ny = cfg_[i].ny;
    if (!dtheta_[i]) { // no limiter: the record stays 0, as the reference's is never set
        std::memset(out, 0, (size_t)nx * ny);
        return WENOFV_OK;
    }
    WENOFV_CUDA(cudaSetDevice(device));
    std::vector<unsigned char> tmp;
    unsigned char *dst = out;
    if (layout == WENOFV_LAYOUT_REF_AOS) {
        tmp.resize((size_t)nx * ny);
        dst = tmp.data();
    }
    WENOFV_CUDA(cudaMemcpyAsync(dst, dtheta_[i], (size_t)nx * ny, cudaMemcpyDeviceToHost, stream));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    if (layout == WENOFV_LAYOUT_REF_AOS)
        for (int x = 0; x < nx; x++)
            for (int y = 0; y < ny; y++) out[(size_t)x * ny + y] = tmp[(size_t)y * nx + x];
    return WENOFV_OK;
}

// The current state is copied on the compute stream into a snapshot buffer (device to
// device, ~10 us for a 1024^2 two-phase state), then read back into pinned staging on a copy
// stream, so the host-bound copy overlaps whatever the compute stream does next.
// snapshot_wait touches only the snapshot's own members (events, staging, caller's array),
// so a worker thread may wait for it while the owning thread keeps stepping the context.
int Engine::snapshot_begin(int i, double *host, int layout)
{
    if (!live(i) || !host) { set_error("bad instance index or null array"); return WENOFV_EINVAL; }
    if (layout != WENOFV_LAYOUT_SOA && layout != WENOFV_LAYOUT_REF_AOS) { set_error("unknown layout"); return WENOFV_EINVAL; }
    if (snap_pending_) { set_error("a snapshot is in flight: call wenofv_snapshot_wait first"); return WENOFV_EBUSY; }
    WENOFV_CUDA(cudaSetDevice(device));
    const InstDesc &d = desc_[i];
    const size_t bytes = (size_t)nvar_of(d.eq_kind) * d.ny * d.pitch * sizeof(double);
    if (!copy_stream_) {
        WENOFV_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
        WENOFV_CUDA(cudaEventCreateWithFlags(&snap_ready_, cudaEventDisableTiming));
        WENOFV_CUDA(cudaEventCreateWithFlags(&snap_done_, cudaEventDisableTiming));
    }
    if (bytes > snap_bytes_) {
        WENOFV_CUDA(cudaStreamSynchronize(stream));
        WENOFV_CUDA(cudaStreamSynchronize(copy_stream_));
        cudaFree(d_snap_);
        if (h_snap_) cudaFreeHost(h_snap_);
        d_snap_ = nullptr;
        h_snap_ = nullptr;
        snap_bytes_ = 0;
        WENOFV_CUDA(cudaMalloc(&d_snap_, bytes));
        WENOFV_CUDA(cudaMallocHost(&h_snap_, bytes));
        snap_bytes_ = bytes;
    }
    const int b = slot_mode ? h_state_[i].cur_buf : cur_;
    WENOFV_CUDA(cudaMemcpyAsync(d_snap_, d.buf[b], bytes, cudaMemcpyDeviceToDevice, stream));
    WENOFV_CUDA(cudaEventRecord(snap_ready_, stream));
    WENOFV_CUDA(cudaStreamWaitEvent(copy_stream_, snap_ready_, 0));
    WENOFV_CUDA(cudaMemcpyAsync(h_snap_, d_snap_, bytes, cudaMemcpyDeviceToHost, copy_stream_));
    WENOFV_CUDA(cudaEventRecord(snap_done_, copy_stream_));
    snap_host_ = host;
    snap_layout_ = layout;
    snap_nv_ = nvar_of(d.eq_kind);
    snap_nx_ = d.nx;
    snap_ny_ = d.ny;
    snap_pitch_ = d.pitch;
    snap_pending_ = true;
    return WENOFV_OK;
}

int Engine::snapshot_wait()
{
    if (!snap_pending_) return WENOFV_OK;
    WENOFV_CUDA(cudaSetDevice(device));
    snap_pending_ = false;
    WENOFV_CUDA(cudaEventSynchronize(snap_done_));
    from_pitch(h_snap_, snap_layout_, snap_nv_, snap_nx_, snap_ny_, snap_pitch_, snap_host_);
    return WENOFV_OK;
}

namespace {
struct Range { // one NVTX range for the lifetime of the object
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
};
} // namespace

int Engine::compute_dt(double *dt_out)
{
    Range nvtx_range("wenofv::compute_dt");
    WENOFV_CUDA(cudaSetDevice(device));
    for (int i = 0; i < n; i++) h_state_[i] = fresh_state(cur_);
    int rc = push_state();
    if (!rc) rc = launch_cfl_all();
    if (!rc) rc = pull_state();
    if (rc) return rc;
    int bad = 0;
    for (int i = 0; i < n; i++) {
        dt_out[i] = h_state_[i].dtcfl;
        if (h_state_[i].flags & WENOFV_FLAG_NAN_DT) bad = 1;
    }
    if (bad) { set_error("NaN in the CFL time step"); return WENOFV_ENUMERIC; }
    return WENOFV_OK;
}

int Engine::step(double dt)
{
    Range nvtx_range("wenofv::step");
    if (const int fr = check_frames()) return fr;
    WENOFV_CUDA(cudaSetDevice(device));
    for (int i = 0; i < n; i++) {
        h_state_[i] = fresh_state(cur_);
        h_state_[i].dt = dt;
    }
    int rc = push_state();
    if (rc) return rc;
    const int parity = cur_ == 0 ? 0 : 1;
    for (int s = 0; s < stage_count(rk) && !rc; s++) rc = launch_stage_all(parity, s, nullptr);
    if (rc) return rc;
    cur_ = end_buffer(rk, parity);
    return WENOFV_OK;
}

int Engine::rhs(double *out, int layout)
{
    Range nvtx_range("wenofv::rhs");
    if (n != 1) { set_error("rhs is defined for a single instance"); return WENOFV_EINVAL; }
    if (const int fr = check_frames()) return fr;
    WENOFV_CUDA(cudaSetDevice(device));
    const InstDesc &d = desc_[0];
    const int nv = nvar_of(d.eq_kind);
    const size_t bytes = (size_t)nv * d.ny * d.pitch * sizeof(double);
    if (!d_rhs_) WENOFV_CUDA(cudaMalloc(&d_rhs_, bytes));
    h_state_[0] = fresh_state(cur_);
    int rc = push_state();
    if (!rc) rc = launch_stage_all(0, 0, d_rhs_);
    if (rc) return rc;
    if (layout == WENOFV_LAYOUT_SOA) {
        WENOFV_CUDA(cudaMemcpy2DAsync(out, (size_t)d.nx * sizeof(double), d_rhs_, (size_t)d.pitch * sizeof(double),
                                      (size_t)d.nx * sizeof(double), (size_t)nv * d.ny, cudaMemcpyDeviceToHost, stream));
        WENOFV_CUDA(cudaStreamSynchronize(stream));
        return WENOFV_OK;
    }
    rc = ensure_stage(bytes);
    if (rc) return rc;
    WENOFV_CUDA(cudaMemcpyAsync(h_stage_, d_rhs_, bytes, cudaMemcpyDeviceToHost, stream));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    from_pitch(h_stage_, layout, nv, d.nx, d.ny, d.pitch, out);
    return WENOFV_OK;
}

void Engine::drop_graphs()
{
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    for (auto &kv : graph_defs_) cudaGraphDestroy(kv.second);
    graphs_.clear();
    graph_defs_.clear();
}

// K captured pairs of RK steps (buffer roles return to buffer 0 after each pair).  The
// launch groups are independent of each other (their instances never share memory), so
// each group's chain of stages is its own branch of the graph, forked from and joined back
// into the context's stream: groups of different template keys run side by side.
int Engine::run_graph(int K)
{
    Range nvtx_range("wenofv::run_graph");
    auto it = graphs_.find(K);
    if (it == graphs_.end()) {
        if (!fork_) WENOFV_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
        cudaGraph_t g;
        WENOFV_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        int rc = 0;
        cudaError_t e = cudaEventRecord(fork_, stream);
        for (Group &gr : groups_)
            if (e == cudaSuccess) e = cudaStreamWaitEvent(gr.gstream, fork_, 0);
        capturing_ = true;
        for (int k = 0; k < K && !rc && e == cudaSuccess; k++)
            for (int p = 0; p < 2 && !rc; p++)
                for (int s = 0; s < stage_count(rk) && !rc; s++) rc = launch_stage_all(p, s, nullptr);
        capturing_ = false;
        for (Group &gr : groups_) {
            if (e == cudaSuccess) e = cudaEventRecord(gr.joined, gr.gstream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, gr.joined, 0);
        }
        const cudaError_t ee = cudaStreamEndCapture(stream, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return cuda_fail(e, "graph fork/join");
        if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
        cudaGraphExec_t ex;
        WENOFV_CUDA(cudaGraphInstantiate(&ex, g, 0));
        graph_defs_[K] = g;
        graphs_[K] = ex;
        it = graphs_.find(K);
    }
    WENOFV_CUDA(cudaGraphLaunch(it->second, stream));
    return WENOFV_OK;
}

int Engine::normalize_buffers()
{
    for (int i = 0; i < n; i++) {
        const int cb = h_state_[i].cur_buf;
        if (cb == 0) continue;
        const InstDesc &d = desc_[i];
        const size_t bytes = (size_t)nvar_of(d.eq_kind) * d.ny * d.pitch * sizeof(double);
        WENOFV_CUDA(cudaMemcpyAsync(d.buf[0], d.buf[cb], bytes, cudaMemcpyDeviceToDevice, stream));
        h_state_[i].cur_buf = 0;
    }
    cur_ = 0;
    return push_state();
}

int Engine::advance(const double *t0, const double *t_end, int64_t max_steps, double *t_out, int64_t *nsteps)
{
    Range nvtx_range("wenofv::advance");
    if (const int fr = check_frames()) return fr;
    WENOFV_CUDA(cudaSetDevice(device));
    // every instance's state into buffer 0, where the captured step pairs start
    for (int i = 0; i < n; i++) h_state_[i].cur_buf = cur_;
    int rc = normalize_buffers();
    if (rc) return rc;
    for (int i = 0; i < n; i++) {
        h_state_[i] = fresh_state(0);
        h_state_[i].mode = MODE_ADVANCE;
        h_state_[i].now = t0 ? t0[i] : 0.0;
        h_state_[i].t_end = t_end[i];
        h_state_[i].max_steps = max_steps > 0 ? max_steps : 0;
    }
    rc = push_state();
    if (!rc) rc = launch_cfl_all();
    if (!rc) rc = pull_state();
    if (rc) return rc;
    for (;;) {
        // pairs of steps for the next graph launch: from the slowest instance's estimate
        double most = 0.0;
        bool all_done = true;
        for (int i = 0; i < n; i++) {
            const InstState &s = h_state_[i];
            if (s.done) continue;
            all_done = false;
            double left = s.dt > 0 ? std::ceil((s.t_end - s.now) / s.dt) : 1.0;
            if (s.max_steps > 0) left = std::min(left, (double)(s.max_steps - s.nsteps));
            most = std::max(most, left);
        }
        if (all_done) break;
        int K = (int)std::ceil(most / 2.0);
        K = std::max(1, std::min(K, 64));
        // round K up to a power of two so that few distinct graphs are instantiated
        int Kp = 1;
        while (Kp < K) Kp <<= 1;
        rc = run_graph(Kp);
        if (!rc) rc = pull_state();
        if (rc) return rc;
    }
    uint32_t flags = 0;
    for (int i = 0; i < n; i++) {
        if (t_out) t_out[i] = h_state_[i].now;
        if (nsteps) nsteps[i] = h_state_[i].nsteps;
        flags |= h_state_[i].flags;
    }
    rc = normalize_buffers();
    if (rc) return rc;
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    if (flags & (WENOFV_FLAG_NAN_DT | WENOFV_FLAG_BAD_THETA | WENOFV_FLAG_NAN_FLUX | WENOFV_FLAG_NAN_STATE | WENOFV_FLAG_BOUNDS)) {
        set_error("numerical error flags 0x%x", flags);
        return WENOFV_ENUMERIC;
    }
    return WENOFV_OK;
}

int Engine::status(int i, uint32_t *flags, int64_t *cell)
{
    if (!live(i)) { set_error("bad instance index"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    const int rc = pull_state();
    if (rc) return rc;
    if (flags) *flags = h_state_[i].flags;
    if (cell) *cell = h_state_[i].bad_cell;
    return WENOFV_OK;
}

int Engine::set_tiling(int rows, int ctas)
{
    WENOFV_CUDA(cudaSetDevice(device));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    rows_per_item_ = rows;
    ctas_per_sm_ = ctas;
    work_dirty_ = true;
    return ensure_work();
}

int Engine::set_threads(int nt)
{
    if (nt != 0 && nt != 128 && nt != 256) { set_error("threads per CTA must be 0 (automatic), 128 or 256"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    nt_override_ = nt;
    work_dirty_ = true;
    return ensure_work();
}

void Engine::tiling(int *rows, int *ctas, int *nt) const
{
    if (rows) *rows = rows_per_item_;
    if (ctas) *ctas = ctas_per_sm_;
    if (nt) *nt = nt_override_;
}

int Engine::device_state(int i, double **U, int *pitch)
{
    if (!live(i)) { set_error("bad instance index"); return WENOFV_EINVAL; }
    if (U) *U = desc_[i].buf[cur_];
    if (pitch) *pitch = desc_[i].pitch;
    return WENOFV_OK;
}

namespace {
// what autotune borrows, given back on every return path: the saved copies of the states,
// the two timing events, and (when the search stops early) the tiling and the loop state
struct TuneScope {
    Engine &e;
    std::vector<double *> saved;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rows0, ctas0, nt0, cur0;
    std::vector<InstState> state0;
    bool done = false;
    TuneScope(Engine &eng, int rows, int ctas, int nt, int cur, const InstState *st, int cap)
        : e(eng), saved(eng.n, nullptr), rows0(rows), ctas0(ctas), nt0(nt), cur0(cur), state0(st, st + cap) {}
    ~TuneScope()
    {
        if (!done) { // an error path: the caller's tiling, buffer and loop state as they were
            cudaStreamSynchronize(e.stream);
            e.restore_after_tune(rows0, ctas0, nt0, cur0, state0.data(), saved);
        }
        for (double *p : saved) cudaFree(p);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        (void)cudaGetLastError();
    }
};
} // namespace

// puts the saved states back into the current buffer and restores tiling and loop state
void Engine::restore_after_tune(int rows, int ctas, int nt, int cur, const InstState *st, const std::vector<double *> &saved)
{
    cur_ = cur;
    for (int i = 0; i < n && i < (int)saved.size(); i++) {
        if (!saved[i]) continue;
        const InstDesc &d = desc_[i];
        const size_t bytes = (size_t)nvar_of(d.eq_kind) * d.ny * d.pitch * sizeof(double);
        cudaMemcpyAsync(d.buf[cur_], saved[i], bytes, cudaMemcpyDeviceToDevice, stream);
    }
    std::memcpy(h_state_, st, cap_ * sizeof(InstState));
    push_state();
    cudaStreamSynchronize(stream);
    rows_per_item_ = rows;
    ctas_per_sm_ = ctas;
    nt_override_ = nt;
    work_dirty_ = true;
    ensure_work();
}

// Times candidate tilings (CTA width x rows per work item x resident CTAs per SM) with manual
// steps on the current state and keeps the fastest: one warm-up step, then TUNE_SAMPLES timed
// steps per candidate, ranked by the median.  The CTA width candidates are the per-instance
// width model (0) and, where any instance has the 256-thread kernel, 128 and 256 for all.  The
// states, the buffer rotation and the loop state (status flags included) are put back
// afterwards, and on any error.
int Engine::autotune(int *rows_out, int *ctas_out, double *best_ms)
{
    constexpr int TUNE_SAMPLES = 3;
    WENOFV_CUDA(cudaSetDevice(device));
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    int rc = pull_state();
    if (rc) return rc;
    TuneScope T(*this, rows_per_item_, ctas_per_sm_, nt_override_, cur_, h_state_, cap_);
    for (int i = 0; i < n; i++) {
        const InstDesc &d = desc_[i];
        const size_t bytes = (size_t)nvar_of(d.eq_kind) * d.ny * d.pitch * sizeof(double);
        WENOFV_CUDA(cudaMalloc(&T.saved[i], bytes));
        WENOFV_CUDA(cudaMemcpyAsync(T.saved[i], d.buf[cur_], bytes, cudaMemcpyDeviceToDevice, stream));
    }
    WENOFV_CUDA(cudaEventCreate(&T.e0));
    WENOFV_CUDA(cudaEventCreate(&T.e1));
    double dt = 0.0;
    {
        std::vector<double> dts(n);
        rc = compute_dt(dts.data());
        if (rc) return rc;
        dt = *std::min_element(dts.begin(), dts.end()) * 0.5;
    }
    bool any_wide = false;
    for (int i = 0; i < n; i++) {
        const int st = cfg_[i].precision == WENOFV_FP64_STRICT;
        any_wide = any_wide || (st ? strict::stage_wide(desc_[i].eq_kind, desc_[i].recon) : fast::stage_wide(desc_[i].eq_kind, desc_[i].recon));
    }
    std::vector<int> nt_c = {0};
    if (any_wide) { nt_c.push_back(128); nt_c.push_back(256); }
    const int rows_c[] = {0, 16, 32, 64}; // 0: the automatic rows per item (item_rows)
    const int ctas_c[] = {0, 2};
    double best = 1e30;
    int br = 32, bc = 0, bn = 0;
    for (int w : nt_c)
        for (int r : rows_c)
        for (int c : ctas_c) {
            nt_override_ = w;
            rc = set_tiling(r, c);
            if (!rc) rc = step(dt); // warm-up
            if (rc) return rc;
            float ms[TUNE_SAMPLES];
            for (int k = 0; k < TUNE_SAMPLES; k++) {
                WENOFV_CUDA(cudaEventRecord(T.e0, stream));
                rc = step(dt);
                if (rc) return rc;
                WENOFV_CUDA(cudaEventRecord(T.e1, stream));
                WENOFV_CUDA(cudaEventSynchronize(T.e1));
                WENOFV_CUDA(cudaEventElapsedTime(&ms[k], T.e0, T.e1));
            }
            std::sort(ms, ms + TUNE_SAMPLES);
            const double med = ms[TUNE_SAMPLES / 2];
            if (med < best) { best = med; br = r; bc = c; bn = w; }
        }
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    T.done = true;
    restore_after_tune(br, bc, bn, T.cur0, T.state0.data(), T.saved);
    if (const cudaError_t e = cudaGetLastError()) return cuda_fail(e, "autotune restore");
    if (rows_out) *rows_out = br;
    if (ctas_out) *ctas_out = bc;
    if (best_ms) *best_ms = best / stage_count(rk); // per stage launch
    return WENOFV_OK;
}

} // namespace wenofv
