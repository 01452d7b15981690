// wenofv_kernels.cu -- instantiations and host launchers of the stage, CFL and probe
// kernels.  Built twice into the library: -DWENOFV_STRICT=1 -fmad=false (namespace
// wenofv::strict, the reference's FP64 operation order) and -DWENOFV_STRICT=0 (namespace
// wenofv::fast, FP64 with contraction and the FP32-bulk form).
#include <cuda_runtime.h>

#include <algorithm>

#include "wenofv_stage.cuh"

namespace wenofv {
#if WENOFV_STRICT
namespace strict {
#else
namespace fast {
#endif

#if WENOFV_STRICT
#define WENOFV_HAS_FP32 0
#else
#define WENOFV_HAS_FP32 1
#endif

// whether (eq, recon) has the 256-thread stage kernel too (StageWide)
int stage_wide(int eq, int recon) { (void)recon; return eq != EQ_LINEAR_ADV && eq != EQ_TWO_PHASE_SG; }
static_assert(StageWide<EQ_TWO_PHASE, 1, double>::value && StageWide<EQ_TWO_PHASE, 4, double>::value &&
                  StageWide<EQ_TWO_PHASE, 1, float>::value && !StageWide<EQ_LINEAR_ADV, 0, double>::value &&
                  !StageWide<EQ_TWO_PHASE_SG, 1, double>::value && StageWide<EQ_EULER, 0, float>::value,
              "stage_wide mirrors StageWide");
// the width a launch runs: 256 where asked for and available, else 128
static int width_of(int eq, int recon, int nt) { return (nt == 256 && stage_wide(eq, recon)) ? 256 : 128; }

// strip width of the work items: 5-point stencils (H = 2) or WENOEXP's 7-point ones (H = 3)
template <int NT> static int tx_of(int eq, int scheme)
{
    if (scheme == 2) return eq == EQ_LINEAR_ADV ? StageGeom<EQ_LINEAR_ADV, 3, NT>::TX : StageGeom<EQ_TWO_PHASE, 3, NT>::TX;
    return eq == EQ_LINEAR_ADV ? StageGeom<EQ_LINEAR_ADV, 2, NT>::TX : StageGeom<EQ_TWO_PHASE, 2, NT>::TX;
}
int stage_tx(int eq, int recon, int fp32, int scheme, int nt)
{
    (void)fp32;
    return width_of(eq, recon, nt) == 256 ? tx_of<256>(eq, scheme) : tx_of<128>(eq, scheme);
}

template <int EQ, int RECON, class R, int SCH, int FLX, int NT> static const void *stage_fn()
{
    return (const void *)stage_kernel<EQ, RECON, R, SCH, FLX, NT>;
}
// the scheme and flux of a launch group as template arguments (scalar advection has one flux)
// (WENOEXP, scheme 2, only in FP64)
template <int EQ, int RECON, class R, int NT> static const void *pick_sf(int scheme, int flux)
{
    if constexpr (NT == 256 && !StageWide<EQ, RECON, R>::value) {
        return nullptr;
    } else if constexpr (RECON == 4) { // PRIMITIVE3: FP64, on the 7-point geometry (scheme 2) whatever SCHEME is
        if constexpr (EQ == EQ_TWO_PHASE && sizeof(R) == sizeof(double)) {
            if (scheme != 2) return nullptr;
            return flux ? stage_fn<EQ, RECON, R, 2, 1, NT>() : stage_fn<EQ, RECON, R, 2, 0, NT>();
        } else {
            return nullptr;
        }
    } else {
        if constexpr (sizeof(R) == sizeof(double)) {
            if (scheme == 2) {
                if (EQ == EQ_LINEAR_ADV) return stage_fn<EQ, RECON, R, 2, 0, NT>();
                return flux ? stage_fn<EQ, RECON, R, 2, 1, NT>() : stage_fn<EQ, RECON, R, 2, 0, NT>();
            }
        } else {
            if (scheme == 2) return nullptr;
        }
        if (EQ == EQ_LINEAR_ADV) return scheme ? stage_fn<EQ, RECON, R, 1, 0, NT>() : stage_fn<EQ, RECON, R, 0, 0, NT>();
        if (scheme) return flux ? stage_fn<EQ, RECON, R, 1, 1, NT>() : stage_fn<EQ, RECON, R, 1, 0, NT>();
        return flux ? stage_fn<EQ, RECON, R, 0, 1, NT>() : stage_fn<EQ, RECON, R, 0, 0, NT>();
    }
}
template <class R, int NT> static const void *pick_eq(int eq, int recon, int scheme, int flux)
{
    switch (eq) {
    case EQ_TWO_PHASE:
        return recon == 1 ? pick_sf<EQ_TWO_PHASE, 1, R, NT>(scheme, flux) : recon == 2 ? pick_sf<EQ_TWO_PHASE, 2, R, NT>(scheme, flux)
             : recon == 3 ? pick_sf<EQ_TWO_PHASE, 3, R, NT>(scheme, flux) : recon == 4 ? pick_sf<EQ_TWO_PHASE, 4, R, NT>(scheme, flux)
                          : pick_sf<EQ_TWO_PHASE, 0, R, NT>(scheme, flux);
    case EQ_EULER: return recon ? pick_sf<EQ_EULER, 1, R, NT>(scheme, flux) : pick_sf<EQ_EULER, 0, R, NT>(scheme, flux);
    case EQ_LINEAR_ADV: return pick_sf<EQ_LINEAR_ADV, 0, R, NT>(scheme, flux);
    case EQ_TWO_PHASE_SG: // FP64, conservative or characteristic reconstruction
        if constexpr (sizeof(R) == sizeof(double)) {
            if (recon > 1) return nullptr;
            return recon ? pick_sf<EQ_TWO_PHASE_SG, 1, R, NT>(scheme, flux) : pick_sf<EQ_TWO_PHASE_SG, 0, R, NT>(scheme, flux);
        } else {
            return nullptr;
        }
    default: return nullptr;
    }
}

static const void *pick_stage(int eq, int recon, int fp32, int scheme, int flux, int nt)
{
    if (scheme < 0 || scheme > 2 || flux < 0 || flux > 1) return nullptr;
    const bool wide = width_of(eq, recon, nt) == 256;
#if WENOFV_HAS_FP32
    if (fp32) return wide ? pick_eq<float, 256>(eq, recon, scheme, flux) : pick_eq<float, 128>(eq, recon, scheme, flux);
#else
    if (fp32) return nullptr;
#endif
    return wide ? pick_eq<double, 256>(eq, recon, scheme, flux) : pick_eq<double, 128>(eq, recon, scheme, flux);
}

// dynamic shared memory of a stage kernel: its StageSmem block, then the primitive ring of
// the primitive reconstructions (the same size for both geometries)
template <int H, int NT> static int smem_of(int eq)
{
    return eq == EQ_TWO_PHASE      ? StageSmemBytes<EQ_TWO_PHASE, H, NT>::value
         : eq == EQ_EULER          ? StageSmemBytes<EQ_EULER, H, NT>::value
         : eq == EQ_TWO_PHASE_SG   ? StageSmemBytes<EQ_TWO_PHASE_SG, H, NT>::value
                                   : StageSmemBytes<EQ_LINEAR_ADV, H, NT>::value;
}
static int stage_dyn_bytes(int eq, int recon, int scheme, int nt)
{
    static_assert(StageDynSmem<EQ_TWO_PHASE, 2, 2, 256>::value == StageDynSmem<EQ_TWO_PHASE, 2, 3, 256>::value, "ring size");
    const bool wide = width_of(eq, recon, nt) == 256;
    const int ring = (eq == EQ_TWO_PHASE && recon >= 2)
                         ? (wide ? StageDynSmem<EQ_TWO_PHASE, 2, 2, 256>::value : StageDynSmem<EQ_TWO_PHASE, 2, 2, 128>::value)
                         : 0;
    const int base = wide ? (scheme == 2 ? smem_of<3, 256>(eq) : smem_of<2, 256>(eq))
                          : (scheme == 2 ? smem_of<3, 128>(eq) : smem_of<2, 128>(eq));
    return base + ring;
}
// dynamic shared memory past the default 48 KB needs an opt-in (not during a stream
// capture, where the engine has already done it through stage_blocks_per_sm)
static cudaError_t allow_dyn(const void *fn, int dyn)
{
    if (dyn <= 0) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
}

int launch_stage(int eq, int recon, int fp32, int scheme, int flux, int nt, const StageLaunch &L, int grid, void *stream)
{
    const void *fn = pick_stage(eq, recon, fp32, scheme, flux, nt);
    if (!fn) return (int)cudaErrorInvalidValue;
    const int dyn = stage_dyn_bytes(eq, recon, scheme, nt);
    if (dyn > 48 * 1024) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaError_t e = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
        if (e != cudaSuccess) return (int)e;
        if (cs == cudaStreamCaptureStatusNone && (e = allow_dyn(fn, dyn)) != cudaSuccess) return (int)e;
    }
    void *args[] = {(void *)&L};
    return (int)cudaLaunchKernel(fn, dim3(grid), dim3(width_of(eq, recon, nt)), args, (size_t)dyn, (cudaStream_t)stream);
}

static const void *cfl_fn(int eq)
{
    return eq == EQ_TWO_PHASE      ? (const void *)cfl_kernel<EQ_TWO_PHASE>
         : eq == EQ_EULER          ? (const void *)cfl_kernel<EQ_EULER>
         : eq == EQ_TWO_PHASE_SG   ? (const void *)cfl_kernel<EQ_TWO_PHASE_SG>
                                   : (const void *)cfl_kernel<EQ_LINEAR_ADV>;
}

// the CFL pass over the work items of a launch group, whose strips are those of its stage kernel
int launch_cfl(int eq, int recon, int fp32, int scheme, int nt, const StageLaunch &L, int grid, void *stream)
{
    StageLaunch Lc = L;
    Lc.tx = stage_tx(eq, recon, fp32, scheme, nt);
    void *args[] = {(void *)&Lc};
    return (int)cudaLaunchKernel(cfl_fn(eq), dim3(grid), dim3(CFL_NT), args, 0, (cudaStream_t)stream);
}

int stage_blocks_per_sm(int eq, int recon, int fp32, int scheme, int flux, int nt)
{
    const void *fn = pick_stage(eq, recon, fp32, scheme, flux, nt);
    if (!fn) return 0;
    const int dyn = stage_dyn_bytes(eq, recon, scheme, nt);
    if (dyn > 48 * 1024 && allow_dyn(fn, dyn) != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, width_of(eq, recon, nt), (size_t)dyn) != cudaSuccess) return 0;
    return n;
}

// ---- probes: the pointwise kernels on arrays (test hooks) -----------------------------
template <class R> __global__ void probe_weno_kernel(int scheme, const double *st, int n, double *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    Weno5<R> W;
    W.init(scheme, (R)st[5 * k], (R)st[5 * k + 1], (R)st[5 * k + 2], (R)st[5 * k + 3], (R)st[5 * k + 4]);
    out[4 * k + 0] = (double)W.template eval<0>();
    out[4 * k + 1] = (double)W.template eval<1>();
    out[4 * k + 2] = (double)W.template eval<2>();
    out[4 * k + 3] = (double)W.template eval<3>();
}

__global__ void probe_weno_exp_kernel(const double *st, int n, double dx4, double *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    WenoExp W;
    W.init(st + 7 * k, dx4);
    W.eval4(out + 4 * k);
}

template <int EQ, class R>
__global__ void probe_riemann_kernel(EqParams P, int flux, const double *UL, const double *UR, int n, int xdir, double *F)
{
    constexpr int NV = EqTraits<EQ>::NV;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double l[NV], r[NV], f[NV];
    for (int v = 0; v < NV; v++) { l[v] = UL[NV * k + v]; r[v] = UR[NV * k + v]; }
    riemann<EQ, R>(P, flux, l, r, f, xdir != 0);
    for (int v = 0; v < NV; v++) F[NV * k + v] = f[v];
}

template <int EQ, class R>
__global__ void probe_eigen_kernel(EqParams P, const double *U, int n, int xdir, double *Lm, double *Rm)
{
    constexpr int NV = EqTraits<EQ>::NV;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double u[NV];
    for (int v = 0; v < NV; v++) u[v] = U[NV * k + v];
    for (int row = 0; row < NV; row++) {
        R lr[NV], rr[NV];
        eigen_rows<EQ, R>(P, u, xdir != 0, row, lr, rr);
        for (int j = 0; j < NV; j++) {
            Lm[16 * k + row * NV + j] = (double)lr[j];
            Rm[16 * k + row * NV + j] = (double)rr[j];
        }
    }
}

int probe_weno(int scheme, int fp32, const double *d_st, int n, double *d_out, void *stream)
{
    const int b = 128, g = (n + b - 1) / b;
    if (n <= 0) return 0;
#if WENOFV_HAS_FP32
    if (fp32) probe_weno_kernel<float><<<g, b, 0, (cudaStream_t)stream>>>(scheme, d_st, n, d_out);
    else
#endif
        probe_weno_kernel<double><<<g, b, 0, (cudaStream_t)stream>>>(scheme, d_st, n, d_out);
    return (int)cudaGetLastError();
}

int probe_weno_exp(const double *d_st, int n, double dx4, double *d_out, void *stream)
{
    const int b = 128, g = (n + b - 1) / b;
    if (n <= 0) return 0;
    probe_weno_exp_kernel<<<g, b, 0, (cudaStream_t)stream>>>(d_st, n, dx4, d_out);
    return (int)cudaGetLastError();
}

int probe_riemann(const EqParams &P, int flux, int fp32, const double *d_UL, const double *d_UR, int n, int xdir, double *d_F, void *stream)
{
    const int b = 128, g = (n + b - 1) / b;
    if (n <= 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (P.kind == EQ_TWO_PHASE_SG) { // FP64 only
        if (fp32) return (int)cudaErrorInvalidValue;
        probe_riemann_kernel<EQ_TWO_PHASE_SG, double><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
        return (int)cudaGetLastError();
    }
#if WENOFV_HAS_FP32
    if (fp32) {
        if (P.kind == EQ_TWO_PHASE) probe_riemann_kernel<EQ_TWO_PHASE, float><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
        else if (P.kind == EQ_EULER) probe_riemann_kernel<EQ_EULER, float><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
        else probe_riemann_kernel<EQ_LINEAR_ADV, float><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
        return (int)cudaGetLastError();
    }
#endif
    if (P.kind == EQ_TWO_PHASE) probe_riemann_kernel<EQ_TWO_PHASE, double><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
    else if (P.kind == EQ_EULER) probe_riemann_kernel<EQ_EULER, double><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
    else probe_riemann_kernel<EQ_LINEAR_ADV, double><<<g, b, 0, s>>>(P, flux, d_UL, d_UR, n, xdir, d_F);
    return (int)cudaGetLastError();
}

int probe_eigen(const EqParams &P, int fp32, const double *d_U, int n, int xdir, double *d_L, double *d_R, void *stream)
{
    const int b = 128, g = (n + b - 1) / b;
    if (n <= 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (P.kind == EQ_TWO_PHASE_SG) { // FP64 only
        if (fp32) return (int)cudaErrorInvalidValue;
        probe_eigen_kernel<EQ_TWO_PHASE_SG, double><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
        return (int)cudaGetLastError();
    }
#if WENOFV_HAS_FP32
    if (fp32) {
        if (P.kind == EQ_TWO_PHASE) probe_eigen_kernel<EQ_TWO_PHASE, float><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
        else if (P.kind == EQ_EULER) probe_eigen_kernel<EQ_EULER, float><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
        else probe_eigen_kernel<EQ_LINEAR_ADV, float><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
        return (int)cudaGetLastError();
    }
#endif
    if (P.kind == EQ_TWO_PHASE) probe_eigen_kernel<EQ_TWO_PHASE, double><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
    else if (P.kind == EQ_EULER) probe_eigen_kernel<EQ_EULER, double><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
    else probe_eigen_kernel<EQ_LINEAR_ADV, double><<<g, b, 0, s>>>(P, d_U, n, xdir, d_L, d_R);
    return (int)cudaGetLastError();
}

#if !WENOFV_STRICT
// FMA throughput of the CUDA-core pipe: independent FMA chains per thread, enough warps to
// fill every SM (the denominator of the stage kernel's compute roofline).
template <class R> __global__ void __launch_bounds__(256) fma_peak_kernel(R *out, int iters, R a, R b)
{
    R x0 = (R)threadIdx.x, x1 = x0 + R(1), x2 = x0 + R(2), x3 = x0 + R(3), x4 = x0 + R(4), x5 = x0 + R(5), x6 = x0 + R(6), x7 = x0 + R(7);
#pragma unroll 1
    for (int k = 0; k < iters; k++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    const R s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == R(-1.2345)) out[threadIdx.x] = s; // keeps the chains alive
}

int fma_peak(int fp32, double *tflops, void *stream)
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    void *out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(double)) != cudaSuccess) return (int)cudaErrorMemoryAllocation;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 8, iters = 2048;
    double best = 0.0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0, s);
        if (fp32) fma_peak_kernel<float><<<blocks, 256, 0, s>>>((float *)out, iters, 0.999999f, 1e-7f);
        else fma_peak_kernel<double><<<blocks, 256, 0, s>>>((double *)out, iters, 0.9999999, 1e-9);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
        if (rep > 0 && ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return (int)cudaGetLastError();
}
#endif

} // namespace strict / fast
} // namespace wenofv
