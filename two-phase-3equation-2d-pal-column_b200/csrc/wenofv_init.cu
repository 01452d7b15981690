// wenofv_init.cu -- device-side initial averages and accuracy norms of the reference's
// periodic two-phase test cases.
//
// initializeAve (src/WENOFV.cpp:232-279) averages getU0 (include/Equations.hpp:979-1002)
// over every cell with the 4x4 Gauss-Legendre rule, and outputAccuracy (:3152-3251) reports
// L_inf, L1 and L2 of the volume fraction against the translated initial data. Here both run
// as one thread per cell on the GPU, so that a solve of a reference test case needs no host
// initialisation. The cell bounds follow the reference's slab grid generator
// (src/WENOFV.cpp:89-123), as the C ABI's grid metric does. The arithmetic is the
// reference's, compiled without contraction. The device sin/exp/pow differ from the host
// C library's by at most a few ulp, so the averages agree with the host-side ones to
// ~1e-15 relative, not bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "wenofv_engine.h"

namespace wenofv {
namespace {

struct InitArgs {
    int testcase, nx, ny, slabs, pitch, nv;
    double u0, v0, epsa, t;
    double xl, xr, yl, yr, dX, dY;
    double rho10, rho20, c1, c2, preb;
    double *U;
};

__constant__ double kGLegX[4] = {-0.861136311594052575223946488893, -0.339981043584856264802665759103,
                                 0.339981043584856264802665759103, 0.861136311594052575223946488893};
__constant__ double kGLegW[4] = {0.347854845137453857373063949222, 0.652145154862546142626936050778,
                                 0.652145154862546142626936050778, 0.347854845137453857373063949222};

__device__ double wrap(double v, double lo, double hi)
{
    while (v >= hi) v -= hi - lo;
    while (v < lo) v += hi - lo;
    return v;
}

// initial volume fraction of phase 1 (include/Equations.hpp:514-515, :538-549, :651-660)
__device__ double z1_0(const InitArgs &a, double x, double y)
{
    if (a.testcase == 0) return a.epsa + (1 - 2 * a.epsa) * pow(sin(2.0 * M_PI * x), 2);
    if (a.testcase == 1) {
        x = wrap(x, -1.0, 1.0);
        y = wrap(y, -1.0, 1.0);
        const double r = sqrt(x * x + y * y);
        return (1 - 2 * a.epsa) * exp(-pow(r, 2) / pow(0.2, 2)) + a.epsa;
    }
    const double r = (a.xr - a.xl) / 10.0;
    const double xc = (a.xl + a.xr) / 2.0, yc = (a.yl + a.yr) / 2.0;
    return (fabs(x - xc) < r && fabs(y - yc) < r) ? 1 - a.epsa : a.epsa;
}

// getU0 with uniform phase pressures g_preb
__device__ void u0_at(const InitArgs &a, double x, double y, double *U)
{
    const double z_1 = z1_0(a, x, y), z_2 = 1.0 - z_1;
    const double rho10 = (a.preb - a.preb) / pow(a.c1, 2) + a.rho10;
    const double rho20 = (a.preb - a.preb) / pow(a.c2, 2) + a.rho20;
    const double z1rho1 = rho10 * z_1, z2rho2 = rho20 * z_2;
    const double rho = z1rho1 + z2rho2;
    U[0] = z1rho1;
    U[1] = z2rho2;
    U[2] = rho * a.u0;
    U[3] = rho * a.v0;
}

__global__ void init_kernel(const InitArgs a)
{
    const long long ncell = (long long)a.nx * a.ny;
    const int per = a.nx / a.slabs, G = 3;
    const double ghostY = (a.yl + 0 * a.ny * a.dY) - a.dY * G;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ncell; k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / a.nx), i = (int)(k - (long long)j * a.nx);
        const int slab = i / per, ei = i - slab * per + G;
        const double ghostX = (a.xl + slab * per * a.dX) - a.dX * G;
        const double xl = ghostX + ei * a.dX, xr = ghostX + (ei + 1) * a.dX;
        const double yl = ghostY + (j + G) * a.dY, yr = ghostY + (j + G + 1) * a.dY;
        const double xc = (xl + xr) / 2, xd = xr - xl, yc = (yl + yr) / 2, yd = yr - yl;
        double acc[4] = {0.0, 0.0, 0.0, 0.0}, U[4];
        for (int p = 0; p < 4; p++)
            for (int q = 0; q < 4; q++) {
                const double gx = xc + 0.5 * xd * kGLegX[p], gy = yc + 0.5 * yd * kGLegX[q];
                const double wx = 0.5 * xd * kGLegW[p], wy = 0.5 * yd * kGLegW[q];
                u0_at(a, gx, gy, U);
                for (int r = 0; r < 4; r++) acc[r] += U[r] * wx * wy;
            }
        const double area = xd * yd;
        const size_t plane = (size_t)a.ny * a.pitch;
        for (int r = 0; r < 4; r++) a.U[r * plane + (size_t)j * a.pitch + i] = acc[r] / area;
    }
}

// outputAccuracy: per cell |exact average of z1 - getVolumeFrac(U)| on the reference's
// single-rank world grid, reduced per block into (sum, sum of squares, max)
__global__ void accuracy_kernel(const InitArgs a, double *partial)
{
    __shared__ double s1[256], s2[256], sm[256];
    const long long ncell = (long long)a.nx * a.ny;
    const int G = 3;
    const double c1_2 = a.c1 * a.c1, c2_2 = a.c2 * a.c2, q = a.rho20 * c2_2 - a.rho10 * c1_2;
    double e1 = 0.0, e2 = 0.0, em = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < ncell; k += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(k / a.nx), i = (int)(k - (long long)j * a.nx);
        const double xl = a.xl - G * a.dX + (i + G) * a.dX, xr = a.xl - G * a.dX + (i + G + 1) * a.dX;
        const double yl = a.yl - G * a.dY + (j + G) * a.dY, yr = a.yl - G * a.dY + (j + G + 1) * a.dY;
        const double xc = (xl + xr) / 2, yc = (yl + yr) / 2;
        double ex = 0.0;
        for (int p = 0; p < 4; p++)
            for (int qq = 0; qq < 4; qq++) {
                const double gx = xc + 0.5 * a.dX * kGLegX[p], gy = yc + 0.5 * a.dY * kGLegX[qq];
                const double wx = 0.5 * a.dX * kGLegW[p], wy = 0.5 * a.dY * kGLegW[qq];
                ex += z1_0(a, gx - a.u0 * a.t, gy - a.v0 * a.t) * wx * wy / a.dX / a.dY;
            }
        const size_t plane = (size_t)a.ny * a.pitch, o = (size_t)j * a.pitch + i;
        const double z1rho1 = a.U[o], z2rho2 = a.U[plane + o];
        const double qs = z2rho2 * c2_2 - z1rho1 * c1_2;
        const double r = ((q - qs) + sqrt((q - qs) * (q - qs) + 4.0 * z1rho1 * c1_2 * z2rho2 * c2_2)) / (2.0 * z2rho2 * c2_2);
        const double err = fabs(ex - r / (1.0 + r));
        e1 += err;
        e2 += err * err;
        em = fmax(em, err);
    }
    s1[threadIdx.x] = e1;
    s2[threadIdx.x] = e2;
    sm[threadIdx.x] = em;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s1[threadIdx.x] += s1[threadIdx.x + w];
            s2[threadIdx.x] += s2[threadIdx.x + w];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[3 * blockIdx.x + 0] = s1[0];
        partial[3 * blockIdx.x + 1] = s2[0];
        partial[3 * blockIdx.x + 2] = sm[0];
    }
}

int args_of(const wenofv_config &c, const wenofv_eq_params &e, const InstDesc &d, const wenofv_testcase *tc, double *U,
            InitArgs *a)
{
    if (!tc || tc->testcase < 0 || tc->testcase > 2) {
        set_error("test case must be 0 (SMOOTH), 1 (VORTEX) or 2 (SHARP)");
        return WENOFV_EINVAL;
    }
    if (e.eq_kind != WENOFV_EQ_TWO_PHASE) { set_error("the test cases are two-phase"); return WENOFV_EINVAL; }
    *a = InitArgs{};
    a->testcase = tc->testcase;
    a->u0 = tc->u0; a->v0 = tc->v0; a->epsa = tc->epsa;
    a->nx = c.nx; a->ny = c.ny; a->slabs = c.ref_slabs > 0 ? c.ref_slabs : 1; a->pitch = d.pitch; a->nv = 4;
    a->xl = c.xl; a->xr = c.xr; a->yl = c.yl; a->yr = c.yr;
    a->dX = (c.xr - c.xl) / c.nx; a->dY = (c.yr - c.yl) / c.ny;
    a->rho10 = e.rho10; a->rho20 = e.rho20; a->c1 = e.sound1; a->c2 = e.sound2; a->preb = e.preb;
    a->U = U;
    return WENOFV_OK;
}

} // namespace

int Engine::init_testcase(int i, const wenofv_testcase *tc)
{
    if (!live(i)) { set_error("bad instance index"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    const InstDesc &d = desc_[i];
    InitArgs a;
    const int b = slot_mode ? h_state_[i].cur_buf : cur_;
    int rc = args_of(cfg_[i], eq_[i], d, tc, d.buf[b], &a);
    if (rc) return rc;
    init_kernel<<<sms_ * 4, 128, 0, stream>>>(a);
    WENOFV_CUDA(cudaGetLastError());
    WENOFV_CUDA(cudaStreamSynchronize(stream));
    return WENOFV_OK;
}

int Engine::accuracy(int i, const wenofv_testcase *tc, double t, double *norms)
{
    if (!live(i) || !norms) { set_error("bad instance index or null output"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    const InstDesc &d = desc_[i];
    InitArgs a;
    const int b = slot_mode ? h_state_[i].cur_buf : cur_;
    int rc = args_of(cfg_[i], eq_[i], d, tc, d.buf[b], &a);
    if (rc) return rc;
    a.t = t;
    const int blocks = sms_ * 2;
    double *partial = nullptr;
    WENOFV_CUDA(cudaMalloc(&partial, 3 * sizeof(double) * blocks));
    accuracy_kernel<<<blocks, 256, 0, stream>>>(a, partial);
    cudaError_t e = cudaGetLastError();
    std::vector<double> h(3 * (size_t)blocks);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(partial);
    if (e != cudaSuccess) return cuda_fail(e, "accuracy kernel");
    double s1 = 0.0, s2 = 0.0, m = 0.0;
    for (int k = 0; k < blocks; k++) {
        s1 += h[3 * k];
        s2 += h[3 * k + 1];
        m = h[3 * k + 2] > m ? h[3 * k + 2] : m;
    }
    const double n = (double)cfg_[i].nx * cfg_[i].ny;
    norms[0] = m;
    norms[1] = s1 / n;
    norms[2] = std::sqrt(s2 / n);
    return WENOFV_OK;
}

} // namespace wenofv
