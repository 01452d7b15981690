// wenofv_capi.cu -- the extern "C" entry points declared in include/wenofv.h (contexts,
// batches and device probes; the serving entry points are in wenofv_server.cu).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "wenofv_engine.h"

using namespace wenofv;

struct wenofv_ctx {
    Engine eng;
};
struct wenofv_batch {
    Engine eng;
};

extern "C" {

int wenofv_abi_version(void) { return WENOFV_ABI_VERSION; }

const char *wenofv_strerror(int code)
{
    switch (code) {
    case WENOFV_OK: return "ok";
    case WENOFV_EINVAL: return "invalid argument";
    case WENOFV_ENOMEM: return "out of device memory or over the HBM budget";
    case WENOFV_ENUMERIC: return "numerical error (NaN time step, NaN flux or illegal limiter theta)";
    case WENOFV_ETIMEDOUT: return "timed out";
    case WENOFV_ECUDA: return "CUDA runtime error";
    case WENOFV_ENOTSUP: return "not supported";
    case WENOFV_EBUSY: return "busy";
    case WENOFV_ENOTFOUND: return "not found";
    default: return "unknown status";
    }
}

const char *wenofv_last_error(void) { return last_error_text(); }

// config/settings.cfg as shipped: SMOOTH 100x100, RK3, CFL 0.5, WENO-Z, no limiter, LLF,
// characteristic reconstruction; the SMOOTH domain [0,1]^2, periodic (include/Equations.hpp:491-496)
void wenofv_default_config(wenofv_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->nx = 100; c->ny = 100;
    c->xl = 0.0; c->xr = 1.0; c->yl = 0.0; c->yr = 1.0;
    c->bc = WENOFV_BC_PERIOD;
    c->rk_method = 2;
    c->cfl = 0.5;
    c->scheme = 1;
    c->pp_limiter = 0;
    c->riemann_flux = 0;
    c->reconstruction = 1;
    c->ref_slabs = 0;
    c->precision = WENOFV_FP64;
    c->device = 0;
}

int wenofv_create(const wenofv_config *cfg, const wenofv_eq_params *eq, wenofv_ctx **out)
{
    if (!out) { set_error("null output pointer"); return WENOFV_EINVAL; }
    *out = nullptr;
    const int v = validate(cfg, eq);
    if (v) return v;
    wenofv_ctx *c = new (std::nothrow) wenofv_ctx;
    if (!c) { set_error("host allocation failed"); return WENOFV_ENOMEM; }
    c->eng.theta_record = true;
    c->eng.solo = true;
    const int rc = c->eng.init(1, cfg, eq);
    if (rc) { delete c; return rc; }
    *out = c;
    return WENOFV_OK;
}

void wenofv_destroy(wenofv_ctx *ctx) { delete ctx; }

int wenofv_init_testcase(wenofv_ctx *ctx, const wenofv_testcase *tc)
{
    if (!ctx || !tc) { set_error("null argument"); return WENOFV_EINVAL; }
    return ctx->eng.init_testcase(0, tc);
}
int wenofv_accuracy(wenofv_ctx *ctx, const wenofv_testcase *tc, double t, double norms[3])
{
    if (!ctx || !tc || !norms) { set_error("null argument"); return WENOFV_EINVAL; }
    return ctx->eng.accuracy(0, tc, t, norms);
}

int wenofv_upload(wenofv_ctx *ctx, const double *U, int layout)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.upload(0, U, layout);
}
int wenofv_set_frame(wenofv_ctx *ctx, const double *frame)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.set_frame(0, frame);
}
int wenofv_download(wenofv_ctx *ctx, double *U, int layout)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.download(0, U, layout);
}
int wenofv_theta_flags(wenofv_ctx *ctx, uint8_t *out, int layout)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.theta_flags(0, out, layout);
}

int wenofv_snapshot_begin(wenofv_ctx *ctx, double *host, int layout)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.snapshot_begin(0, host, layout);
}

int wenofv_snapshot_wait(wenofv_ctx *ctx)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.snapshot_wait();
}

int wenofv_compute_dt(wenofv_ctx *ctx, double *dt)
{
    if (!ctx || !dt) { set_error("null argument"); return WENOFV_EINVAL; }
    return ctx->eng.compute_dt(dt);
}
int wenofv_step(wenofv_ctx *ctx, double dt)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    if (!(dt >= 0.0)) { set_error("dt must be a non-negative number"); return WENOFV_EINVAL; }
    return ctx->eng.step(dt);
}
int wenofv_rhs(wenofv_ctx *ctx, double *rhs, int layout)
{
    if (!ctx || !rhs) { set_error("null argument"); return WENOFV_EINVAL; }
    return ctx->eng.rhs(rhs, layout);
}
int wenofv_advance(wenofv_ctx *ctx, double t_now, double t_end, int64_t max_steps, double *t_out, int64_t *nsteps)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.advance(&t_now, &t_end, max_steps, t_out, nsteps);
}
int wenofv_status(wenofv_ctx *ctx, uint32_t *flags, int64_t *first_cell)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.status(0, flags, first_cell);
}
int wenofv_synchronize(wenofv_ctx *ctx)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(ctx->eng.device));
    WENOFV_CUDA(cudaStreamSynchronize(ctx->eng.stream));
    return WENOFV_OK;
}
void *wenofv_stream(wenofv_ctx *ctx) { return ctx ? (void *)ctx->eng.stream : nullptr; }
int wenofv_device_state(wenofv_ctx *ctx, double **U, int *pitch)
{
    if (!ctx) { set_error("null context"); return WENOFV_EINVAL; }
    return ctx->eng.device_state(0, U, pitch);
}

// ---- batch --------------------------------------------------------------------------------
int wenofv_batch_create(int n, const wenofv_config *cfgs, const wenofv_eq_params *eqs, wenofv_batch **out)
{
    if (!out || !cfgs || !eqs) { set_error("null argument"); return WENOFV_EINVAL; }
    *out = nullptr;
    wenofv_batch *b = new (std::nothrow) wenofv_batch;
    if (!b) { set_error("host allocation failed"); return WENOFV_ENOMEM; }
    const int rc = b->eng.init(n, cfgs, eqs);
    if (rc) { delete b; return rc; }
    *out = b;
    return WENOFV_OK;
}
void wenofv_batch_destroy(wenofv_batch *b) { delete b; }
int wenofv_batch_upload(wenofv_batch *b, int i, const double *U, int layout)
{
    if (!b) { set_error("null batch"); return WENOFV_EINVAL; }
    return b->eng.upload(i, U, layout);
}
int wenofv_batch_set_frame(wenofv_batch *b, int i, const double *frame)
{
    if (!b) { set_error("null batch"); return WENOFV_EINVAL; }
    return b->eng.set_frame(i, frame);
}
int wenofv_batch_download(wenofv_batch *b, int i, double *U, int layout)
{
    if (!b) { set_error("null batch"); return WENOFV_EINVAL; }
    return b->eng.download(i, U, layout);
}
int wenofv_batch_advance(wenofv_batch *b, const double *t_end, int64_t max_steps, int64_t *nsteps)
{
    if (!b || !t_end) { set_error("null argument"); return WENOFV_EINVAL; }
    return b->eng.advance(nullptr, t_end, max_steps, nullptr, nsteps);
}
int wenofv_batch_set_tiling(wenofv_batch *b, int rows_per_item, int ctas_per_sm)
{
    if (!b || rows_per_item < 0 || ctas_per_sm < 0) { set_error("bad argument"); return WENOFV_EINVAL; }
    return b->eng.set_tiling(rows_per_item, ctas_per_sm);
}
int wenofv_batch_stream(wenofv_batch *b, void **stream)
{
    if (!b || !stream) { set_error("null argument"); return WENOFV_EINVAL; }
    *stream = (void *)b->eng.stream;
    return WENOFV_OK;
}
int wenofv_batch_set_threads(wenofv_batch *b, int threads_per_cta)
{
    if (!b) { set_error("null batch"); return WENOFV_EINVAL; }
    return b->eng.set_threads(threads_per_cta);
}

int wenofv_batch_tiling(wenofv_batch *b, int *rows_per_item, int *ctas_per_sm, int *threads_per_cta)
{
    if (!b) { set_error("null batch"); return WENOFV_EINVAL; }
    b->eng.tiling(rows_per_item, ctas_per_sm, threads_per_cta);
    return WENOFV_OK;
}

int wenofv_batch_autotune(wenofv_batch *b, int *rows_per_item, int *ctas_per_sm, double *best_ms)
{
    if (!b) { set_error("null batch"); return WENOFV_EINVAL; }
    return b->eng.autotune(rows_per_item, ctas_per_sm, best_ms);
}

// ---- probes ---------------------------------------------------------------------------------
static EqParams to_params(const wenofv_eq_params *e)
{
    return eq_params_of(*e);
}

struct DevBufs {
    std::vector<void *> p;
    ~DevBufs() { for (void *q : p) cudaFree(q); }
    double *alloc(size_t n)
    {
        void *q = nullptr;
        if (cudaMalloc(&q, n * sizeof(double) + 8) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (double *)q;
    }
};

int wenofv_probe_weno(int scheme, int precision, const double *stencils, int n, double *out, int device)
{
    if (n < 0 || (n > 0 && (!stencils || !out))) { set_error("bad arguments"); return WENOFV_EINVAL; }
    if (n == 0) return WENOFV_OK;
    WENOFV_CUDA(cudaSetDevice(device));
    DevBufs B;
    double *s = B.alloc((size_t)5 * n), *o = B.alloc((size_t)4 * n);
    if (!s || !o) { set_error("device allocation failed"); return WENOFV_ENOMEM; }
    WENOFV_CUDA(cudaMemcpy(s, stencils, (size_t)5 * n * sizeof(double), cudaMemcpyHostToDevice));
    const int rc = precision == WENOFV_FP64_STRICT ? strict::probe_weno(scheme, 0, s, n, o, nullptr)
                                                   : fast::probe_weno(scheme, precision == WENOFV_FP32_BULK, s, n, o, nullptr);
    if (rc) return cuda_fail((cudaError_t)rc, "probe_weno");
    WENOFV_CUDA(cudaMemcpy(out, o, (size_t)4 * n * sizeof(double), cudaMemcpyDeviceToHost));
    return WENOFV_OK;
}

int wenofv_probe_weno_exp(int precision, const double *stencils, int n, double dx, double *out, int device)
{
    if (n < 0 || (n > 0 && (!stencils || !out)) || precision == WENOFV_FP32_BULK) {
        set_error("bad arguments (WENOEXP has no FP32 form)");
        return WENOFV_EINVAL;
    }
    if (n == 0) return WENOFV_OK;
    WENOFV_CUDA(cudaSetDevice(device));
    DevBufs B;
    double *s = B.alloc((size_t)7 * n), *o = B.alloc((size_t)4 * n);
    if (!s || !o) { set_error("device allocation failed"); return WENOFV_ENOMEM; }
    WENOFV_CUDA(cudaMemcpy(s, stencils, (size_t)7 * n * sizeof(double), cudaMemcpyHostToDevice));
    const double dx4 = std::pow(dx, 4); // as the engine forms it for a grid
    const int rc = precision == WENOFV_FP64_STRICT ? strict::probe_weno_exp(s, n, dx4, o, nullptr)
                                                   : fast::probe_weno_exp(s, n, dx4, o, nullptr);
    if (rc) return cuda_fail((cudaError_t)rc, "probe_weno_exp");
    WENOFV_CUDA(cudaMemcpy(out, o, (size_t)4 * n * sizeof(double), cudaMemcpyDeviceToHost));
    return WENOFV_OK;
}

int wenofv_probe_riemann(const wenofv_eq_params *eq, int flux, int precision, const double *UL, const double *UR, int n,
                         double nx, double ny, double *F, int device)
{
    if (!eq || n < 0 || (n > 0 && (!UL || !UR || !F))) { set_error("bad arguments"); return WENOFV_EINVAL; }
    if (!((nx == 1.0 && ny == 0.0) || (nx == 0.0 && ny == 1.0))) { set_error("normal must be (1,0) or (0,1)"); return WENOFV_EINVAL; }
    if (n == 0) return WENOFV_OK;
    WENOFV_CUDA(cudaSetDevice(device));
    const int nv = nvar_of(eq->eq_kind);
    DevBufs B;
    double *l = B.alloc((size_t)nv * n), *r = B.alloc((size_t)nv * n), *f = B.alloc((size_t)nv * n);
    if (!l || !r || !f) { set_error("device allocation failed"); return WENOFV_ENOMEM; }
    WENOFV_CUDA(cudaMemcpy(l, UL, (size_t)nv * n * sizeof(double), cudaMemcpyHostToDevice));
    WENOFV_CUDA(cudaMemcpy(r, UR, (size_t)nv * n * sizeof(double), cudaMemcpyHostToDevice));
    const EqParams P = to_params(eq);
    const int xdir = nx == 1.0;
    const int rc = precision == WENOFV_FP64_STRICT ? strict::probe_riemann(P, flux, 0, l, r, n, xdir, f, nullptr)
                                                   : fast::probe_riemann(P, flux, precision == WENOFV_FP32_BULK, l, r, n, xdir, f, nullptr);
    if (rc) return cuda_fail((cudaError_t)rc, "probe_riemann");
    WENOFV_CUDA(cudaMemcpy(F, f, (size_t)nv * n * sizeof(double), cudaMemcpyDeviceToHost));
    return WENOFV_OK;
}

int wenofv_probe_eigen(const wenofv_eq_params *eq, int precision, const double *U, int n, double nx, double ny, double *L,
                       double *R, int device)
{
    if (!eq || n < 0 || (n > 0 && (!U || !L || !R))) { set_error("bad arguments"); return WENOFV_EINVAL; }
    if (!((nx == 1.0 && ny == 0.0) || (nx == 0.0 && ny == 1.0))) { set_error("normal must be (1,0) or (0,1)"); return WENOFV_EINVAL; }
    if (n == 0) return WENOFV_OK;
    WENOFV_CUDA(cudaSetDevice(device));
    const int nv = nvar_of(eq->eq_kind);
    DevBufs B;
    double *u = B.alloc((size_t)nv * n), *l = B.alloc((size_t)16 * n), *r = B.alloc((size_t)16 * n);
    if (!u || !l || !r) { set_error("device allocation failed"); return WENOFV_ENOMEM; }
    WENOFV_CUDA(cudaMemcpy(u, U, (size_t)nv * n * sizeof(double), cudaMemcpyHostToDevice));
    WENOFV_CUDA(cudaMemset(l, 0, (size_t)16 * n * sizeof(double)));
    WENOFV_CUDA(cudaMemset(r, 0, (size_t)16 * n * sizeof(double)));
    const EqParams P = to_params(eq);
    const int xdir = nx == 1.0;
    const int rc = precision == WENOFV_FP64_STRICT ? strict::probe_eigen(P, 0, u, n, xdir, l, r, nullptr)
                                                   : fast::probe_eigen(P, precision == WENOFV_FP32_BULK, u, n, xdir, l, r, nullptr);
    if (rc) return cuda_fail((cudaError_t)rc, "probe_eigen");
    WENOFV_CUDA(cudaMemcpy(L, l, (size_t)16 * n * sizeof(double), cudaMemcpyDeviceToHost));
    WENOFV_CUDA(cudaMemcpy(R, r, (size_t)16 * n * sizeof(double), cudaMemcpyDeviceToHost));
    return WENOFV_OK;
}

int wenofv_probe_fma_peak(int precision, int device, double *tflops)
{
    if (!tflops) { set_error("null argument"); return WENOFV_EINVAL; }
    WENOFV_CUDA(cudaSetDevice(device));
    const int rc = fast::fma_peak(precision == WENOFV_FP32_BULK, tflops, nullptr);
    if (rc) return cuda_fail((cudaError_t)rc, "fma_peak");
    return WENOFV_OK;
}

} // extern "C"
