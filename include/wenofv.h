/*
 * wenofv.h -- C ABI of the B200 (sm_100a) WENOFV time-advance library (libwenofv_b200.so).
 *
 * The library replaces the hot path of the reference solver's CWENOFV class
 * (infinity-07/two-phase-3equation-2D-pal-column): the ghost-cell fill, the
 * dimension-by-dimension WENO-JS/WENO-Z/WENOEXP reconstruction at Gauss-Lobatto points, the
 * bound-preserving theta limiter, the LLF/HLLC Riemann fluxes with Gauss-Lobatto face
 * quadrature, the SSP-RK stage combination and the CFL max-wavespeed reduction.  The whole
 * domain stays resident in one GPU's HBM; the reference's 4-rank MPI x-slab
 * decomposition is not needed.
 *
 * Citations are path:line inside the reference project.  All entry points return a
 * WENOFV_* status (0 = success) and never exit, trap or block on stdin.  One context is
 * used by one host thread at a time; contexts are independent of each other.  Calls are
 * asynchronous on the context's CUDA stream except where a function reads a result back
 * (download, compute_dt, rhs, advance, status), which synchronise that stream.
 */
#ifndef WENOFV_H
#define WENOFV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WENOFV_ABI_VERSION 2 /* 2: wenofv_eq_params gained the stiffened-gas fields */

/* status codes (the reference prints, waits on std::cin and exits instead:
 * src/WENOFV.cpp:34-38, :521-531, :1927-1932, :2287-2292; include/Equations.hpp:345-359) */
enum {
    WENOFV_OK = 0,
    WENOFV_EINVAL = 1,    /* invalid configuration or argument */
    WENOFV_ENOMEM = 2,    /* device allocation failed or the HBM budget is exceeded */
    WENOFV_ENUMERIC = 3,  /* NaN time step, NaN flux or illegal limiter theta (see status) */
    WENOFV_ETIMEDOUT = 4, /* a bounded wait ran out */
    WENOFV_ECUDA = 5,     /* CUDA runtime error (message in wenofv_last_error) */
    WENOFV_ENOTSUP = 6,   /* option combination not supported */
    WENOFV_EBUSY = 7,     /* request still running (serving API) */
    WENOFV_ENOTFOUND = 8  /* unknown request id (serving API) */
};

/* equation kinds; TWO_PHASE is TwoPhaseEquation (include/Equations.hpp:52-1044) */
enum { WENOFV_EQ_TWO_PHASE = 0, WENOFV_EQ_LINEAR_ADV = 1, WENOFV_EQ_EULER = 2, WENOFV_EQ_TWO_PHASE_SG = 3 };
/* boundary kinds with the numbers of BOUNDARYTYPE (include/Equations.hpp:25-32): PERIOD;
 * NEUMANN ("reflective, slip") and FREESLIP: mirror ghost cells with the normal momentum
 * negated; NOSLIP: mirror ghost cells with both momenta negated.  The reference declares the
 * wall kinds but does not implement them (src/WENOFV.cpp:2254-2292), so their ghost rule is
 * this library's.  NEUMANN2 ("boundary from the initial data", also declared and not
 * implemented) takes every ghost cell from a fixed frame of averages that the caller sets
 * with wenofv_set_frame / wenofv_batch_set_frame before the first step; the serving API and
 * wenofv_step_noalloc reject it.  OUTFLOW (zero-gradient) has no counterpart in the
 * reference. */
enum {
    WENOFV_BC_PERIOD = 0,
    WENOFV_BC_NEUMANN = 1,
    WENOFV_BC_NOSLIP = 2,
    WENOFV_BC_NEUMANN2 = 3,
    WENOFV_BC_FREESLIP = 4,
    WENOFV_BC_OUTFLOW = 5
};
/* arithmetic forms */
enum {
    WENOFV_FP64 = 0,        /* FP64 with fused multiply-add contraction */
    WENOFV_FP64_STRICT = 1, /* FP64 in the reference's operation order, no contraction */
    WENOFV_FP32_BULK = 2    /* FP32 reconstruction/flux; FP64 pressure recovery, theta and
                               RK accumulation */
};
/* host array layouts for upload/download/rhs */
enum {
    WENOFV_LAYOUT_SOA = 0,    /* U[v][j][i], i (x) fastest */
    WENOFV_LAYOUT_REF_AOS = 1 /* U[i][j][v]: the order of the reference's m_Uh[ei][ej].vector[r]
                                 over interior cells (include/WENOFV.hpp:171) */
};
/* bits of the device status word */
enum {
    WENOFV_FLAG_NAN_DT = 1u,     /* NaN in the CFL time step (src/WENOFV.cpp:502-531) */
    WENOFV_FLAG_BAD_THETA = 2u,  /* limiter theta outside [0,1] (src/WENOFV.cpp:1927-1932) */
    WENOFV_FLAG_NAN_FLUX = 4u,   /* NaN Riemann flux (include/Equations.hpp:345-359) */
    WENOFV_FLAG_NAN_STATE = 8u,  /* NaN in an updated cell average */
    WENOFV_FLAG_BOUNDS = 16u     /* an index outside its buffer (self-checking build only) */
};

/* Equation parameters.  Field order and meaning of rho10..preb follow TwoPhaseEquation's
 * g_rho10, g_rho20, g_sound1, g_sound2, g_preb (include/Equations.hpp:67-69); the linear EOS
 * p_k = sound_k^2 (rho_k - rho_k0) drops preb exactly as getPressure does (:112-116). */
typedef struct {
    int eq_kind;
    double rho10, rho20, sound1, sound2, preb;
    double gamma;        /* Euler ratio of specific heats */
    double adv_u, adv_v; /* linear advection velocity */
    /* WENOFV_EQ_TWO_PHASE_SG (an extension): stiffened-gas phases on their isentropes through
     * (preb, rho10) and (preb, rho20), p_k = (preb + pinf_k) (rho_k / rho_k0)^gamma_k - pinf_k;
     * sound1/sound2 are ignored (the library uses the linearised c_k^2 = gamma_k (preb +
     * pinf_k) / rho_k0 for the first guess of the pressure equilibrium); FP64 forms and
     * RECONSTRUCTIONTYPE 0-1 only */
    double gamma1, pinf1, gamma2, pinf2;
    /* gravity of the two-phase kinds, assembleSourceTerm's g_g0 (src/WENOFV.cpp:1831-1872):
     * the y-momentum RHS gains -rho g; 9.81 for DAMBREAK/RTI, 2 pi for STANDING_WAVE, 0 for
     * the periodic test cases */
    double gravity;
} wenofv_eq_params;

/* Solver options: the settings.cfg keys (config/settings.cfg:11-24, read at
 * src/WENOFV.cpp:43-62) plus the domain, boundary, grid metric, arithmetic form and device. */
typedef struct {
    int nx, ny;            /* ELEMNUMX, ELEMNUMY */
    double xl, xr, yl, yr; /* TwoPhaseEquation::xL, xR, yL, yR */
    int bc;                /* WENOFV_BC_* */
    int rk_method;         /* RKMETH: 0 RK1, 1 RK2, 2 RK3 */
    double cfl;            /* CFL */
    int scheme;            /* SCHEME: 0 WENO-JS, 1 WENO-Z, 2 WENOEXP (FP64 forms only) */
    int pp_limiter;        /* PPlimiter: 0 off, 1 on */
    int riemann_flux;      /* RIEMANNFLUX: 0 LLF, 1 HLLC */
    int reconstruction;    /* RECONSTRUCTIONTYPE: 0 conservative, 1 characteristic, 2 primitive
                              (z1, rho1, u, v), 3 primitive2 (z1, p, u, v), 4 primitive3 (z1 by
                              WENOEXP/THINC, p, u, v by WENO-Z whatever SCHEME is; FP64 forms
                              only); 2-4 for the two-phase model (src/WENOFV.cpp:884-1372);
                              5 (ThincOnlyForZ1, not dispatched by the reference) is not supported */
    int ref_slabs;         /* 0: uniform cell sizes; P > 0: cell sizes exactly as the
                              reference's P-slab grid generator rounds them (src/WENOFV.cpp:89-123) */
    int precision;         /* WENOFV_FP64, WENOFV_FP64_STRICT, WENOFV_FP32_BULK */
    int device;            /* CUDA device ordinal */
} wenofv_config;

typedef struct wenofv_ctx wenofv_ctx;

int wenofv_abi_version(void);
const char *wenofv_strerror(int code);
/* text of the last error on the calling thread (CUDA message or argument check) */
const char *wenofv_last_error(void);
/* fills *cfg with the reference's shipped settings.cfg defaults (config/settings.cfg) */
void wenofv_default_config(wenofv_config *cfg);

/* CWENOFV::initializeSolver (src/WENOFV.cpp:16-231): validate options, build the grid
 * metric and allocate the device state (three FP64 state buffers, the status block). */
int wenofv_create(const wenofv_config *cfg, const wenofv_eq_params *eq, wenofv_ctx **out);
/* releases every device allocation of the context */
void wenofv_destroy(wenofv_ctx *ctx);

/* writes the interior cell averages (CWENOFV::m_Uh after initializeAve, src/WENOFV.cpp:232-279) */
int wenofv_upload(wenofv_ctx *ctx, const double *U, int layout);
/* reads the interior cell averages (what getWorldUh gathers, src/WENOFV.cpp:2059-2117) */
int wenofv_download(wenofv_ctx *ctx, double *U, int layout);
/* NEUMANN2 only: the fixed ghost averages, host SoA [v][ny+8][nx+8] with cell (i, j) at
 * [v][j+4][i+4]; the entries of the interior are not read.  Copied synchronously, held for
 * every later stage.  Replaces the ghost fill of BOUNDARYTYPE NEUMANN2, which the reference
 * declares (include/Equations.hpp:30, set for ZALESAK at :696) but whose branch of
 * setBoundaryAverages2 (src/WENOFV.cpp:2254-2292) it never wrote. */
int wenofv_set_frame(wenofv_ctx *ctx, const double *frame);

/* CWENOFV::calculateDeltaT (src/WENOFV.cpp:474-540): min over cells of
 * CFL / (lambda_x/dx + lambda_y/dy), starting from 1.0; WENOFV_ENUMERIC on a NaN */
int wenofv_compute_dt(wenofv_ctx *ctx, double *dt);
/* CWENOFV::performTimeIntegration (src/WENOFV.cpp:541-566): one SSP-RK step with this dt */
int wenofv_step(wenofv_ctx *ctx, double dt);
/* CWENOFV::assembleRHS (src/WENOFV.cpp:568-615) of the current state, written to host rhs */
int wenofv_rhs(wenofv_ctx *ctx, double *rhs, int layout);
/* the stepping loop of CWENOFV::run towards one output time (src/WENOFV.cpp:318-354):
 * while |now - t_end| > 1e-10 { dt = min(calculateDeltaT, t_end - now); step; now += dt; }
 * The loop runs on the device in CUDA graphs; max_steps <= 0 means no limit. */
int wenofv_advance(wenofv_ctx *ctx, double t_now, double t_end, int64_t max_steps, double *t_out,
                   int64_t *nsteps);
/* device status word (WENOFV_FLAG_*) and the first offending cell (j*nx+i, -1 if none) */
int wenofv_status(wenofv_ctx *ctx, uint32_t *flags, int64_t *first_cell);
/* waits for all work queued on the context's stream */
int wenofv_synchronize(wenofv_ctx *ctx);
/* the context's cudaStream_t (for event timing by the caller) */
void *wenofv_stream(wenofv_ctx *ctx);
/* device pointer of the current interior state, SoA with row pitch *pitch doubles and
 * plane stride pitch*ny (valid until the next step) */
int wenofv_device_state(wenofv_ctx *ctx, double **U, int *pitch);
/* the per-cell record of useBoundPreservingLimiter (src/WENOFV.cpp:1906-1909), m_totalTheta
 * as getWorldTheta gathers it for the theta column of outputAve / outputSliceAve
 * (src/WENOFV.cpp:2587, :2725): out[cell] = 1 where the final RK stage of the latest step
 * limited the cell (theta < 1 - 1e-8), else 0; nx*ny bytes, [j][i] (SOA) or [i][j]
 * (REF_AOS).  All 0 without PPlimiter (the reference never writes it then). */
int wenofv_theta_flags(wenofv_ctx *ctx, uint8_t *out, int layout);
/* Asynchronous snapshot of the current state for output (the gathers of outputResults,
 * src/WENOFV.cpp:2447-2523): the state is copied on the device at this point of the
 * context's stream, then read back into host on a separate copy stream, so the read-back
 * overlaps later steps.  host must stay valid until wenofv_snapshot_wait returns (pinned
 * memory makes the copy a DMA; pageable memory is also accepted).  One snapshot in flight
 * per context (WENOFV_EBUSY otherwise). */
int wenofv_snapshot_begin(wenofv_ctx *ctx, double *host, int layout);
int wenofv_snapshot_wait(wenofv_ctx *ctx);

/* The reference's periodic test cases (TESTCASE 0 SMOOTH, 1 VORTEX, 2 SHARP) with the
 * velocity and volume-fraction floor of TwoPhaseEquation::setEquationParameters
 * (include/Equations.hpp:490-689); the phase parameters are the context's. */
typedef struct {
    int testcase;
    double u0, v0, epsa;
} wenofv_testcase;
/* CWENOFV::initializeAve (src/WENOFV.cpp:232-279) on the GPU: the 4x4 Gauss-Legendre
 * averages of getU0 (include/Equations.hpp:979-1002) over the slab grid, written as the
 * context's state (the device sin/exp differ from the host C library's by a few ulp) */
int wenofv_init_testcase(wenofv_ctx *ctx, const wenofv_testcase *tc);
/* CWENOFV::outputAccuracy (src/WENOFV.cpp:3152-3251) on the GPU: norms = (L_inf, L1, L2) of
 * the volume fraction against the initial data translated by (u0, v0) t */
int wenofv_accuracy(wenofv_ctx *ctx, const wenofv_testcase *tc, double t, double norms[3]);
/* One SSP-RK step (cfg->rk_method) of a caller-owned device state without allocating any
 * device memory: for callers that cannot call cudaMalloc (they manage GPU memory through
 * their own pool or framework allocator, which a direct cudaMalloc would bypass and may
 * exceed; they reserve all free device memory at start-up; or they cannot afford the device
 * synchronisation of cudaMalloc/cudaFree inside a latency-bound loop).  d_U and
 * d_U_next are distinct device arrays, SoA [v][ny][pitch] with pitch >= nx; d_U is only
 * read.  The stage kernel's scratch (one intermediate RK state, grid metric, descriptor,
 * loop state, work list, counter) is a fixed 4.2 MiB device array inside the library, held
 * by every GPU that loads it until exit; so nvar*ny*pitch <= 524288, 2*nx + ny <= 8192 and
 * ceil(nx/strip)*ceil(ny/16) <= 8192, otherwise WENOFV_EINVAL.  The first call on a device
 * looks up that array's address and should come before any stream capture.  Calls share
 * the array: calls whose work overlaps on the GPU race.  The call synchronises `stream`
 * (a cudaStream_t, NULL = default stream) once after its host-to-device set-up copies, and
 * again at the end when flags is non-NULL (then *flags receives the WENOFV_FLAG_* word).
 * The caller's current device is the same on return as on entry.  The step takes dt from the
 * caller (finite, >= 0) and does not return the CFL step of the new state: a caller that
 * needs it calls wenofv_compute_dt on a context.  No counterpart in the reference. */
int wenofv_step_noalloc(const wenofv_config *cfg, const wenofv_eq_params *eq, const double *d_U, double *d_U_next,
                        int pitch, double dt, void *stream, uint32_t *flags);

/* ---- batched ensemble: many uneven instances per persistent launch (no counterpart in
 *      the reference, which solves one grid per MPI job) ---------------------------------- */
typedef struct wenofv_batch wenofv_batch;
/* all instances share device and rk_method; grids, schemes, fluxes, limiter, equations
 * and precision may differ per instance */
int wenofv_batch_create(int n, const wenofv_config *cfgs, const wenofv_eq_params *eqs, wenofv_batch **out);
void wenofv_batch_destroy(wenofv_batch *b);
int wenofv_batch_upload(wenofv_batch *b, int i, const double *U, int layout);
int wenofv_batch_download(wenofv_batch *b, int i, double *U, int layout);
/* wenofv_set_frame for instance i of a batch */
int wenofv_batch_set_frame(wenofv_batch *b, int i, const double *frame);
/* advances instance k from t=0 to t_end[k]; nsteps[k] receives its step count */
int wenofv_batch_advance(wenofv_batch *b, const double *t_end, int64_t max_steps, int64_t *nsteps);
/* rows per work item and CTAs per SM of the persistent stage kernel (0 = automatic) */
int wenofv_batch_set_tiling(wenofv_batch *b, int rows_per_item, int ctas_per_sm);
int wenofv_batch_stream(wenofv_batch *b, void **stream);
/* threads per CTA of the stage kernels: 0 (the default) chooses per instance, 256 (strips of 58
 * columns, 56 on the 7-point geometry) where the grid's width fills them well, else 128 (26 or
 * 24 columns); 128 or 256 forces that width for every instance that has it (the stiffened gas
 * and scalar advection run 128 only) */
int wenofv_batch_set_threads(wenofv_batch *b, int threads_per_cta);
/* the current tiling settings (0 = automatic) */
int wenofv_batch_tiling(wenofv_batch *b, int *rows_per_item, int *ctas_per_sm, int *threads_per_cta);
/* measures candidate tilings (threads per CTA x rows per work item x CTAs per SM; rows 0 =
 * the automatic choice among them) on the batch's current state (state unchanged) and keeps
 * the best; wenofv_batch_tiling reports it */
int wenofv_batch_autotune(wenofv_batch *b, int *rows_per_item, int *ctas_per_sm, double *best_ms);

/* ---- serving: continuous batching of solve requests under an HBM budget (no
 *      counterpart in the reference) ------------------------------------------------------- */
typedef struct wenofv_server wenofv_server;
typedef struct {
    double t_submit, t_admit, t_done; /* host seconds on the server's clock */
    int64_t steps;
    uint32_t flags;
    int status;
} wenofv_request_info;
/* starts a server on `device` with up to max_slots requests on the GPU at once.  The slots'
 * device memory is one arena allocated here: hbm_budget_bytes, or the device's free memory
 * less 1 GiB when that is smaller; admitting a request then allocates nothing. */
int wenofv_server_create(int device, size_t hbm_budget_bytes, int max_slots, wenofv_server **out);
void wenofv_server_destroy(wenofv_server *s);
/* queues a solve of U0 (SoA) from t=0 to t_end, or max_steps steps if that comes first
 * (max_steps <= 0: no limit); the server copies U0.  RKMETH must be 2 (SSP-RK3). */
int wenofv_server_submit(wenofv_server *s, const wenofv_config *cfg, const wenofv_eq_params *eq,
                         const double *U0, double t_end, int64_t max_steps, int64_t *request_id);
/* WENOFV_EBUSY while the request runs; otherwise its status (WENOFV_OK copies the result,
 * SoA) and the request is forgotten */
int wenofv_server_poll(wenofv_server *s, int64_t request_id, double *U, wenofv_request_info *info);
/* seconds on the server's clock */
double wenofv_server_clock(wenofv_server *s);
/* counters: admitted, completed, queued, active, resident bytes */
int wenofv_server_stats(wenofv_server *s, int64_t *admitted, int64_t *completed, int64_t *queued,
                        int64_t *active, int64_t *resident_bytes);

/* ---- device probes of the pointwise kernels (test hooks; they replace calls to the
 *      header-only reference kernels include/Utility.hpp and include/Equations.hpp) ------- */
/* WENO5threconstruction / WENO5Zthreconstruction (include/Utility.hpp:5-95, :193-290) at
 * the 4 Gauss-Lobatto points: stencils n x 5, out n x 4 */
int wenofv_probe_weno(int scheme, int precision, const double *stencils, int n, double *out, int device);
/* wenoExpthreconstruction (include/Utility.hpp:291-470) at the 4 Gauss-Lobatto points:
 * stencils n x 7, cell size dx (the threshold is pow(dx, 4)), out n x 4; FP64 forms only */
int wenofv_probe_weno_exp(int precision, const double *stencils, int n, double dx, double *out, int device);
/* getRiemannFlux (include/Equations.hpp:329-483): UL, UR, F are n x nvar */
int wenofv_probe_riemann(const wenofv_eq_params *eq, int flux, int precision, const double *UL,
                         const double *UR, int n, double nx, double ny, double *F, int device);
/* getLEigenMatrix / getREigenMatrix (include/Equations.hpp:189-327): L, R are n x 16 row-major */
int wenofv_probe_eigen(const wenofv_eq_params *eq, int precision, const double *U, int n, double nx,
                       double ny, double *L, double *R, int device);
/* measured FMA throughput of the FP64 (or, with WENOFV_FP32_BULK, FP32) CUDA-core pipe in
 * TFLOP/s: the denominator of the stage kernel's compute roofline (no reference counterpart) */
int wenofv_probe_fma_peak(int precision, int device, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
