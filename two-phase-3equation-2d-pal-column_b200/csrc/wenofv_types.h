// wenofv_types.h -- plain structures shared by the device kernels (strict and fast builds)
// and the host side of the C ABI.  No CUDA types in here.
#pragma once
#include <stddef.h>

namespace wenofv {

struct EqParams {
    int kind; // 0 two-phase, 1 linear advection, 2 Euler, 3 two-phase stiffened gas (include/wenofv.h)
    double rho10, rho20, sound1, sound2, preb, gamma, adv_u, adv_v;
    double gamma1, pinf1, gamma2, pinf2;
    double gravity; // two-phase kinds: rhs[rho v] -= rho g
};

enum { EQ_TWO_PHASE = 0, EQ_LINEAR_ADV = 1, EQ_EULER = 2, EQ_TWO_PHASE_SG = 3 };

// one instance (a grid and its options) as the stage kernel sees it
struct InstDesc {
    double *buf[3];               // state buffers, SoA [v][ny][pitch]
    const double *dxc, *dxl, *dy; // grid metric: column widths (own / left neighbour as seen
                                  // by the column's slab) and row heights
    int nx, ny, pitch, bc;
    int scheme, flux, limiter, recon, eq_kind, pad;
    double cfl, dX, dY;
    double dx4; // pow(dX, 4) as the host C library rounds it: WENOEXP's smoothness threshold
    EqParams eq;
    const double *frame; // NEUMANN2: fixed ghost averages [v][ny+8][nx+8], interior at (4, 4)
    unsigned char *theta_flag; // optional [ny][nx]: 1 where the final stage's limiter theta < 1 - 1e-8
};

// mutable per-instance state of the device-side time loop
struct InstState {
    double now, t_end, dt, dtcfl;
    unsigned long long accum; // bits of the running CFL minimum (positive doubles order as integers)
    long long nsteps, max_steps, bad_cell;
    unsigned int flags;
    int done, mode, cur_buf;
};
enum { MODE_MANUAL = 0, MODE_ADVANCE = 1 };
enum { FIN_STEP = 0, FIN_INIT = 1 };

// a strip of columns [i0, i0+TX) and rows [j0, j1) of one instance
struct WorkItem {
    int inst, i0, j0, j1;
};

struct StageLaunch {
    const InstDesc *inst;
    InstState *state;
    const WorkItem *work;
    int nwork;
    const int *fin_ids; // instances this launch finalizes
    int nfin;
    const int *counts; // optional device copy of {nwork, nfin}: the serving engine updates its
                       // work lists in place, so captured graphs keep fixed launch arguments
    unsigned int *counter;
    int bin, bun, bout; // buffer roles: stage input, U^n, output
    int first_stage, final_stage, rk1;
    double A, B, C;  // U_out = (A*U^n + B*U) + (C*dt)*rhs
    double *rhs_out; // non-null: write the RHS (layout of instance 0) instead of the update
    int tx;          // strip width of the work items (the CFL pass reads it)
};

// host launchers exported by each build of wenofv_kernels.cu
#define WENOFV_DECLARE_LAUNCHERS(NS)                                                                     \
    namespace NS {                                                                                       \
    int stage_wide(int eq, int recon);                                                                   \
    int stage_tx(int eq, int recon, int fp32, int scheme, int nt);                                       \
    int launch_stage(int eq, int recon, int fp32, int scheme, int flux, int nt, const StageLaunch &L,    \
                     int grid, void *stream);                                                           \
    int launch_cfl(int eq, int recon, int fp32, int scheme, int nt, const StageLaunch &L, int grid,      \
                   void *stream);                                                                       \
    int stage_blocks_per_sm(int eq, int recon, int fp32, int scheme, int flux, int nt);                  \
    int probe_weno(int scheme, int fp32, const double *d_st, int n, double *d_out, void *stream);       \
    int probe_weno_exp(const double *d_st, int n, double dx4, double *d_out, void *stream);             \
    int probe_riemann(const EqParams &P, int flux, int fp32, const double *d_UL, const double *d_UR,   \
                      int n, int xdir, double *d_F, void *stream);                                       \
    int probe_eigen(const EqParams &P, int fp32, const double *d_U, int n, int xdir, double *d_L,       \
                    double *d_R, void *stream);                                                          \
    }

WENOFV_DECLARE_LAUNCHERS(strict)
WENOFV_DECLARE_LAUNCHERS(fast)
namespace fast {
int fma_peak(int fp32, double *tflops, void *stream);
}

} // namespace wenofv
