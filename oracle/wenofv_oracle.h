/*
 * wenofv_oracle.h -- CPU restatement of the reference's WENOFV time-advance path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the sm_100a kernels: only the
 * tests, __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load it.  The
 * product path (the C-ABI library) never calls it and has no CPU fallback.
 *
 * Every function follows the reference's arithmetic in the same operation order (cited
 * per function as path:line inside the reference project), so that for the two-phase
 * linear-EOS system it reproduces the compiled reference bit for bit.  Linear advection,
 * Euler and outflow boundaries are extensions that the reference does not implement;
 * for those the oracle is the restated algorithm itself (parity unpinned by the reference).
 *
 * Data layout of every state array crossing this interface: SoA, U[v*ny*nx + j*nx + i],
 * interior cells only (no ghosts), i = x index (contiguous), j = y index.
 */
#ifndef WENOFV_ORACLE_H
#define WENOFV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Equation kinds (same numbering as include/wenofv.h). */
enum { OFV_EQ_TWO_PHASE = 0, OFV_EQ_LINEAR_ADV = 1, OFV_EQ_EULER = 2, OFV_EQ_TWO_PHASE_SG = 3 };
/* Boundary kinds: PERIOD = 0 as include/Equations.hpp:27; OUTFLOW is an extension. */
enum { OFV_BC_PERIOD = 0, OFV_BC_NEUMANN = 1, OFV_BC_NOSLIP = 2, OFV_BC_NEUMANN2 = 3, OFV_BC_FREESLIP = 4, OFV_BC_OUTFLOW = 5 };

typedef struct {
    int kind;
    /* TwoPhaseEquation parameters (include/Equations.hpp:67-69) */
    double rho10, rho20, sound1, sound2, preb;
    /* Euler ratio of specific heats */
    double gamma;
    /* linear advection velocity */
    double adv_u, adv_v;
    /* stiffened-gas phases (OFV_EQ_TWO_PHASE_SG, an extension): p_k(rho) on the isentrope
     * through (preb, rho_k0), rho10 and rho20 being the densities at preb */
    double gamma1, pinf1, gamma2, pinf2;
    /* assembleSourceTerm's g_g0 (src/WENOFV.cpp:1831-1872): rhs[rho v] -= rho g for the two-phase
     * kinds; 9.81 for DAMBREAK/RTI, 2 pi for STANDING_WAVE, 0 otherwise */
    double gravity;
} ofv_eq;

typedef struct {
    int nx, ny;            /* ELEMNUMX, ELEMNUMY */
    double xl, xr, yl, yr; /* domain */
    int bc;                /* OFV_BC_* */
    int rk;                /* RKMETH: 0 RK1, 1 RK2, 2 RK3 */
    double cfl;            /* CFL */
    int scheme;            /* SCHEME: 0 WENO-JS, 1 WENO-Z, 2 WENOEXP */
    int limiter;           /* PPlimiter */
    int flux;              /* RIEMANNFLUX: 0 LLF, 1 HLLC */
    int recon;             /* RECONSTRUCTIONTYPE: 0 conservative, 1 characteristic, 2 primitive
                              (z1, rho1, u, v), 3 primitive2 (z1, p, u, v); 2-3 two-phase only */
    int ref_slabs;         /* 0: uniform cell sizes; P>0: the reference's P-slab x metric */
    int threads;           /* OpenMP threads (0 = library default) */
    ofv_eq eq;
    /* NEUMANN2 (BOUNDARYTYPE 3, "boundary from the initial data", include/Equations.hpp:30):
     * fixed ghost averages, SoA [v][ny+8][nx+8] with the interior at offset (4, 4); the
     * interior entries are not read.  Unused by the other kinds. */
    const double *frame;
} ofv_problem;

int ofv_nvar(const ofv_eq *eq);

/* pointwise kernels */
double ofv_weno_js(const double v[5], int gp);
double ofv_weno_z(const double v[5], int gp);
/* wenoExpthreconstruction (include/Utility.hpp:291-470) on a 7-point stencil, cell size dx */
double ofv_weno_exp(const double v[7], int gp, double dx);
/* wenoExpWithThincReconstruction (include/Utility.hpp:473-688), PRIMITIVE3's z1 kernel */
double ofv_weno_exp_thinc(const double v[7], int gp, double dx);
/* 0 (default): WENOEXP's l^3 by the C library's pow, as the reference; 1: l^3 rounded once,
 * the device kernels' form */
void ofv_set_cube_rounded(int on);
/* 0 (default): THINC's exp, log and tanh as the C library returns them; 1: each moved one
 * ulp up (a probe of how much the result depends on the last bit of the math library) */
void ofv_set_thinc_ulp(int on);
double ofv_volume_frac(const ofv_eq *eq, const double *U);
double ofv_pressure(const ofv_eq *eq, const double *U);
double ofv_sound_speed(const ofv_eq *eq, const double *U);
double ofv_max_eig(const ofv_eq *eq, const double *U, double nx, double ny);
void ofv_riemann(const ofv_eq *eq, int flux, const double *UL, const double *UR,
                 double nx, double ny, double *F);
void ofv_eigen_L(const ofv_eq *eq, const double *U, double nx, double ny, double *L);
void ofv_eigen_R(const ofv_eq *eq, const double *U, double nx, double ny, double *R);

/* grid metric: dxc[nx], dxl[nx], dy[ny] (see ofv_metric in the .c file) */
void ofv_metric(const ofv_problem *p, double *dxc, double *dxl, double *dy);

/* whole-grid operators */
double ofv_compute_dt(const ofv_problem *p, const double *U, int *nan_flag);
/* rhs of one stage; theta_flags (may be NULL) receives the per-cell limiter flag */
void ofv_rhs(const ofv_problem *p, const double *U, double *rhs, double *theta_flags);
/* face states after the limiter for interior cells: out[cell][face B,T,L,R][var][gp] */
void ofv_face_states(const ofv_problem *p, const double *U, double *out);
void ofv_step(const ofv_problem *p, double *U, double dt);
/* time loop of CWENOFV::run to one target time; returns the number of steps taken */
int ofv_advance(const ofv_problem *p, double *U, double t0, double t_end, double *t_out,
                int max_steps, double *dts);

#ifdef __cplusplus
}
#endif
#endif
