/*
 * wenofv_oracle.c -- CPU restatement of the reference's WENOFV time-advance path.
 *
 * TEST INFRASTRUCTURE ONLY (see wenofv_oracle.h).  Citations are path:line inside the
 * reference project.  The code is plain C99 that also compiles as C++ so that the
 * flop-counting build (-DOFV_COUNTING, ofv_count.hpp) can run the same arithmetic.
 *
 * Two deliberate structural differences from the reference, neither of which changes a
 * single bit of the result:
 *   1. The reference reconstructs the 7 y-columns of every cell's 7x7 stencil per cell
 *      (src/WENOFV.cpp:670-687, :806-833).  Column k of cell (i,j) is exactly the centre
 *      column of cell (i+k-3, j), computed from the same operands, so the y-sweep is done
 *      once per (column,row) and shared.
 *   2. Ghost-cell face states arrive in the reference by MPI exchange and a periodic copy
 *      (src/WENOFV.cpp:1558-1668, :1542-1556).  Here they are reconstructed directly from
 *      4-layer ghost-filled averages (the 7-point WENOEXP stencil of a halo cell reaches
 *      the 4th layer), which applies the same arithmetic to the same operands as the
 *      neighbouring interior cell.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef OFV_COUNTING
#include "ofv_count.hpp"
typedef ofv_cnt real_t;
ofv_counters g_ofv_cnt;
#define OFV_ISNAN(x) ofv_isnan(x)
#else
typedef double real_t;
#define OFV_ISNAN(x) isnan(x)
#endif

#include "wenofv_oracle.h"

#define G 3  /* ghost layers of the reference's grid, src/WENOFV.cpp:59 */
#define GE 4 /* ghost layers of the oracle's work arrays: WENOEXP's 7-point stencils of the halo
                cells reach one layer further than the reference's own stencils */

/* std::min / std::max as used unqualified by the reference (MyMath.h:22 imports std). */
static inline real_t std_min(real_t a, real_t b) { return (b < a) ? b : a; }
static inline real_t std_max(real_t a, real_t b) { return (a < b) ? b : a; }
/* sc_math::Min, third_party/scTools/MyMath.h:52-55: a NaN 'a' yields b. */
static inline real_t sc_min(real_t a, real_t b) { return (a < b) ? a : b; }

/* Gauss-Lobatto 4-point weights as written at third_party/scTools/GaussQuadratureInRef.hpp:252-262 */
static const double GL_W[4] = {0.166666666666666666666666666667, 0.833333333333333333333333333333,
                               0.833333333333333333333333333333, 0.166666666666666666666666666667};

int ofv_nvar(const ofv_eq *eq) { return eq->kind == OFV_EQ_LINEAR_ADV ? 1 : 4; }

/* ------------------------------------------------------------------------------------ */
/* WENO point reconstructions at Gauss-Lobatto point gp (0 left edge, 3 right edge)       */
/* ------------------------------------------------------------------------------------ */

/* linear weights, include/Utility.hpp:12-39 (identical in :203-230) */
static void weno_d(int gp, real_t *d0, real_t *d1, real_t *d2)
{
    switch (gp) {
    case 0: *d0 = 0.3; *d1 = 0.6; *d2 = 0.1; break;
    case 1:
        *d0 = (91.0 - 9.0 * sqrt(5.0)) / 440.0;
        *d1 = 129.0 / 220.0;
        *d2 = (91.0 + 9.0 * sqrt(5.0)) / 440.0;
        break;
    case 2:
        *d0 = (91.0 + 9.0 * sqrt(5.0)) / 440.0;
        *d1 = 129.0 / 220.0;
        *d2 = (91.0 - 9.0 * sqrt(5.0)) / 440.0;
        break;
    default: *d0 = 0.1; *d1 = 0.6; *d2 = 0.3; break;
    }
}

/* candidate polynomials at gp, include/Utility.hpp:64-90 (identical in :233-259) */
static void weno_h(int gp, real_t umm, real_t um, real_t u, real_t up, real_t upp, real_t *h0,
                   real_t *h1, real_t *h2)
{
    switch (gp) {
    case 0:
        *h0 = -1.0 / 6.0 * umm + 5.0 / 6.0 * um + 1.0 / 3.0 * u;
        *h1 = 1.0 / 3.0 * um + 5.0 / 6.0 * u - 1.0 / 6 * up;
        *h2 = 11.0 / 6.0 * u - 7.0 / 6.0 * up + 1.0 / 3.0 * upp;
        break;
    case 1:
        *h0 = (-1.0 / 60.0 - sqrt(5.0) / 20.0) * umm + (1.0 / 30.0 + sqrt(5.0) / 5.0) * um +
              (59.0 / 60.0 - 3 * sqrt(5.0) / 20.0) * u;
        *h1 = (-1.0 / 60.0 + sqrt(5.0) / 20.0) * um + (31.0 / 30.0) * u + (-1.0 / 60 - sqrt(5.0) / 20.0) * up;
        *h2 = (59.0 / 60.0 + 3 * sqrt(5.0) / 20) * u + (1.0 / 30.0 - sqrt(5.0) / 5.0) * up +
              (-1.0 / 60.0 + sqrt(5.0) / 20.0) * upp;
        break;
    case 2:
        *h0 = (-1.0 / 60.0 + sqrt(5.0) / 20.0) * umm + (1.0 / 30.0 - sqrt(5.0) / 5.0) * um +
              (59.0 / 60.0 + 3 * sqrt(5.0) / 20) * u;
        *h1 = (-1.0 / 60 - sqrt(5.0) / 20.0) * um + (31.0 / 30.0) * u + (-1.0 / 60.0 + sqrt(5.0) / 20.0) * up;
        *h2 = (59.0 / 60.0 - 3 * sqrt(5.0) / 20.0) * u + (1.0 / 30.0 + sqrt(5.0) / 5.0) * up +
              (-1.0 / 60.0 - sqrt(5.0) / 20.0) * upp;
        break;
    default:
        *h0 = 1.0 / 3.0 * umm - 7.0 / 6.0 * um + 11.0 / 6.0 * u;
        *h1 = -1.0 / 6 * um + 5.0 / 6.0 * u + 1.0 / 3.0 * up;
        *h2 = 1.0 / 3.0 * u + 5.0 / 6.0 * up - 1.0 / 6.0 * upp;
        break;
    }
}

/* WENO-JS (Jiang & Shu 1996), include/Utility.hpp:5-95 */
static real_t weno_js(real_t umm, real_t um, real_t u, real_t up, real_t upp, int gp)
{
    real_t d0, d1, d2, h0, h1, h2;
    weno_d(gp, &d0, &d1, &d2);
    real_t t0 = umm - 4 * um + 3 * u, s0 = umm - 2 * um + u;
    real_t t1 = um - up, s1 = um - 2 * u + up;
    real_t t2 = 3 * u - 4 * up + upp, s2 = u - 2 * up + upp;
    /* pow(x, 2) of :48-50 folds to x*x in the compiled reference */
    const real_t beta0 = 0.25 * (t0 * t0) + 13.0 / 12.0 * (s0 * s0);
    const real_t beta1 = 0.25 * (t1 * t1) + 13.0 / 12.0 * (s1 * s1);
    const real_t beta2 = 0.25 * (t2 * t2) + 13.0 / 12.0 * (s2 * s2);
    const double eps = 1.0e-6;
    real_t w0 = d0 / ((eps + beta0) * (eps + beta0));
    real_t w1 = d1 / ((eps + beta1) * (eps + beta1));
    real_t w2 = d2 / ((eps + beta2) * (eps + beta2));
    const real_t sum = w0 + w1 + w2;
    w0 = w0 / sum;
    w1 = w1 / sum;
    w2 = w2 / sum;
    weno_h(gp, umm, um, u, up, upp, &h0, &h1, &h2);
    return w0 * h0 + w1 * h1 + w2 * h2;
}

/* WENO-Z (Borges et al. 2008) with min/max stencil normalisation, include/Utility.hpp:193-290 */
static real_t weno_z(real_t umm, real_t um, real_t u, real_t up, real_t upp, int gp)
{
    real_t d0, d1, d2, p0, p1, p2;
    weno_d(gp, &d0, &d1, &d2);
    weno_h(gp, umm, um, u, up, upp, &p0, &p1, &p2); /* from the raw values, :233-259 */
    const real_t umax = std_max(std_max(std_max(umm, um), std_max(upp, up)), u);
    const real_t umin = std_min(std_min(std_min(umm, um), std_min(upp, up)), u);
    umm = (umm - umin) / (umax - umin + 1e-20);
    um = (um - umin) / (umax - umin + 1e-20);
    u = (u - umin) / (umax - umin + 1e-20);
    up = (up - umin) / (umax - umin + 1e-20);
    upp = (upp - umin) / (umax - umin + 1e-20);
    real_t t0 = umm - 4 * um + 3 * u, s0 = umm - 2 * um + u;
    real_t t1 = um - up, s1 = um - 2 * u + up;
    real_t t2 = 3 * u - 4 * up + upp, s2 = u - 2 * up + upp;
    const real_t beta0 = 0.25 * (t0 * t0) + 13.0 / 12.0 * (s0 * s0);
    const real_t beta1 = 0.25 * (t1 * t1) + 13.0 / 12.0 * (s1 * s1);
    const real_t beta2 = 0.25 * (t2 * t2) + 13.0 / 12.0 * (s2 * s2);
    const double eps = 1.0e-10;
    real_t tau = fabs(beta0 - beta2);
    real_t w0 = d0 * (1 + tau / (beta0 + eps));
    real_t w1 = d1 * (1 + tau / (beta1 + eps));
    real_t w2 = d2 * (1 + tau / (beta2 + eps));
    real_t sum = w0 + w1 + w2;
    w0 = w0 / sum;
    w1 = w1 / sum;
    w2 = w2 / sum;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

/* l^3 of WENOEXP's linear weights.  By default the C library's pow(l, 3), as the reference
 * calls it (gcc keeps pow(x, 3) a library call without -ffast-math; glibc's pow is within
 * 0.52 ulp, not always correctly rounded).  ofv_set_cube_rounded(1) selects l^3 rounded once
 * instead -- the exact square x*x = p + e (e by fma), times x with the exact error of p*x --
 * the form of the device kernels, so that they can be compared bit for bit. */
static int g_cube_rn = 0;
void ofv_set_cube_rounded(int on) { g_cube_rn = on; }
static real_t cube_of(real_t l)
{
#ifndef OFV_COUNTING
    if (g_cube_rn) {
        const double x = l, p = x * x, e = fma(x, x, -p), hi = p * x, lo = fma(p, x, -hi);
        return hi + (lo + e * x);
    }
#endif
    return pow(l, 3);
}

/* WENOEXP's linear weights at Gauss point gp, cubics in l2h2 (include/Utility.hpp:362-392,
 * the same in :553-583) */
static void exp_linear_weights(int gp, real_t l2h2, real_t *d0, real_t *d1, real_t *d2)
{
    const real_t l2 = pow(l2h2, 2), l3 = cube_of(l2h2);
    if (gp == 0 || gp == 3) {
        const real_t a = 0.3 - 0.057142858 * l2h2 + 0.0071428571 * l2 - 0.00077200577 * l3;
        const real_t b = 0.6 + 0.078571429 * l2h2 - 0.0101190476 * l2 + 0.00112012987 * l3;
        const real_t e = 0.1 - 0.021428571 * l2h2 + 0.0029761905 * l2 - 0.00034812410 * l3;
        *d0 = gp == 0 ? a : e; *d1 = b; *d2 = gp == 0 ? e : a;
    } else {
        const real_t a = 0.16108042 - 0.035187607 * l2h2 + 0.0049466098 * l2 - 0.00058211525 * l3;
        const real_t b = 0.58636364 + 0.087692641 * l2h2 - 0.0120401515 * l2 + 0.00139436871 * l3;
        const real_t e = 0.25255594 - 0.052505034 * l2h2 + 0.0070935417 * l2 - 0.00081225346 * l3;
        *d0 = gp == 1 ? a : e; *d1 = b; *d2 = gp == 1 ? e : a;
    }
}

/* WENOEXP (SCHEME 2), include/Utility.hpp:291-470: the linear weights are cubic polynomials
 * in lambda^2 h^2 = dif5 / dif3 (from the 6 points on the side of the Gauss point, clipped at
 * 1, or 0 where |dif3| < dx^4), the smoothness indicators are absolute values on the
 * normalised stencil, and w_k = d_k (1 + 2 tau^2 / (beta_k^2 + 1e-16)). */
static real_t weno_exp(const real_t *v7, int gp, double dx)
{
    real_t mmm = v7[0], mm = v7[1], m = v7[2], c = v7[3], p = v7[4], pp = v7[5], ppp = v7[6];
    real_t dif5, dif3;
    if (gp >= 2) {
        dif5 = (-mm + 5.0 * m - 10.0 * c + 10.0 * p - 5.0 * pp + ppp);
        dif3 = (mm - 11.0 * m + 28.0 * c - 28.0 * p + 11.0 * pp - ppp) / 6.0;
    } else {
        dif5 = (-mmm + 5.0 * mm - 10.0 * m + 10.0 * c - 5.0 * p + pp);
        dif3 = (mmm - 11.0 * mm + 28.0 * m - 28.0 * c + 11.0 * p - pp) / 6.0;
    }
    real_t l2h2 = 0;
    if (!(fabs(dif3) < pow(dx, 4))) {
        l2h2 = dif5 / dif3;
        if (fabs(l2h2) > 1) l2h2 = 1;
    }
    real_t h0, h1, h2, d0, d1, d2;
    weno_h(gp, mm, m, c, p, pp, &h0, &h1, &h2); /* candidate values from the raw stencil */
    exp_linear_weights(gp, l2h2, &d0, &d1, &d2);
    const real_t umax = std_max(std_max(std_max(mm, m), std_max(c, p)), pp);
    const real_t umin = std_min(std_min(std_min(mm, m), std_min(c, p)), pp);
    mm = (mm - umin) / (umax - umin + 1e-20);
    m = (m - umin) / (umax - umin + 1e-20);
    c = (c - umin) / (umax - umin + 1e-20);
    p = (p - umin) / (umax - umin + 1e-20);
    pp = (pp - umin) / (umax - umin + 1e-20);
    const real_t beta0 = 1.0 * 1.0 / 2.0 * fabs(mm - 4 * m + 3 * c) + fabs(mm - 2 * m + c);
    const real_t beta1 = 1.0 * 1.0 / 2.0 * fabs(m - p) + fabs(m - 2 * c + p);
    const real_t beta2 = 1.0 * 1.0 / 2.0 * fabs(3 * c - 4 * p + pp) + fabs(c - 2 * p + pp);
    const real_t tau = mm - 4.0 * m + 6.0 * c - 4.0 * p + pp;
    const double epsilon = 1e-16;
    real_t w0 = d0 * (1.0 + 2 * pow(tau, 2.0) / (pow(beta0, 2.0) + epsilon));
    real_t w1 = d1 * (1.0 + 2 * pow(tau, 2.0) / (pow(beta1, 2.0) + epsilon));
    real_t w2 = d2 * (1.0 + 2 * pow(tau, 2.0) / (pow(beta2, 2.0) + epsilon));
    const real_t S = w0 + w1 + w2;
    w0 /= S;
    w1 /= S;
    w2 /= S;
    return w0 * h0 + w1 * h1 + w2 * h2;
}

/* exp, log and tanh of the THINC profile: the C library's, or (ofv_set_thinc_ulp(1), a
 * sensitivity probe for tests) each result moved one ulp up.  exp at exactly +-1.5 stays
 * exact there: those are the degenerate profiles (C = 0 or 1) whose xc is exactly 0 or inf
 * because B equals the compile-time constant exp(+-beta). */
static int g_thinc_ulp = 0;
void ofv_set_thinc_ulp(int on) { g_thinc_ulp = on; }
static real_t thinc_exp(real_t x)
{
#ifndef OFV_COUNTING
    if (g_thinc_ulp && x != 1.5 && x != -1.5) return nextafter(exp(x), INFINITY);
#endif
    return exp(x);
}
static real_t thinc_log(real_t x)
{
#ifndef OFV_COUNTING
    if (g_thinc_ulp) return nextafter(log(x), INFINITY);
#endif
    return log(x);
}
static real_t thinc_tanh(real_t x)
{
#ifndef OFV_COUNTING
    if (g_thinc_ulp) return nextafter(tanh(x), INFINITY);
#endif
    return tanh(x);
}

/* Gauss-Lobatto points of the reference interval (GaussLobatto_ref(4),
 * third_party/scTools/GaussQuadratureInRef.hpp:250-259) */
static const double GLOB_X[4] = {-1, -0.447213595499957939281834733746, 0.447213595499957939281834733746, 1};

/* wenoExpWithThincReconstruction, include/Utility.hpp:473-688: PRIMITIVE3's reconstruction of
 * z1.  Where the centre value is a mixture (1e-6 < u < 1 - 1e-6) a THINC profile (a tanh of
 * steepness 1.5 through the cell, from its two neighbours); elsewhere WENOEXP's linear weights
 * (l2h2 unclipped) with WENO-Z's smoothness indicators on the normalised stencil and
 * w_k = d_k (1 + |beta0 - beta2| / (beta_k + 1e-16)).  The THINC branch's unused A
 * (:668) is left out. */
static real_t weno_exp_thinc(const real_t *v7, int gp, double dx)
{
    real_t mmm = v7[0], mm = v7[1], m = v7[2], c = v7[3], p = v7[4], pp = v7[5], ppp = v7[6];
    real_t dif5, dif3;
    if (gp >= 2) {
        dif5 = (-mm + 5.0 * m - 10.0 * c + 10.0 * p - 5.0 * pp + ppp);
        dif3 = (mm - 11.0 * m + 28.0 * c - 28.0 * p + 11.0 * pp - ppp) / 6.0;
    } else {
        dif5 = (-mmm + 5.0 * mm - 10.0 * m + 10.0 * c - 5.0 * p + pp);
        dif3 = (mmm - 11.0 * mm + 28.0 * m - 28.0 * c + 11.0 * p - pp) / 6.0;
    }
    real_t l2h2 = 0;
    if (!(fabs(dif3) < pow(dx, 4))) l2h2 = dif5 / dif3;
    const int thinc = (1e-6 < c) & (c < 1 - 1e-6);
    if (!thinc) {
        real_t h0, h1, h2, d0, d1, d2;
        weno_h(gp, mm, m, c, p, pp, &h0, &h1, &h2);
        exp_linear_weights(gp, l2h2, &d0, &d1, &d2);
        const real_t umax = std_max(std_max(std_max(mm, m), std_max(c, p)), pp);
        const real_t umin = std_min(std_min(std_min(mm, m), std_min(c, p)), pp);
        mm = (mm - umin) / (umax - umin + 1e-20);
        m = (m - umin) / (umax - umin + 1e-20);
        c = (c - umin) / (umax - umin + 1e-20);
        p = (p - umin) / (umax - umin + 1e-20);
        pp = (pp - umin) / (umax - umin + 1e-20);
        const real_t beta0 = 0.25 * pow(mm - 4 * m + 3 * c, 2) + 13.0 / 12.0 * pow(mm - 2 * m + c, 2);
        const real_t beta1 = 0.25 * pow(m - p, 2) + 13.0 / 12.0 * pow(m - 2 * c + p, 2);
        const real_t beta2 = 0.25 * pow(3 * c - 4 * p + pp, 2) + 13.0 / 12.0 * pow(c - 2 * p + pp, 2);
        const double eps = 1.0e-16;
        const real_t tau = fabs(beta0 - beta2);
        real_t w0 = d0 * (1 + tau / (beta0 + eps));
        real_t w1 = d1 * (1 + tau / (beta1 + eps));
        real_t w2 = d2 * (1 + tau / (beta2 + eps));
        const real_t S = w0 + w1 + w2;
        w0 /= S;
        w1 /= S;
        w2 /= S;
        return w0 * h0 + w1 * h1 + w2 * h2;
    }
    const real_t Qmin = std_min(m, p);
    const real_t Qmax = std_max(m, p) - Qmin;
    const real_t theta = (p - c >= 0) ? 1 : -1; /* sc_math::Sign, third_party/scTools/MyMath.h:47-50 */
    const double beta = 1.5;
    const real_t C = (c - Qmin + 1e-20) / (Qmax + 1e-20);
    const real_t B = thinc_exp(theta * beta * (2.0 * C - 1.0));
    const real_t xc = (exp(beta) - B) / (B - exp(-beta));
    const real_t xcc = thinc_log(xc) / (2.0 * beta);
    if ((c - m) * (p - c) < 0) return c;
    return 0.5 * Qmax * (1 + theta * thinc_tanh(beta * ((GLOB_X[gp] + 1) / 2 - xcc))) + Qmin;
}

/* useWENO dispatch, src/WENOFV.cpp:1873-1893, on a 7-point stencil v7 (the 5-point schemes
 * use its middle 5) */
static inline real_t weno7(int scheme, const real_t *v7, int gp, double dx)
{
    if (scheme == 2) return weno_exp(v7, gp, dx);
    const real_t *v = v7 + 1;
    return scheme == 1 ? weno_z(v[0], v[1], v[2], v[3], v[4], gp) : weno_js(v[0], v[1], v[2], v[3], v[4], gp);
}
/* variable k of a primitive reconstruction: PRIMITIVE3 (src/WENOFV.cpp:1293-1331) takes z1
 * through wenoExpWithThincReconstruction and the others through WENO-Z, whatever SCHEME is */
static inline real_t weno7_var(int scheme, int recon, int k, const real_t *v7, int gp, double dx)
{
    if (recon == 4) return k == 0 ? weno_exp_thinc(v7, gp, dx) : weno_z(v7[1], v7[2], v7[3], v7[4], v7[5], gp);
    return weno7(scheme, v7, gp, dx);
}


double ofv_weno_js(const double v[5], int gp) { return weno_js(v[0], v[1], v[2], v[3], v[4], gp); }
double ofv_weno_z(const double v[5], int gp) { return weno_z(v[0], v[1], v[2], v[3], v[4], gp); }
double ofv_weno_exp(const double v[7], int gp, double dx)
{
    real_t r[7];
    for (int k = 0; k < 7; k++) r[k] = v[k];
    return (double)weno_exp(r, gp, dx);
}
double ofv_weno_exp_thinc(const double v[7], int gp, double dx)
{
    real_t r[7];
    for (int k = 0; k < 7; k++) r[k] = v[k];
    return (double)weno_exp_thinc(r, gp, dx);
}

/* ------------------------------------------------------------------------------------ */
/* Two-phase 3-equation model, linear acoustic EOS (include/Equations.hpp:52-483)         */
/* U = (z1 rho1, z2 rho2, rho u, rho v)                                                   */
/* ------------------------------------------------------------------------------------ */

/* Stiffened-gas phases on their isentropes (OFV_EQ_TWO_PHASE_SG; an extension, not in the
 * reference): p_k(rho) = (preb + pi_k) (rho / rho_k0)^gamma_k - pi_k, whose expansion at preb
 * is the reference's linear model with c_k^2 = gamma_k (preb + pi_k) / rho_k0.  Pressure
 * equilibrium z1rho1 / rho_1(p) + z2rho2 / rho_2(p) = 1 is solved for p by Newton steps from
 * the linear model's state (kept above -min(pi_k), where both densities exist), until a step
 * is below 1e-14 (|p| + max(pi_k) + |preb|), at most SG_NEWTON; z1 = z1rho1 / rho_1(p).
 * Phase sound speeds c_k^2 = gamma_k (p + pi_k) / rho_k. */
#define SG_NEWTON 12
static real_t tp_volume_frac(const ofv_eq *e, const real_t *U);
static real_t tp_pressure_z(const ofv_eq *e, const real_t *U, real_t z1);
static void sg_linearised(const ofv_eq *e, ofv_eq *lin)
{
    *lin = *e;
    lin->kind = OFV_EQ_TWO_PHASE;
    lin->sound1 = sqrt(e->gamma1 * (e->preb + e->pinf1) / e->rho10);
    lin->sound2 = sqrt(e->gamma2 * (e->preb + e->pinf2) / e->rho20);
}
/* the last solve of each thread, so that the volume fraction, pressure, sound speed and phase
 * sound speeds of one state (asked for one by one, as the reference's functions are) cost
 * one solve; the result does not depend on the cache */
#ifdef OFV_COUNTING
#define OFV_TLS thread_local
#else
#define OFV_TLS __thread
#endif
static OFV_TLS double sg_key[9], sg_val[2];
static OFV_TLS int sg_valid = 0;
static void sg_solve_uncached(const ofv_eq *e, const real_t *U, real_t *z1_out, real_t *p_out);
static void sg_solve(const ofv_eq *e, const real_t *U, real_t *z1_out, real_t *p_out)
{
    const double key[9] = {(double)U[0], (double)U[1], e->rho10, e->rho20, e->preb, e->gamma1, e->pinf1, e->gamma2, e->pinf2};
    if (sg_valid && memcmp(key, sg_key, sizeof key) == 0) {
        *z1_out = sg_val[0];
        *p_out = sg_val[1];
        return;
    }
    sg_solve_uncached(e, U, z1_out, p_out);
    memcpy(sg_key, key, sizeof key);
    sg_val[0] = (double)*z1_out;
    sg_val[1] = (double)*p_out;
    sg_valid = 1;
}
static void sg_solve_uncached(const ofv_eq *e, const real_t *U, real_t *z1_out, real_t *p_out)
{
    ofv_eq lin;
    sg_linearised(e, &lin);
    const real_t m1 = U[0], m2 = U[1];
    const double pref = e->preb, g1 = e->gamma1, g2 = e->gamma2, pi1 = e->pinf1, pi2 = e->pinf2;
    const double a1 = 1.0 / (pref + pi1), a2 = 1.0 / (pref + pi2), ig1 = 1.0 / g1, ig2 = 1.0 / g2;
    const double lo = -(pi1 < pi2 ? pi1 : pi2);
    const double scale = (pi1 > pi2 ? pi1 : pi2) + fabs(pref);
    real_t p = pref + tp_pressure_z(&lin, U, tp_volume_frac(&lin, U));
    if (!(p > lo)) p = 0.5 * (pref + lo);
    for (int it = 0; it < SG_NEWTON; it++) {
        const real_t r1 = e->rho10 * pow((p + pi1) * a1, ig1);
        const real_t r2 = e->rho20 * pow((p + pi2) * a2, ig2);
        const real_t h = m1 / r1 + m2 / r2 - 1.0;
        const real_t dh = -(m1 / (r1 * (g1 * (p + pi1))) + m2 / (r2 * (g2 * (p + pi2))));
        real_t pn = p - h / dh;
        if (!(pn > lo)) pn = 0.5 * (p + lo);
        const real_t dp = pn - p;
        p = pn;
        if (fabs(dp) <= 1e-14 * (fabs(p) + scale)) break;
    }
    *z1_out = m1 / (e->rho10 * pow((p + pi1) * a1, ig1));
    *p_out = p;
}
/* the phase sound speeds squared (constant in the linear model) */
static void tp_phase_c2(const ofv_eq *e, const real_t *U, real_t z1, real_t *c1_2, real_t *c2_2)
{
    if (e->kind == OFV_EQ_TWO_PHASE_SG) {
        real_t zz, p;
        sg_solve(e, U, &zz, &p);
        *c1_2 = e->gamma1 * (p + e->pinf1) * z1 / U[0];
        *c2_2 = e->gamma2 * (p + e->pinf2) * (1.0 - z1) / U[1];
        return;
    }
    *c1_2 = (real_t)e->sound1 * e->sound1;
    *c2_2 = (real_t)e->sound2 * e->sound2;
}

/* getVolumeFrac, include/Equations.hpp:84-99 */
static real_t tp_volume_frac(const ofv_eq *e, const real_t *U)
{
    if (e->kind == OFV_EQ_TWO_PHASE_SG) {
        real_t z1, p;
        sg_solve(e, U, &z1, &p);
        return z1;
    }
    const real_t z1rho1 = U[0], z2rho2 = U[1];
    const real_t c1_2 = (real_t)e->sound1 * e->sound1;
    const real_t c2_2 = (real_t)e->sound2 * e->sound2;
    const real_t q = e->rho20 * c2_2 - e->rho10 * c1_2;
    const real_t qs = z2rho2 * c2_2 - z1rho1 * c1_2;
    const real_t r = ((q - qs) + sqrt((q - qs) * (q - qs) + 4.0 * z1rho1 * c1_2 * z2rho2 * c2_2)) / (2.0 * z2rho2 * c2_2);
    return r / (1.0 + r);
}

/* getPressure, include/Equations.hpp:101-124: the dominant phase's pressure (g_preb dropped) */
static real_t tp_pressure_z(const ofv_eq *e, const real_t *U, real_t z1)
{
    if (e->kind == OFV_EQ_TWO_PHASE_SG) { /* the equilibrium pressure, less g_preb as in the linear model */
        real_t zz, p;
        sg_solve(e, U, &zz, &p);
        return p - e->preb;
    }
    const real_t z2 = 1.0 - z1;
    const real_t c1_2 = (real_t)e->sound1 * e->sound1;
    const real_t c2_2 = (real_t)e->sound2 * e->sound2;
    const real_t pre1 = c1_2 * (U[0] / z1 - e->rho10);
    const real_t pre2 = c2_2 * (U[1] / z2 - e->rho20);
    if (z1 < z2)
        return pre2;
    return pre1;
}

/* getSoundSpeed (Wood), include/Equations.hpp:126-146 */
static real_t tp_sound_z(const ofv_eq *e, const real_t *U, real_t z1)
{
    if (e->kind == OFV_EQ_TWO_PHASE_SG) { /* Wood: 1 / (rho c^2) = sum_k z_k / (gamma_k (p + pi_k)) */
        real_t zz, p;
        sg_solve(e, U, &zz, &p);
        const real_t rho = U[0] + U[1];
        return 1.0 / sqrt(rho * (z1 / (e->gamma1 * (p + e->pinf1)) + (1.0 - z1) / (e->gamma2 * (p + e->pinf2))));
    }
    const real_t z2 = 1.0 - z1;
    const real_t rho = U[0] + U[1];
    const real_t rho1 = U[0] / z1;
    const real_t rho2 = U[1] / z2;
    const real_t c1_2 = (real_t)e->sound1 * e->sound1;
    const real_t c2_2 = (real_t)e->sound2 * e->sound2;
    const real_t sc = sqrt(rho * (z1 / (rho1 * c1_2) + z2 / (rho2 * c2_2)));
    return 1.0 / sc;
}

/* ------------------------------------------------------------------------------------ */
/* Euler, gamma-law gas, U = (rho, rho u, rho v, E).  Extension: not in the reference.    */
/* ------------------------------------------------------------------------------------ */
static real_t eu_pressure(const ofv_eq *e, const real_t *U)
{
    const real_t u = U[1] / U[0], v = U[2] / U[0];
    return (e->gamma - 1.0) * (U[3] - 0.5 * U[0] * (u * u + v * v));
}
static real_t eu_sound(const ofv_eq *e, const real_t *U, real_t p) { return sqrt(e->gamma * p / U[0]); }

/* ------------------------------------------------------------------------------------ */
/* equation dispatch                                                                      */
/* ------------------------------------------------------------------------------------ */

/* getMaxEigenValue, include/Equations.hpp:149-156 */
static real_t max_eig(const ofv_eq *e, const real_t *U, double nx, double ny)
{
    if (e->kind == OFV_EQ_LINEAR_ADV)
        return fabs((real_t)e->adv_u * nx + (real_t)e->adv_v * ny);
    if (e->kind == OFV_EQ_EULER) {
        const real_t p = eu_pressure(e, U);
        const real_t c = eu_sound(e, U, p);
        const real_t u = U[1] / U[0], v = U[2] / U[0];
        return fabs(u * nx + v * ny) + c;
    }
    const real_t z1 = tp_volume_frac(e, U);
    const real_t soundspeed = tp_sound_z(e, U, z1);
    const real_t u = U[2] / (U[0] + U[1]);
    const real_t v = U[3] / (U[0] + U[1]);
    return fabs(u * nx + v * ny) + soundspeed;
}

/* getPhyFlux, include/Equations.hpp:158-186 (two-phase); analogous Euler/advection fluxes */
static void phy_flux(const ofv_eq *e, const real_t *Uh, real_t *F, double nx, double ny)
{
    if (e->kind == OFV_EQ_LINEAR_ADV) {
        F[0] = ((real_t)e->adv_u * nx + (real_t)e->adv_v * ny) * Uh[0];
        return;
    }
    if (e->kind == OFV_EQ_EULER) {
        const real_t p = eu_pressure(e, Uh);
        const real_t u = Uh[1] / Uh[0], v = Uh[2] / Uh[0];
        const real_t vn = u * nx + v * ny;
        F[0] = Uh[0] * vn;
        F[1] = Uh[1] * vn + p * nx;
        F[2] = Uh[2] * vn + p * ny;
        F[3] = (Uh[3] + p) * vn;
        return;
    }
    const real_t z1rho1 = Uh[0], z2rho2 = Uh[1];
    const real_t rho = z1rho1 + z2rho2;
    const real_t u = Uh[2] / rho;
    const real_t v = Uh[3] / rho;
    const real_t pre = tp_pressure_z(e, Uh, tp_volume_frac(e, Uh));
    if (nx > ny) {
        F[0] = z1rho1 * u;
        F[1] = z2rho2 * u;
        F[2] = rho * (u * u) + pre;
        F[3] = rho * u * v;
    } else {
        F[0] = z1rho1 * v;
        F[1] = z2rho2 * v;
        F[2] = rho * v * u;
        F[3] = rho * (v * v) + pre;
    }
}

/* getLLFRiemannFlux, include/Equations.hpp:363-378 */
static void llf_flux(const ofv_eq *e, const real_t *UL, const real_t *UR, real_t *F, double nx, double ny)
{
    const int nv = ofv_nvar(e);
    const real_t ws_L = max_eig(e, UL, nx, ny);
    const real_t ws_R = max_eig(e, UR, nx, ny);
    const real_t ws = std_max(ws_L, ws_R);
    real_t FUL[4], FUR[4];
    phy_flux(e, UL, FUL, nx, ny);
    phy_flux(e, UR, FUR, nx, ny);
    for (int r = 0; r != nv; ++r)
        F[r] = 0.5 * (FUL[r] + FUR[r] - ws * (UR[r] - UL[r]));
}

/* getHLLCRiemannFlux (Zhang & Zhang 2025), include/Equations.hpp:381-483 */
static void tp_hllc_flux(const ofv_eq *e, const real_t *UL, const real_t *UR, real_t *F, double nx, double ny)
{
    real_t FUL[4], FUR[4], U[4];
    const real_t z1rho1_L = UL[0], z2rho2_L = UL[1], rhou_L = UL[2], rhov_L = UL[3];
    const real_t rho_L = z1rho1_L + z2rho2_L;
    const real_t u_L = rhou_L / rho_L;
    const real_t v_L = rhov_L / rho_L;
    const real_t z1_L = tp_volume_frac(e, UL);
    const real_t pre_L = tp_pressure_z(e, UL, z1_L);
    const real_t vn_L = u_L * nx + v_L * ny;
    const real_t c_L = tp_sound_z(e, UL, z1_L);

    const real_t z1rho1_R = UR[0], z2rho2_R = UR[1], rhou_R = UR[2], rhov_R = UR[3];
    const real_t rho_R = z1rho1_R + z2rho2_R;
    const real_t u_R = rhou_R / rho_R;
    const real_t v_R = rhov_R / rho_R;
    const real_t z1_R = tp_volume_frac(e, UR);
    const real_t pre_R = tp_pressure_z(e, UR, z1_R);
    const real_t vn_R = u_R * nx + v_R * ny;
    const real_t c_R = tp_sound_z(e, UR, z1_R);

    FUL[0] = z1rho1_L * vn_L;
    FUL[1] = z2rho2_L * vn_L;
    FUL[2] = rhou_L * vn_L + pre_L * nx;
    FUL[3] = rhov_L * vn_L + pre_L * ny;
    FUR[0] = z1rho1_R * vn_R;
    FUR[1] = z2rho2_R * vn_R;
    FUR[2] = rhou_R * vn_R + pre_R * nx;
    FUR[3] = rhov_R * vn_R + pre_R * ny;

    const real_t sL = sqrt(rho_L), sR = sqrt(rho_R);
    const real_t vn_roe = (vn_L * sL + vn_R * sR) / (sL + sR);
    real_t c2_roe = (c_L * c_L * sL + c_R * c_R * sR) / (sL + sR);
    c2_roe += 0.5 * sL * sR / (sL + sR) / (sL + sR) * (vn_R - vn_L) * (vn_R - vn_L);
    const real_t c_roe = sqrt(c2_roe);

    const real_t S_L = std_min(vn_L - c_L, vn_roe - c_roe);
    const real_t S_R = std_max(vn_R + c_R, vn_roe + c_roe);
    const real_t S_star = ((S_L - vn_L) * rho_L * vn_L - (S_R - vn_R) * rho_R * vn_R + pre_R - pre_L) /
                          ((S_L - vn_L) * rho_L - (S_R - vn_R) * rho_R);
    if (S_star >= 0) {
        if (S_L >= 0.0) {
            for (int r = 0; r != 4; r++)
                F[r] = FUL[r];
        } else {
            const real_t k = (S_L - vn_L) / (S_L - S_star);
            U[0] = z1rho1_L;
            U[1] = z2rho2_L;
            U[2] = rho_L * (u_L + (S_star - vn_L) * nx);
            U[3] = rho_L * (v_L + (S_star - vn_L) * ny);
            for (int r = 0; r != 4; r++)
                F[r] = S_L * (k * U[r] - UL[r]) + FUL[r];
        }
    } else {
        if (S_R <= 0) {
            for (int r = 0; r != 4; r++)
                F[r] = FUR[r];
        } else {
            const real_t k = (S_R - vn_R) / (S_R - S_star);
            U[0] = z1rho1_R;
            U[1] = z2rho2_R;
            U[2] = rho_R * (u_R + (S_star - vn_R) * nx);
            U[3] = rho_R * (v_R + (S_star - vn_R) * ny);
            for (int r = 0; r != 4; r++)
                F[r] = S_R * (k * U[r] - UR[r]) + FUR[r];
        }
    }
}

/* HLLC for the Euler equations (Toro, ch. 10) with Einfeldt/Roe wave-speed bounds.
 * Extension: the reference has no Euler system. */
static void eu_hllc_flux(const ofv_eq *e, const real_t *UL, const real_t *UR, real_t *F, double nx, double ny)
{
    const double g = e->gamma;
    const real_t rL = UL[0], uL = UL[1] / rL, vL = UL[2] / rL;
    const real_t rR = UR[0], uR = UR[1] / rR, vR = UR[2] / rR;
    const real_t pL = eu_pressure(e, UL), pR = eu_pressure(e, UR);
    const real_t cL = eu_sound(e, UL, pL), cR = eu_sound(e, UR, pR);
    const real_t vnL = uL * nx + vL * ny, vnR = uR * nx + vR * ny;
    const real_t HL = (UL[3] + pL) / rL, HR = (UR[3] + pR) / rR;
    const real_t sL = sqrt(rL), sR = sqrt(rR);
    const real_t inv = 1.0 / (sL + sR);
    const real_t ur = (sL * uL + sR * uR) * inv, vr = (sL * vL + sR * vR) * inv;
    const real_t Hr = (sL * HL + sR * HR) * inv;
    const real_t vnr = ur * nx + vr * ny;
    const real_t cr = sqrt((g - 1.0) * (Hr - 0.5 * (ur * ur + vr * vr)));
    const real_t S_L = std_min(vnL - cL, vnr - cr);
    const real_t S_R = std_max(vnR + cR, vnr + cr);
    const real_t S_star = (pR - pL + rL * vnL * (S_L - vnL) - rR * vnR * (S_R - vnR)) /
                          (rL * (S_L - vnL) - rR * (S_R - vnR));
    real_t FL[4], FR[4];
    phy_flux(e, UL, FL, nx, ny);
    phy_flux(e, UR, FR, nx, ny);
    if (S_L >= 0.0) {
        for (int r = 0; r < 4; r++) F[r] = FL[r];
    } else if (S_star >= 0.0) {
        const real_t k = rL * (S_L - vnL) / (S_L - S_star);
        real_t Us[4];
        Us[0] = k;
        Us[1] = k * (uL + (S_star - vnL) * nx);
        Us[2] = k * (vL + (S_star - vnL) * ny);
        Us[3] = k * (UL[3] / rL + (S_star - vnL) * (S_star + pL / (rL * (S_L - vnL))));
        for (int r = 0; r < 4; r++) F[r] = FL[r] + S_L * (Us[r] - UL[r]);
    } else if (S_R > 0.0) {
        const real_t k = rR * (S_R - vnR) / (S_R - S_star);
        real_t Us[4];
        Us[0] = k;
        Us[1] = k * (uR + (S_star - vnR) * nx);
        Us[2] = k * (vR + (S_star - vnR) * ny);
        Us[3] = k * (UR[3] / rR + (S_star - vnR) * (S_star + pR / (rR * (S_R - vnR))));
        for (int r = 0; r < 4; r++) F[r] = FR[r] + S_R * (Us[r] - UR[r]);
    } else {
        for (int r = 0; r < 4; r++) F[r] = FR[r];
    }
}

/* getRiemannFlux dispatch, include/Equations.hpp:329-343.  For the scalar advection
 * equation HLLC reduces to the upwind flux, which is the LLF flux with |a.n|. */
static void riemann(const ofv_eq *e, int flux, const real_t *UL, const real_t *UR, real_t *F, double nx, double ny)
{
    if (flux == 1 && (e->kind == OFV_EQ_TWO_PHASE || e->kind == OFV_EQ_TWO_PHASE_SG))
        tp_hllc_flux(e, UL, UR, F, nx, ny);
    else if (flux == 1 && e->kind == OFV_EQ_EULER)
        eu_hllc_flux(e, UL, UR, F, nx, ny);
    else
        llf_flux(e, UL, UR, F, nx, ny);
}

/* ------------------------------------------------------------------------------------ */
/* characteristic projections (row-major 4x4)                                             */
/* ------------------------------------------------------------------------------------ */

/* getREigenMatrix, include/Equations.hpp:189-256 */
static void tp_eigen_R(const ofv_eq *e, const real_t *U, double nx, double ny, real_t *M)
{
    const real_t z1rho1 = U[0], z2rho2 = U[1];
    const real_t rho = z1rho1 + z2rho2;
    const real_t u = U[2] / rho, v = U[3] / rho;
    const real_t z1 = tp_volume_frac(e, U);
    const real_t z2 = 1.0 - z1;
    const real_t c = tp_sound_z(e, U, z1);
    real_t c1_2, c2_2;
    tp_phase_c2(e, U, z1, &c1_2, &c2_2);
    const real_t zrho1 = z1rho1 * c1_2 / (z1 * z1);
    const real_t zrho2 = z2rho2 * c2_2 / (z2 * z2);
    const real_t sc1_2 = c1_2 / z1 - c1_2 / z1 * zrho1 / (zrho1 + zrho2);
    const real_t sc2_2 = c2_2 / z2 - c2_2 / z2 * zrho2 / (zrho1 + zrho2);
#define R_(a, b) M[(a) * 4 + (b)]
    const int xdir = fabs((real_t)nx) > fabs((real_t)ny);
    R_(0, 0) = z1rho1 / rho;
    R_(1, 0) = z2rho2 / rho;
    R_(2, 0) = xdir ? u - c : u;
    R_(3, 0) = xdir ? v : v - c;
    R_(0, 1) = -sc2_2 / (sc1_2 - sc2_2);
    R_(1, 1) = sc1_2 / (sc1_2 - sc2_2);
    R_(2, 1) = u;
    R_(3, 1) = v;
    R_(0, 2) = 0;
    R_(1, 2) = 0;
    R_(2, 2) = xdir ? 0 : 1;
    R_(3, 2) = xdir ? 1 : 0;
    R_(0, 3) = z1rho1 / rho;
    R_(1, 3) = z2rho2 / rho;
    R_(2, 3) = xdir ? u + c : u;
    R_(3, 3) = xdir ? v : v + c;
#undef R_
}

/* getLEigenMatrix, include/Equations.hpp:259-327 */
static void tp_eigen_L(const ofv_eq *e, const real_t *U, double nx, double ny, real_t *M)
{
    const real_t z1rho1 = U[0], z2rho2 = U[1];
    const real_t rho = z1rho1 + z2rho2;
    const real_t u = U[2] / rho, v = U[3] / rho;
    const real_t z1 = tp_volume_frac(e, U);
    const real_t z2 = 1.0 - z1;
    const real_t c = tp_sound_z(e, U, z1);
    const real_t c2 = c * c; /* pow(c, 2) */
    real_t c1_2, c2_2;
    tp_phase_c2(e, U, z1, &c1_2, &c2_2);
    const real_t zrho1 = z1rho1 * c1_2 / (z1 * z1);
    const real_t zrho2 = z2rho2 * c2_2 / (z2 * z2);
    const real_t sc1_2 = c1_2 / z1 - c1_2 / z1 * zrho1 / (zrho1 + zrho2);
    const real_t sc2_2 = c2_2 / z2 - c2_2 / z2 * zrho2 / (zrho1 + zrho2);
#define L_(a, b) M[(a) * 4 + (b)]
    const int xdir = fabs((real_t)nx) > fabs((real_t)ny);
    const real_t un = xdir ? u : v; /* the normal velocity of each branch */
    const real_t ut = xdir ? v : u;
    L_(0, 0) = (sc1_2 + c * un) / (2.0 * c2);
    L_(0, 1) = (sc2_2 + c * un) / (2.0 * c2);
    L_(0, 2) = xdir ? -1.0 / (2.0 * c) : (real_t)0;
    L_(0, 3) = xdir ? (real_t)0 : -1.0 / (2.0 * c);
    L_(1, 0) = -z2rho2 * (sc1_2 - sc2_2) / (rho * c2);
    L_(1, 1) = z1rho1 * (sc1_2 - sc2_2) / (rho * c2);
    L_(1, 2) = 0;
    L_(1, 3) = 0;
    L_(2, 0) = -ut;
    L_(2, 1) = -ut;
    L_(2, 2) = xdir ? 0 : 1.0;
    L_(2, 3) = xdir ? 1.0 : 0;
    L_(3, 0) = (sc1_2 - c * un) / (2.0 * c2);
    L_(3, 1) = (sc2_2 - c * un) / (2.0 * c2);
    L_(3, 2) = xdir ? 1.0 / (2.0 * c) : (real_t)0;
    L_(3, 3) = xdir ? (real_t)0 : 1.0 / (2.0 * c);
#undef L_
}

/* Euler eigenvectors in direction n = (nx, ny); extension (standard, e.g. Toro ch. 3). */
static void eu_eigen(const ofv_eq *e, const real_t *U, double nx, double ny, real_t *L, real_t *R)
{
    const double g = e->gamma;
    const real_t rho = U[0], u = U[1] / rho, v = U[2] / rho;
    const real_t p = eu_pressure(e, U);
    const real_t c = eu_sound(e, U, p);
    const real_t H = (U[3] + p) / rho;
    const real_t q2 = 0.5 * (u * u + v * v);
    const real_t vn = u * nx + v * ny, vt = v * nx - u * ny;
    if (R) {
        const real_t Rm[16] = {1.0, 1.0, 0.0, 1.0,
                               u - c * nx, u, -ny, u + c * nx,
                               v - c * ny, v, nx, v + c * ny,
                               H - c * vn, q2, vt, H + c * vn};
        for (int k = 0; k < 16; k++) R[k] = Rm[k];
    }
    if (L) {
        const real_t b1 = (g - 1.0) / (c * c), b2 = q2 * b1;
        const real_t Lm[16] = {0.5 * (b2 + vn / c), 0.5 * (-b1 * u - nx / c), 0.5 * (-b1 * v - ny / c), 0.5 * b1,
                               1.0 - b2, b1 * u, b1 * v, -b1,
                               -vt, -ny, nx, 0.0,
                               0.5 * (b2 - vn / c), 0.5 * (-b1 * u + nx / c), 0.5 * (-b1 * v + ny / c), 0.5 * b1};
        for (int k = 0; k < 16; k++) L[k] = Lm[k];
    }
}

static void eigen_L(const ofv_eq *e, const real_t *U, double nx, double ny, real_t *M)
{
    if (e->kind == OFV_EQ_EULER) eu_eigen(e, U, nx, ny, M, NULL);
    else if (e->kind == OFV_EQ_TWO_PHASE || e->kind == OFV_EQ_TWO_PHASE_SG) tp_eigen_L(e, U, nx, ny, M);
    else M[0] = 1.0;
}
static void eigen_R(const ofv_eq *e, const real_t *U, double nx, double ny, real_t *M)
{
    if (e->kind == OFV_EQ_EULER) eu_eigen(e, U, nx, ny, NULL, M);
    else if (e->kind == OFV_EQ_TWO_PHASE || e->kind == OFV_EQ_TWO_PHASE_SG) tp_eigen_R(e, U, nx, ny, M);
    else M[0] = 1.0;
}

/* Array2D * Array1D, third_party/scTools/Array.h:605-627: C[i] = 0; C[i] += A[i][j]*B[j], j ascending */
static inline void matvec(int nv, const real_t *A, const real_t *B, real_t *C)
{
    for (int i = 0; i < nv; ++i) {
        real_t s = 0.0;
        for (int j = 0; j < nv; ++j)
            s += A[i * nv + j] * B[j];
        C[i] = s;
    }
}

/* public pointwise wrappers (double in / double out) */
static void to_real(const double *a, real_t *b, int n) { for (int k = 0; k < n; k++) b[k] = a[k]; }
static void to_dbl(const real_t *a, double *b, int n) { for (int k = 0; k < n; k++) b[k] = (double)a[k]; }

double ofv_volume_frac(const ofv_eq *eq, const double *U)
{
    real_t u[4]; to_real(U, u, 4);
    return (double)tp_volume_frac(eq, u);
}
double ofv_pressure(const ofv_eq *eq, const double *U)
{
    real_t u[4]; to_real(U, u, 4);
    if (eq->kind == OFV_EQ_EULER) return (double)eu_pressure(eq, u);
    return (double)tp_pressure_z(eq, u, tp_volume_frac(eq, u));
}
double ofv_sound_speed(const ofv_eq *eq, const double *U)
{
    real_t u[4]; to_real(U, u, 4);
    if (eq->kind == OFV_EQ_EULER) return (double)eu_sound(eq, u, eu_pressure(eq, u));
    return (double)tp_sound_z(eq, u, tp_volume_frac(eq, u));
}
double ofv_max_eig(const ofv_eq *eq, const double *U, double nx, double ny)
{
    real_t u[4] = {0, 0, 0, 0}; to_real(U, u, ofv_nvar(eq));
    return (double)max_eig(eq, u, nx, ny);
}
void ofv_riemann(const ofv_eq *eq, int flux, const double *UL, const double *UR, double nx, double ny, double *F)
{
    const int nv = ofv_nvar(eq);
    real_t l[4] = {0, 0, 0, 0}, r[4] = {0, 0, 0, 0}, f[4];
    to_real(UL, l, nv); to_real(UR, r, nv);
    riemann(eq, flux, l, r, f, nx, ny);
    to_dbl(f, F, nv);
}
void ofv_eigen_L(const ofv_eq *eq, const double *U, double nx, double ny, double *L)
{
    const int nv = ofv_nvar(eq);
    real_t u[4] = {0, 0, 0, 0}, m[16];
    to_real(U, u, nv);
    eigen_L(eq, u, nx, ny, m);
    to_dbl(m, L, nv * nv);
}
void ofv_eigen_R(const ofv_eq *eq, const double *U, double nx, double ny, double *R)
{
    const int nv = ofv_nvar(eq);
    real_t u[4] = {0, 0, 0, 0}, m[16];
    to_real(U, u, nv);
    eigen_R(eq, u, nx, ny, m);
    to_dbl(m, R, nv * nv);
}

/* ------------------------------------------------------------------------------------ */
/* grid metric                                                                            */
/* ------------------------------------------------------------------------------------ */

/* Cell sizes as the reference's grid generator produces them (src/WENOFV.cpp:89-123):
 * each rank p of the x-slab decomposition builds its cells from its own ghost origin,
 * so the cell widths carry rank-dependent rounding.  dxc[i] is the width of column i,
 * dxl[i] the width of the column to its left as seen by column i's rank (they differ
 * only at slab starts), dy[j] the height of row j.  ref_slabs = 0 gives exact uniform
 * widths (the reference's m_deltaX / m_deltaY). */
void ofv_metric(const ofv_problem *p, double *dxc, double *dxl, double *dy)
{
    const double dX = (p->xr - p->xl) / p->nx;
    const double dY = (p->yr - p->yl) / p->ny;
    if (p->ref_slabs <= 0) {
        for (int i = 0; i < p->nx; i++) dxc[i] = dxl[i] = dX;
        for (int j = 0; j < p->ny; j++) dy[j] = dY;
        return;
    }
    const int m = p->nx / p->ref_slabs;
    for (int g = 0; g < p->nx; g++) {
        const int rank = g / m;
        const int ei = g - rank * m + G;
        const double procXLeft = p->xl + rank * m * dX;
        const double ghostLeft = procXLeft - dX * G;
        const double xr0 = ghostLeft + (ei + 1) * dX, xl0 = ghostLeft + ei * dX;
        const double xr1 = ghostLeft + ei * dX, xl1 = ghostLeft + (ei - 1) * dX;
        dxc[g] = xr0 - xl0;
        dxl[g] = xr1 - xl1;
    }
    const double procYLeft = p->yl + 0 * p->ny * dY;
    const double ghostBottom = procYLeft - dY * G;
    for (int j = 0; j < p->ny; j++) {
        const int ej = j + G;
        dy[j] = (ghostBottom + (ej + 1) * dY) - (ghostBottom + ej * dY);
    }
}

/* ------------------------------------------------------------------------------------ */
/* whole-grid operators                                                                   */
/* ------------------------------------------------------------------------------------ */

typedef struct {
    const ofv_problem *p;
    int nx, ny, nv, ex, H;       /* ex = nx + 2GE (extended row length), H = stencil half-width */
    real_t *E;                   /* ghost-extended averages [v][(j+GE)*ex + i+GE] */
    real_t *Y;                   /* y-sweep [(j+1)*ex + i+GE][gp*4+v], rows -1..ny */
    real_t *FS;                  /* face states [(j+1)*(nx+2) + i+1][face*16 + v*4 + gp] */
    real_t *AX, *AY;             /* face averages: AX[(j*(nx+1) + i)*4+v], AY[(j*nx + i)*4+v] */
    double *dxc, *dxl, *dy, dX, dY;
} ofv_ws;

static inline real_t *Ecell(ofv_ws *w, int v, int i, int j) { return &w->E[(size_t)v * (w->ny + 2 * GE) * w->ex + (size_t)(j + GE) * w->ex + (i + GE)]; }
static inline real_t *Ycell(ofv_ws *w, int i, int j) { return &w->Y[((size_t)(j + 1) * w->ex + (i + GE)) * 16]; }
static inline real_t *Fcell(ofv_ws *w, int i, int j) { return &w->FS[((size_t)(j + 1) * (w->nx + 2) + (i + 1)) * 64]; }

static void ws_init(ofv_ws *w, const ofv_problem *p)
{
    w->p = p;
    w->nx = p->nx; w->ny = p->ny; w->nv = ofv_nvar(&p->eq); w->ex = p->nx + 2 * GE;
    w->H = (p->scheme == 2 || p->recon == 4) ? 3 : 2;
    w->E = (real_t *)calloc((size_t)w->nv * w->ex * (p->ny + 2 * GE), sizeof(real_t));
    w->Y = (real_t *)calloc((size_t)w->ex * (p->ny + 2) * 16, sizeof(real_t));
    w->FS = (real_t *)calloc((size_t)(p->nx + 2) * (p->ny + 2) * 64, sizeof(real_t));
    w->AX = (real_t *)calloc((size_t)(p->nx + 1) * p->ny * 4, sizeof(real_t));
    w->AY = (real_t *)calloc((size_t)p->nx * (p->ny + 1) * 4, sizeof(real_t));
    w->dxc = (double *)malloc(sizeof(double) * p->nx);
    w->dxl = (double *)malloc(sizeof(double) * p->nx);
    w->dy = (double *)malloc(sizeof(double) * p->ny);
    ofv_metric(p, w->dxc, w->dxl, w->dy);
    w->dX = (p->xr - p->xl) / p->nx;
    w->dY = (p->yr - p->yl) / p->ny;
}
static void ws_free(ofv_ws *w)
{
    free(w->E); free(w->Y); free(w->FS); free(w->AX); free(w->AY);
    free(w->dxc); free(w->dxl); free(w->dy);
}

/* Ghost fill.  PERIOD reproduces the ring exchange plus the periodic y copy over the full
 * extended x range (src/WENOFV.cpp:2175-2269), i.e. a 2-D periodic wrap including corners.
 * OUTFLOW (extension) is a zero-gradient copy of the nearest interior cell.  The walls
 * NEUMANN / FREESLIP (the normal momentum negated) and NOSLIP (both momenta negated), which
 * the reference declares but does not implement, mirror the interior across the boundary
 * (again for grids narrower than the halo), a sign change per reflection.  NEUMANN2, also
 * declared and not implemented there, reads each ghost cell from a fixed frame of averages
 * (the initial data around the domain), the same for every stage. */
static int mirror(int k, int n, int *flips)
{
    *flips = 0;
    for (int it = 0; it < 64 && (k < 0 || k >= n); it++) {
        k = k < 0 ? -1 - k : 2 * n - 1 - k;
        (*flips)++;
    }
    return k < 0 ? 0 : (k >= n ? n - 1 : k);
}
static void fill_ghosts(ofv_ws *w, const double *U)
{
    const int nx = w->nx, ny = w->ny;
    for (int v = 0; v < w->nv; v++)
        for (int j = -GE; j < ny + GE; j++)
            for (int i = -GE; i < nx + GE; i++) {
                int si, sj;
                double sign = 1.0;
                const int bc = w->p->bc;
                if (bc == OFV_BC_OUTFLOW) {
                    si = i < 0 ? 0 : (i >= nx ? nx - 1 : i);
                    sj = j < 0 ? 0 : (j >= ny ? ny - 1 : j);
                } else if (bc == OFV_BC_NEUMANN || bc == OFV_BC_NOSLIP || bc == OFV_BC_FREESLIP) {
                    int fx, fy;
                    si = mirror(i, nx, &fx);
                    sj = mirror(j, ny, &fy);
                    const int kind = w->p->eq.kind;
                    const int mx = kind == OFV_EQ_EULER ? 1 : 2, my = mx + 1;
                    int nflip = 0;
                    if (kind != OFV_EQ_LINEAR_ADV) {
                        if (v == mx) nflip = fx + (bc == OFV_BC_NOSLIP ? fy : 0);
                        else if (v == my) nflip = fy + (bc == OFV_BC_NOSLIP ? fx : 0);
                    }
                    if (nflip & 1) sign = -1.0;
                } else if (bc == OFV_BC_NEUMANN2) {
                    if (i < 0 || i >= nx || j < 0 || j >= ny) {
                        const size_t fw = (size_t)nx + 8, fplane = fw * ((size_t)ny + 8);
                        *Ecell(w, v, i, j) = w->p->frame[v * fplane + (size_t)(j + 4) * fw + (size_t)(i + 4)];
                        continue;
                    }
                    si = i;
                    sj = j;
                } else { /* a true modulo: grids narrower than the 3 ghost layers wrap more than once */
                    si = ((i % nx) + nx) % nx;
                    sj = ((j % ny) + ny) % ny;
                }
                *Ecell(w, v, i, j) = sign * U[(size_t)v * nx * ny + (size_t)sj * nx + si];
            }
}

static void cell_avg(ofv_ws *w, int i, int j, real_t *u)
{
    for (int v = 0; v < w->nv; v++) u[v] = *Ecell(w, v, i, j);
}

/* Primitive variables of the two-phase model for RECONSTRUCTIONTYPE 2 (PRIMITIVE: z1,
 * rho1, u, v; src/WENOFV.cpp:944-959) and 3 (PRIMITIVE2: z1, p, u, v; :1102-1121), and
 * their inverse at the Gauss points (:1002-1025 and :1178-1189). */
static void to_primitive(const ofv_eq *e, int recon, const real_t *U, real_t *P)
{
    const real_t z1 = tp_volume_frac(e, U);
    P[0] = z1;
    if (recon == 2) {
        P[1] = U[0] / z1;
    } else {
        const real_t c1_2 = (real_t)e->sound1 * e->sound1, c2_2 = (real_t)e->sound2 * e->sound2;
        if (z1 > 0.5)
            P[1] = e->preb + c1_2 * (U[0] / z1 - e->rho10);
        else
            P[1] = e->preb + c2_2 * (U[1] / (1.0 - z1) - e->rho20);
    }
    P[2] = U[2] / (U[0] + U[1]);
    P[3] = U[3] / (U[0] + U[1]);
}
static void from_primitive(const ofv_eq *e, int recon, const real_t *P, real_t *U)
{
    const real_t z1 = P[0];
    const real_t c1_2 = (real_t)e->sound1 * e->sound1, c2_2 = (real_t)e->sound2 * e->sound2;
    real_t z1rho1, z2rho2;
    if (recon == 2) {
        const real_t rho1 = P[1];
        z2rho2 = c1_2 / c2_2 * (rho1 - e->rho10) + e->rho20;
        z2rho2 = z2rho2 * (1.0 - z1);
        z1rho1 = z1 * rho1;
    } else {
        const real_t pr = P[1];
        z1rho1 = ((pr - e->preb) / c1_2 + e->rho10) * z1;
        z2rho2 = ((pr - e->preb) / c2_2 + e->rho20) * (1.0 - z1);
    }
    const real_t rho = z1rho1 + z2rho2;
    U[0] = z1rho1;
    U[1] = z2rho2;
    U[2] = rho * P[2];
    U[3] = rho * P[3];
}

/* y-direction sweep of one column position (src/WENOFV.cpp:670-687 conservative,
 * :796-833 characteristic, :963-979 primitive): 4 Gauss-Lobatto y points x nv variables */
static void y_sweep(ofv_ws *w, int i, int j)
{
    const ofv_problem *p = w->p;
    const int nv = w->nv, m0 = 3 - w->H, m1 = 3 + w->H; /* stencil slots m0..m1 of 7 */
    real_t *out = Ycell(w, i, j);
    if (p->recon == 1 && nv > 1) {
        real_t uc[4], L[16], R[16], pr[7][4], col[7][4], st[7], cg[4][4];
        cell_avg(w, i, j, uc);
        eigen_L(&p->eq, uc, 0, 1, L);
        eigen_R(&p->eq, uc, 0, 1, R);
        for (int m = m0; m <= m1; m++) {
            cell_avg(w, i, j - 3 + m, col[m]);
            matvec(nv, L, col[m], pr[m]);
        }
        for (int gp = 0; gp < 4; gp++) {
            for (int k = 0; k < nv; k++) {
                for (int m = m0; m <= m1; m++) st[m] = pr[m][k];
                cg[gp][k] = weno7(p->scheme, st, gp, w->dX);
            }
            real_t phys[4];
            matvec(nv, R, cg[gp], phys);
            for (int v = 0; v < nv; v++) out[gp * 4 + v] = phys[v];
        }
    } else if (p->recon >= 2 && nv > 1) {
        real_t col[7][4], prim[7][4], st[7];
        for (int m = m0; m <= m1; m++) {
            cell_avg(w, i, j - 3 + m, col[m]);
            to_primitive(&p->eq, p->recon, col[m], prim[m]);
        }
        for (int v = 0; v < nv; v++) {
            for (int m = m0; m <= m1; m++) st[m] = prim[m][v];
            for (int gp = 0; gp < 4; gp++) out[gp * 4 + v] = weno7_var(p->scheme, p->recon, v, st, gp, w->dX);
        }
    } else {
        real_t st[7];
        for (int v = 0; v < nv; v++) {
            for (int m = m0; m <= m1; m++) st[m] = *Ecell(w, v, i, j - 3 + m);
            for (int gp = 0; gp < 4; gp++) out[gp * 4 + v] = weno7(p->scheme, st, gp, w->dX);
        }
    }
}

/* getPositivityPreservingTheta + the scaling of useBoundPreservingLimiter,
 * src/WENOFV.cpp:1895-2000.  fs = [face B,T,L,R][v][gp]; returns the limiter flag. */
static int pp_limit(ofv_ws *w, const real_t *ubar, real_t *fs)
{
    const ofv_eq *e = &w->p->eq;
    const int nv = w->nv;
    const int nlim = (e->kind == OFV_EQ_TWO_PHASE || e->kind == OFV_EQ_TWO_PHASE_SG) ? 2 : (e->kind == OFV_EQ_EULER ? 1 : 0);
    if (nlim == 0) return 0;
    const double zeps = 1e-12, omega1 = 0.1, omegaR = 1.0 - 2 * omega1;
    const real_t a1 = max_eig(e, ubar, 1, 0);
    const real_t a2 = max_eig(e, ubar, 0, 1);
    const real_t mu1 = (a1 / w->dX) / (a1 / w->dX + a2 / w->dY);
    const real_t mu2 = (a2 / w->dY) / (a1 / w->dX + a2 / w->dY);
    real_t th[2];
    for (int r = 0; r < nlim; r++) {
        th[r] = 1.0;
        const real_t uave = ubar[r];
        const real_t eps = std_min(zeps, uave);
        real_t rem = uave;
        const real_t *B = fs + 0 * 16 + r * 4, *T = fs + 1 * 16 + r * 4;
        const real_t *Lf = fs + 2 * 16 + r * 4, *Rf = fs + 3 * 16 + r * 4;
        for (int gp = 0; gp != 4; gp++) {
            rem -= omega1 * GL_W[gp] / 2 * mu2 * B[gp];
            rem -= omega1 * GL_W[gp] / 2 * mu2 * T[gp];
            rem -= omega1 * GL_W[gp] / 2 * mu1 * Lf[gp];
            rem -= omega1 * GL_W[gp] / 2 * mu1 * Rf[gp];
        }
        rem /= omegaR;
        real_t mloc = rem;
        for (int gp = 0; gp != 4; gp++) {
            mloc = sc_min(mloc, B[gp]);
            mloc = sc_min(mloc, T[gp]);
            mloc = sc_min(mloc, Lf[gp]);
            mloc = sc_min(mloc, Rf[gp]);
        }
        th[r] = sc_min(fabs((uave - eps) / (uave - mloc)), th[r]);
    }
    const real_t theta = nlim == 2 ? sc_min(th[0], th[1]) : th[0];
    const int flag = theta < 1 - 1e-8;
    if (theta >= 0.0 && theta <= 1.0) {
        for (int f = 0; f < 4; f++)
            for (int v = 0; v < nv; v++)
                for (int gp = 0; gp < 4; gp++) {
                    real_t *x = &fs[f * 16 + v * 4 + gp];
                    *x = theta * (*x - ubar[v]) + ubar[v];
                }
    }
    return flag;
}

/* x-direction sweep of one cell (src/WENOFV.cpp:690-721 conservative, :836-880
 * characteristic) followed by the limiter; writes the cell's face states. */
static int x_sweep(ofv_ws *w, int i, int j)
{
    const ofv_problem *p = w->p;
    const int nv = w->nv;
    real_t ugp[4][4][4]; /* [gpi][gpj][v] */
    real_t *fs = Fcell(w, i, j);
    real_t uc[4];
    cell_avg(w, i, j, uc);
    const int m0 = 3 - w->H, m1 = 3 + w->H; /* stencil slots m0..m1 of 7 */
    if (p->recon == 1 && nv > 1) {
        real_t L[16], R[16], tc[7][4][4], st[7], c[4];
        eigen_L(&p->eq, uc, 1, 0, L);
        eigen_R(&p->eq, uc, 1, 0, R);
        for (int m = m0; m <= m1; m++) {
            const real_t *y = Ycell(w, i - 3 + m, j);
            for (int gp = 0; gp < 4; gp++) matvec(nv, L, y + gp * 4, tc[m][gp]);
        }
        for (int gpj = 0; gpj < 4; gpj++)
            for (int gpi = 0; gpi < 4; gpi++) {
                if (!(gpi == 0 || gpi == 3 || gpj == 0 || gpj == 3)) continue;
                for (int k = 0; k < nv; k++) {
                    for (int m = m0; m <= m1; m++) st[m] = tc[m][gpj][k];
                    c[k] = weno7(p->scheme, st, gpi, w->dX);
                }
                matvec(nv, R, c, ugp[gpi][gpj]);
            }
    } else {
        real_t st[7];
        for (int gpj = 0; gpj < 4; gpj++)
            for (int v = 0; v < nv; v++) {
                for (int m = m0; m <= m1; m++) st[m] = Ycell(w, i - 3 + m, j)[gpj * 4 + v];
                for (int gpi = 0; gpi < 4; gpi++) {
                    if (!(gpi == 0 || gpi == 3 || gpj == 0 || gpj == 3)) continue;
                    ugp[gpi][gpj][v] = weno7_var(p->scheme, p->recon, v, st, gpi, w->dX);
                }
            }
        if (p->recon >= 2 && nv > 1) /* the primitive values back to conservative ones */
            for (int gpi = 0; gpi < 4; gpi++)
                for (int gpj = 0; gpj < 4; gpj++) {
                    if (!(gpi == 0 || gpi == 3 || gpj == 0 || gpj == 3)) continue;
                    real_t prim[4];
                    for (int v = 0; v < 4; v++) prim[v] = ugp[gpi][gpj][v];
                    from_primitive(&p->eq, p->recon, prim, ugp[gpi][gpj]);
                }
    }
    for (int v = 0; v < nv; v++)
        for (int gp = 0; gp < 4; gp++) {
            fs[0 * 16 + v * 4 + gp] = ugp[gp][0][v]; /* bottom */
            fs[1 * 16 + v * 4 + gp] = ugp[gp][3][v]; /* top */
            fs[2 * 16 + v * 4 + gp] = ugp[0][gp][v]; /* left */
            fs[3 * 16 + v * 4 + gp] = ugp[3][gp][v]; /* right */
        }
    if (p->limiter) return pp_limit(w, uc, fs);
    return 0;
}

/* reconstruction of all needed face states: interior cells plus the one-cell halo ring */
static void reconstruct(ofv_ws *w, const double *U, double *theta_flags)
{
    const int nx = w->nx, ny = w->ny;
    fill_ghosts(w, U);
    int j;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (j = -1; j <= ny; j++)
        for (int i = -1 - w->H; i <= nx + w->H; i++) {
            /* halo rows only need columns -H..nx-1+H (their cells need no x-halo) */
            if ((j < 0 || j >= ny) && (i < -w->H || i > nx - 1 + w->H)) continue;
            y_sweep(w, i, j);
        }
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (j = -1; j <= ny; j++)
        for (int i = -1; i <= nx; i++) {
            const int halo_row = (j < 0 || j >= ny), halo_col = (i < 0 || i >= nx);
            if (halo_row && halo_col) continue;
            const int flag = x_sweep(w, i, j);
            if (theta_flags && !halo_row && !halo_col) theta_flags[(size_t)j * nx + i] = flag;
        }
}

void ofv_face_states(const ofv_problem *p, const double *U, double *out)
{
    ofv_ws w;
    ws_init(&w, p);
    reconstruct(&w, U, NULL);
    for (int j = 0; j < p->ny; j++)
        for (int i = 0; i < p->nx; i++) {
            const real_t *fs = Fcell(&w, i, j);
            for (int f = 0; f < 4; f++)
                for (int v = 0; v < w.nv; v++)
                    for (int gp = 0; gp < 4; gp++)
                        out[((size_t)j * p->nx + i) * 16 * w.nv + f * 4 * w.nv + v * 4 + gp] = (double)fs[f * 16 + v * 4 + gp];
        }
    ws_free(&w);
}

/* assembleRHS (src/WENOFV.cpp:568-615) after reconstruction: Riemann fluxes at every face
 * Gauss-Lobatto point, GL quadrature and the scatter to the two neighbours
 * (assembleBoundaryFaceTerm, src/WENOFV.cpp:1670-1829).  Source term: none for the
 * runnable cases (src/WENOFV.cpp:1831-1872). */
static void rhs_ws(ofv_ws *w, const double *U, double *rhs, double *theta_flags)
{
    const ofv_problem *p = w->p;
    const int nx = w->nx, ny = w->ny, nv = w->nv;
    reconstruct(w, U, theta_flags);
    int j;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (j = 0; j < ny; j++) {
        for (int i = 0; i <= nx; i++) { /* x-face between cells i-1 and i */
            const real_t *fl = Fcell(w, i - 1, j), *fr = Fcell(w, i, j);
            real_t ave[4] = {0.0, 0.0, 0.0, 0.0};
            for (int gp = 0; gp < 4; gp++) {
                real_t UL[4], UR[4], F[4];
                for (int v = 0; v < nv; v++) {
                    UL[v] = fl[3 * 16 + v * 4 + gp]; /* right face of the left cell */
                    UR[v] = fr[2 * 16 + v * 4 + gp]; /* left face of the right cell */
                }
                riemann(&p->eq, p->flux, UL, UR, F, 1, 0);
                const double gw = GL_W[gp] * w->dy[j] / 2.0;
                for (int v = 0; v < nv; v++) ave[v] += F[v] * gw;
            }
            for (int v = 0; v < nv; v++) w->AX[((size_t)j * (nx + 1) + i) * 4 + v] = ave[v];
        }
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (j = 0; j <= ny; j++) { /* y-face between rows j-1 and j */
        for (int i = 0; i < nx; i++) {
            const real_t *fb = Fcell(w, i, j - 1), *ft = Fcell(w, i, j);
            real_t ave[4] = {0.0, 0.0, 0.0, 0.0};
            for (int gp = 0; gp < 4; gp++) {
                real_t UL[4], UR[4], F[4];
                for (int v = 0; v < nv; v++) {
                    UL[v] = fb[1 * 16 + v * 4 + gp]; /* top face of the lower cell */
                    UR[v] = ft[0 * 16 + v * 4 + gp]; /* bottom face of the upper cell */
                }
                riemann(&p->eq, p->flux, UL, UR, F, 0, 1);
                const double gw = GL_W[gp] * w->dxc[i] / 2.0;
                for (int v = 0; v < nv; v++) ave[v] += F[v] * gw;
            }
            for (int v = 0; v < nv; v++) w->AY[((size_t)j * nx + i) * 4 + v] = ave[v];
        }
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            for (int v = 0; v < nv; v++) {
                const real_t aL = w->AX[((size_t)j * (nx + 1) + i) * 4 + v];
                const real_t aR = w->AX[((size_t)j * (nx + 1) + i + 1) * 4 + v];
                const real_t aB = w->AY[((size_t)j * nx + i) * 4 + v];
                const real_t aT = w->AY[((size_t)(j + 1) * nx + i) * 4 + v];
                real_t r = 0.0;
                r += aL / w->dxl[i] / w->dy[j];
                r += -aR / w->dxc[i] / w->dy[j];
                r += aB / w->dxc[i] / w->dy[j];
                r -= aT / w->dxc[i] / w->dy[j];
                if (v == 3 && p->eq.gravity != 0.0 && (p->eq.kind == OFV_EQ_TWO_PHASE || p->eq.kind == OFV_EQ_TWO_PHASE_SG)) {
                    /* assembleSourceTerm, src/WENOFV.cpp:1843-1853 */
                    const size_t k = (size_t)j * nx + i;
                    const real_t rho = (real_t)U[k] + (real_t)U[(size_t)nx * ny + k];
                    r -= rho * p->eq.gravity;
                }
                rhs[(size_t)v * nx * ny + (size_t)j * nx + i] = (double)r;
            }
}

void ofv_rhs(const ofv_problem *p, const double *U, double *rhs, double *theta_flags)
{
#ifdef _OPENMP
    if (p->threads > 0) omp_set_num_threads(p->threads);
#endif
    ofv_ws w;
    ws_init(&w, p);
    rhs_ws(&w, U, rhs, theta_flags);
    ws_free(&w);
}

/* calculateDeltaT, src/WENOFV.cpp:474-540 (without the MPI min, which is exact) */
double ofv_compute_dt(const ofv_problem *p, const double *U, int *nan_flag)
{
    const int nx = p->nx, ny = p->ny, nv = ofv_nvar(&p->eq);
    const double dX = (p->xr - p->xl) / nx, dY = (p->yr - p->yl) / ny;
    real_t timestep = 1.0;
    int nan = 0;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            real_t u[4];
            for (int v = 0; v < nv; v++) u[v] = U[(size_t)v * nx * ny + (size_t)j * nx + i];
            const real_t ex = max_eig(&p->eq, u, 1, 0);
            const real_t ey = max_eig(&p->eq, u, 0, 1);
            const real_t tmp = p->cfl / (ex / dX + ey / dY);
            if (OFV_ISNAN(tmp)) nan = 1;
            if (tmp > timestep) continue;
            timestep = tmp;
        }
    if (nan_flag) *nan_flag = nan;
    return (double)timestep;
}

/* performTimeIntegration / RunRK1-3, src/WENOFV.cpp:376-473, 541-566 */
void ofv_step(const ofv_problem *p, double *U, double dt)
{
#ifdef _OPENMP
    if (p->threads > 0) omp_set_num_threads(p->threads);
#endif
    const size_t n = (size_t)ofv_nvar(&p->eq) * p->nx * p->ny;
    double *rhs = (double *)malloc(sizeof(double) * n);
    ofv_ws w;
    ws_init(&w, p);
    if (p->rk == 0) {
        rhs_ws(&w, U, rhs, NULL);
        for (size_t k = 0; k < n; k++) U[k] += dt * rhs[k];
    } else {
        double *Un = (double *)malloc(sizeof(double) * n);
        memcpy(Un, U, sizeof(double) * n);
        const int ns = p->rk == 1 ? 2 : 3;
        static const double A2[2] = {1.0, 0.5}, B2[2] = {0.0, 0.5}, C2[2] = {1.0, 0.5};
        const double A3[3] = {1.0, 3.0 / 4.0, 1.0 / 3.0}, B3[3] = {0.0, 1.0 / 4.0, 2.0 / 3.0},
                     C3[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
        for (int s = 0; s < ns; s++) {
            rhs_ws(&w, U, rhs, NULL);
            const double a = ns == 2 ? A2[s] : A3[s], b = ns == 2 ? B2[s] : B3[s], c = ns == 2 ? C2[s] : C3[s];
            for (size_t k = 0; k < n; k++) U[k] = a * Un[k] + b * U[k] + c * dt * rhs[k];
        }
        free(Un);
    }
    ws_free(&w);
    free(rhs);
}

/* the inner loop of CWENOFV::run to one target time, src/WENOFV.cpp:320-332 */
int ofv_advance(const ofv_problem *p, double *U, double t0, double t_end, double *t_out, int max_steps, double *dts)
{
    double now = t0;
    int count = 0;
    while (fabs(now - t_end) > 1e-10 && (max_steps <= 0 || count < max_steps)) {
        const double remaining = t_end - now;
        double timestep = ofv_compute_dt(p, U, NULL);
        timestep = (remaining < timestep) ? remaining : timestep; /* std::min */
        ofv_step(p, U, timestep);
        if (dts) dts[count] = timestep;
        now += timestep;
        count++;
    }
    if (t_out) *t_out = now;
    return count;
}
