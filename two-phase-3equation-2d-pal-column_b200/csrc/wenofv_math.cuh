// wenofv_math.cuh -- pointwise device kernels of the WENOFV hot path (sm_100a).
//
// Compiled twice: WENOFV_STRICT=1 with -fmad=false reproduces the reference's FP64
// operation order exactly (no contraction, every division and sqrt where the reference
// has it); WENOFV_STRICT=0 lets the compiler contract into FMAs and uses reciprocals
// where the reference divides repeatedly by the same value.  Real is double, or float for
// the FP32-bulk form (whose pressure recovery stays FP64).
//
// Citations are path:line inside the reference project.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "wenofv_types.h"

#ifndef WENOFV_STRICT
#error "define WENOFV_STRICT (0 or 1)"
#endif

namespace wenofv {
#if WENOFV_STRICT
namespace strict {
#else
namespace fast {
#endif

// std::min / std::max (used unqualified by the reference via `using namespace std`)
template <class R> __device__ __forceinline__ R std_min(R a, R b) { return (b < a) ? b : a; }
template <class R> __device__ __forceinline__ R std_max(R a, R b) { return (a < b) ? b : a; }
// sc_math::Min, third_party/scTools/MyMath.h:52-55
template <class R> __device__ __forceinline__ R sc_min(R a, R b) { return (a < b) ? a : b; }
// the spread of an FP32 WENO stencil by fminf/fmaxf (one instruction each, where the
// compare-and-select of std::min takes two; a NaN in the stencil still reaches the result
// through the smoothness indicators); FP64 keeps the reference's std::min/std::max, which
// measured faster than fmin/fmax for doubles here
template <class R> __device__ __forceinline__ R spread_min(R a, R b)
{
    if constexpr (sizeof(R) < sizeof(double)) return fminf(a, b);
    else return std_min(a, b);
}
template <class R> __device__ __forceinline__ R spread_max(R a, R b)
{
    if constexpr (sizeof(R) < sizeof(double)) return fmaxf(a, b);
    else return std_max(a, b);
}

// ------------------------------------------------------------------------------------
// WENO at Gauss-Lobatto points (include/Utility.hpp:5-95 JS, :193-290 Z)
// ------------------------------------------------------------------------------------

// linear weights, include/Utility.hpp:12-39
template <class R, int GP> __device__ __forceinline__ void weno_d(R &d0, R &d1, R &d2)
{
    if (GP == 0) { d0 = R(0.3); d1 = R(0.6); d2 = R(0.1); }
    else if (GP == 1) { d0 = R((91.0 - 9.0 * sqrt(5.0)) / 440.0); d1 = R(129.0 / 220.0); d2 = R((91.0 + 9.0 * sqrt(5.0)) / 440.0); }
    else if (GP == 2) { d0 = R((91.0 + 9.0 * sqrt(5.0)) / 440.0); d1 = R(129.0 / 220.0); d2 = R((91.0 - 9.0 * sqrt(5.0)) / 440.0); }
    else { d0 = R(0.1); d1 = R(0.6); d2 = R(0.3); }
}

// candidate polynomials, include/Utility.hpp:64-90 (coefficients folded in double)
template <class R, int GP>
__device__ __forceinline__ void weno_h(R umm, R um, R u, R up, R upp, R &h0, R &h1, R &h2)
{
    if (GP == 0) {
        h0 = R(-1.0 / 6.0) * umm + R(5.0 / 6.0) * um + R(1.0 / 3.0) * u;
        h1 = R(1.0 / 3.0) * um + R(5.0 / 6.0) * u - R(1.0 / 6) * up;
        h2 = R(11.0 / 6.0) * u - R(7.0 / 6.0) * up + R(1.0 / 3.0) * upp;
    } else if (GP == 1) {
        h0 = R(-1.0 / 60.0 - sqrt(5.0) / 20.0) * umm + R(1.0 / 30.0 + sqrt(5.0) / 5.0) * um +
             R(59.0 / 60.0 - 3 * sqrt(5.0) / 20.0) * u;
        h1 = R(-1.0 / 60.0 + sqrt(5.0) / 20.0) * um + R(31.0 / 30.0) * u + R(-1.0 / 60 - sqrt(5.0) / 20.0) * up;
        h2 = R(59.0 / 60.0 + 3 * sqrt(5.0) / 20) * u + R(1.0 / 30.0 - sqrt(5.0) / 5.0) * up +
             R(-1.0 / 60.0 + sqrt(5.0) / 20.0) * upp;
    } else if (GP == 2) {
        h0 = R(-1.0 / 60.0 + sqrt(5.0) / 20.0) * umm + R(1.0 / 30.0 - sqrt(5.0) / 5.0) * um +
             R(59.0 / 60.0 + 3 * sqrt(5.0) / 20) * u;
        h1 = R(-1.0 / 60 - sqrt(5.0) / 20.0) * um + R(31.0 / 30.0) * u + R(-1.0 / 60.0 + sqrt(5.0) / 20.0) * up;
        h2 = R(59.0 / 60.0 - 3 * sqrt(5.0) / 20.0) * u + R(1.0 / 30.0 + sqrt(5.0) / 5.0) * up +
             R(-1.0 / 60.0 - sqrt(5.0) / 20.0) * upp;
    } else {
        h0 = R(1.0 / 3.0) * umm - R(7.0 / 6.0) * um + R(11.0 / 6.0) * u;
        h1 = R(-1.0 / 6) * um + R(5.0 / 6.0) * u + R(1.0 / 3.0) * up;
        h2 = R(1.0 / 3.0) * u + R(5.0 / 6.0) * up - R(1.0 / 6.0) * upp;
    }
}

template <class R> __device__ __forceinline__ void weno_betas(R umm, R um, R u, R up, R upp, R &b0, R &b1, R &b2)
{
    const R t0 = umm - R(4) * um + R(3) * u, s0 = umm - R(2) * um + u;
    const R t1 = um - up, s1 = um - R(2) * u + up;
    const R t2 = R(3) * u - R(4) * up + upp, s2 = u - R(2) * up + upp;
    // pow(x, 2) of include/Utility.hpp:48-50 / :271-273 is x*x
    b0 = R(0.25) * (t0 * t0) + R(13.0 / 12.0) * (s0 * s0);
    b1 = R(0.25) * (t1 * t1) + R(13.0 / 12.0) * (s1 * s1);
    b2 = R(0.25) * (t2 * t2) + R(13.0 / 12.0) * (s2 * s2);
}

// One 5-point stencil prepared once and evaluated at several Gauss-Lobatto points: the
// smoothness indicators (and WENO-Z's normalisation) depend on the stencil only, so they
// are shared across points, which reproduces the per-point reference calls bit for bit.
// ZS: the scheme as a compile-time constant (0 WENO-JS, 1 WENO-Z) in the stage kernels, or -1
// to take it from init's argument (the pointwise probes)
template <class R, int ZS = -1> struct Weno5 {
    R umm, um, u, up, upp; // raw values (candidate polynomials use these)
    R g0, g1, g2;          // JS: (eps+beta_k)^2 [strict] or 1/(eps+beta_k)^2 [fast]; Z: 1 + tau/(beta_k+eps)
    int z;

    // contracted FP64 build: one division for the three weights of a stencil and one for
    // the normalisations of all Gauss points evaluated from it (products of the
    // denominators, all bounded away from 0 and far below overflow), and WENO-Z without
    // normalising the stencil: beta is quadratic and translation invariant, so beta(n) =
    // beta(v) / s^2 with s = umax - umin + 1e-20, and tau/(beta(n) + eps) =
    // tau(v)/(beta(v) + eps s^2)
    static constexpr bool SHARED = !WENOFV_STRICT && sizeof(R) == sizeof(double);

    __device__ __forceinline__ void init(int scheme, R v0, R v1, R v2, R v3, R v4)
    {
        umm = v0; um = v1; u = v2; up = v3; upp = v4;
        const int sch = ZS < 0 ? scheme : ZS;
        z = sch;
        if constexpr (SHARED) {
            R b0, b1, b2;
            weno_betas(v0, v1, v2, v3, v4, b0, b1, b2);
            R a0, a1, a2;
            if (sch == 1) {
                const R umax = spread_max(spread_max(spread_max(v0, v1), spread_max(v4, v3)), v2);
                const R umin = spread_min(spread_min(spread_min(v0, v1), spread_min(v4, v3)), v2);
                const R sc = umax - umin + R(1e-20);
                const R e2 = R(1.0e-10) * sc * sc;
                a0 = b0 + e2; a1 = b1 + e2; a2 = b2 + e2;
            } else {
                a0 = (R(1.0e-6) + b0) * (R(1.0e-6) + b0);
                a1 = (R(1.0e-6) + b1) * (R(1.0e-6) + b1);
                a2 = (R(1.0e-6) + b2) * (R(1.0e-6) + b2);
            }
            const R a01 = a0 * a1;
            const R inv = R(1) / (a01 * a2);
            const R r0 = a1 * a2 * inv, r1 = a0 * a2 * inv, r2 = a01 * inv;
            if (sch == 1) {
                const R tau = fabs(b0 - b2);
                g0 = R(1) + tau * r0; g1 = R(1) + tau * r1; g2 = R(1) + tau * r2;
            } else {
                g0 = r0; g1 = r1; g2 = r2;
            }
            return;
        }
        if (sch == 1) {
            // WENO-Z: normalise the stencil to [0,1], include/Utility.hpp:261-268
            const R umax = spread_max(spread_max(spread_max(v0, v1), spread_max(v4, v3)), v2);
            const R umin = spread_min(spread_min(spread_min(v0, v1), spread_min(v4, v3)), v2);
            R n0, n1, n2, n3, n4;
#if WENOFV_STRICT
            n0 = (v0 - umin) / (umax - umin + R(1e-20));
            n1 = (v1 - umin) / (umax - umin + R(1e-20));
            n2 = (v2 - umin) / (umax - umin + R(1e-20));
            n3 = (v3 - umin) / (umax - umin + R(1e-20));
            n4 = (v4 - umin) / (umax - umin + R(1e-20));
#else
            const R inv = R(1) / (umax - umin + R(1e-20));
            n0 = (v0 - umin) * inv; n1 = (v1 - umin) * inv; n2 = (v2 - umin) * inv;
            n3 = (v3 - umin) * inv; n4 = (v4 - umin) * inv;
#endif
            R b0, b1, b2;
            weno_betas(n0, n1, n2, n3, n4, b0, b1, b2);
            const R eps = R(1.0e-10);
            const R tau = fabs(b0 - b2);
            g0 = R(1) + tau / (b0 + eps);
            g1 = R(1) + tau / (b1 + eps);
            g2 = R(1) + tau / (b2 + eps);
        } else {
            R b0, b1, b2;
            weno_betas(v0, v1, v2, v3, v4, b0, b1, b2);
            const R eps = R(1.0e-6);
#if WENOFV_STRICT
            g0 = (eps + b0) * (eps + b0);
            g1 = (eps + b1) * (eps + b1);
            g2 = (eps + b2) * (eps + b2);
#else
            g0 = R(1) / ((eps + b0) * (eps + b0));
            g1 = R(1) / ((eps + b1) * (eps + b1));
            g2 = R(1) / ((eps + b2) * (eps + b2));
#endif
        }
    }

    template <int GP> __device__ __forceinline__ R eval() const
    {
        R d0, d1, d2, h0, h1, h2;
        weno_d<R, GP>(d0, d1, d2);
        weno_h<R, GP>(umm, um, u, up, upp, h0, h1, h2);
        R w0, w1, w2;
        if ((ZS < 0 ? z : ZS) != 0) {
            w0 = d0 * g0; w1 = d1 * g1; w2 = d2 * g2;
        } else {
#if WENOFV_STRICT
            w0 = d0 / g0; w1 = d1 / g1; w2 = d2 / g2;
#else
            w0 = d0 * g0; w1 = d1 * g1; w2 = d2 * g2;
#endif
        }
        const R sum = w0 + w1 + w2;
#if WENOFV_STRICT
        w0 = w0 / sum; w1 = w1 / sum; w2 = w2 / sum;
        return w0 * h0 + w1 * h1 + w2 * h2;
#else
        return (w0 * h0 + w1 * h1 + w2 * h2) / sum;
#endif
    }

    // numerator and denominator of the value at GP (the shared-division form)
    template <int GP> __device__ __forceinline__ R num_den(R &den) const
    {
        R d0, d1, d2, h0, h1, h2;
        weno_d<R, GP>(d0, d1, d2);
        weno_h<R, GP>(umm, um, u, up, upp, h0, h1, h2);
        const R w0 = d0 * g0, w1 = d1 * g1, w2 = d2 * g2;
        den = w0 + w1 + w2;
        return w0 * h0 + w1 * h1 + w2 * h2;
    }
    // the values at all four Gauss-Lobatto points
    __device__ __forceinline__ void eval4(R *o) const
    {
        if constexpr (SHARED) {
            R q0, q1, q2, q3;
            const R n0 = num_den<0>(q0), n1 = num_den<1>(q1), n2 = num_den<2>(q2), n3 = num_den<3>(q3);
            const R q01 = q0 * q1, q23 = q2 * q3;
            const R inv = R(1) / (q01 * q23);
            o[0] = n0 * (q1 * q23) * inv;
            o[1] = n1 * (q0 * q23) * inv;
            o[2] = n2 * (q01 * q3) * inv;
            o[3] = n3 * (q01 * q2) * inv;
        } else {
            o[0] = eval<0>(); o[1] = eval<1>(); o[2] = eval<2>(); o[3] = eval<3>();
        }
    }
    // the values at the two end points (the cell faces)
    __device__ __forceinline__ void eval03(R &o0, R &o3) const
    {
        if constexpr (SHARED) {
            R q0, q3;
            const R n0 = num_den<0>(q0), n3 = num_den<3>(q3);
            const R inv = R(1) / (q0 * q3);
            o0 = n0 * q3 * inv;
            o3 = n3 * q0 * inv;
        } else {
            o0 = eval<0>(); o3 = eval<3>();
        }
    }
};

// x^3 rounded once: the exact square p + e (e = fma(x, x, -p)) times x, as hi + lo with
// the exact product error of p x, so only the final sum rounds (error ~2^-104 before it)
__device__ __forceinline__ double cube_rn(double x)
{
    const double p = x * x;
    const double e = fma(x, x, -p);
    const double hi = p * x;
    const double lo = fma(p, x, -hi);
    return hi + (lo + e * x);
}

// WENOEXP (SCHEME 2, include/Utility.hpp:291-470) on a 7-point stencil.  The linear weights
// are cubics in lambda^2 h^2 = dif5 / dif3, from the 6 points on the Gauss point's side
// (gp 0, 1: v0..v5; gp 2, 3: v1..v6), clipped to 1 and set to 0 where |dif3| < dx^4; the
// candidates are WENO5's, from the raw values; the smoothness indicators and tau use the
// stencil normalised to [0, 1] and w_k = d_k (1 + 2 tau^2 / (beta_k^2 + 1e-16)).  The
// factors 1 + 2 tau^2 / (beta_k^2 + 1e-16) depend on the stencil only and are formed once.
// The reference's pow(l, 3) is the C library's (within 0.52 ulp of l^3); here it is l^3
// rounded once (cube_rn), so the linear weights can differ from the reference's in the last
// bit where the C library's pow is not correctly rounded.  FP64 only.  The contracted build
// shares divisions as Weno5 does: one for both sides' dif5 / dif3, one for the three
// factors and one for the normalisations of all Gauss points evaluated together (10
// divisions per stencil in the reference's order, 4 here).
struct WenoExp {
    double umm, um, u, up, upp; // raw centre-5 values
    double f0, f1, f2;          // 1 + 2 tau^2 / (beta_k^2 + eps)
    double lam[2];              // lambda^2 h^2 of the left (gp 0, 1) and right (gp 2, 3) side

    static __device__ __forceinline__ double side(double a, double b, double c, double d, double e, double f, double dx4)
    {
        const double dif5 = (-a + 5.0 * b - 10.0 * c + 10.0 * d - 5.0 * e + f);
        const double dif3 = (a - 11.0 * b + 28.0 * c - 28.0 * d + 11.0 * e - f) / 6.0;
        double l = 0.0;
        if (!(fabs(dif3) < dx4)) {
            l = dif5 / dif3;
            if (fabs(l) > 1) l = 1;
        }
        return l;
    }

    __device__ __forceinline__ void init(const double *v, double dx4)
    {
        umm = v[1]; um = v[2]; u = v[3]; up = v[4]; upp = v[5];
#if WENOFV_STRICT
        lam[0] = side(v[0], v[1], v[2], v[3], v[4], v[5], dx4);
        lam[1] = side(v[1], v[2], v[3], v[4], v[5], v[6], dx4);
#else
        // 6 dif3 compared against 6 dx^4; lambda^2 h^2 = 6 dif5 / (6 dif3) with one division
        const double a5 = -v[0] + 5.0 * v[1] - 10.0 * v[2] + 10.0 * v[3] - 5.0 * v[4] + v[5];
        const double a3 = v[0] - 11.0 * v[1] + 28.0 * v[2] - 28.0 * v[3] + 11.0 * v[4] - v[5];
        const double b5 = -v[1] + 5.0 * v[2] - 10.0 * v[3] + 10.0 * v[4] - 5.0 * v[5] + v[6];
        const double b3 = v[1] - 11.0 * v[2] + 28.0 * v[3] - 28.0 * v[4] + 11.0 * v[5] - v[6];
        const double th = 6.0 * dx4;
        const bool za = fabs(a3) < th, zb = fabs(b3) < th;
        const double qa = za ? 1.0 : a3, qb = zb ? 1.0 : b3;
        const double inv3 = 6.0 / (qa * qb);
        double la = za ? 0.0 : a5 * qb * inv3, lb = zb ? 0.0 : b5 * qa * inv3;
        if (fabs(la) > 1) la = 1;
        if (fabs(lb) > 1) lb = 1;
        lam[0] = la;
        lam[1] = lb;
#endif
        const double umax = std_max(std_max(std_max(umm, um), std_max(u, up)), upp);
        const double umin = std_min(std_min(std_min(umm, um), std_min(u, up)), upp);
        double n0, n1, n2, n3, n4;
#if WENOFV_STRICT
        n0 = (umm - umin) / (umax - umin + 1e-20);
        n1 = (um - umin) / (umax - umin + 1e-20);
        n2 = (u - umin) / (umax - umin + 1e-20);
        n3 = (up - umin) / (umax - umin + 1e-20);
        n4 = (upp - umin) / (umax - umin + 1e-20);
#else
        const double inv = 1.0 / (umax - umin + 1e-20);
        n0 = (umm - umin) * inv; n1 = (um - umin) * inv; n2 = (u - umin) * inv;
        n3 = (up - umin) * inv; n4 = (upp - umin) * inv;
#endif
        // theta * 1.0 / 2.0 with theta = 1 is the exact 0.5
        const double b0 = 0.5 * fabs(n0 - 4 * n1 + 3 * n2) + fabs(n0 - 2 * n1 + n2);
        const double b1 = 0.5 * fabs(n1 - n3) + fabs(n1 - 2 * n2 + n3);
        const double b2 = 0.5 * fabs(3 * n2 - 4 * n3 + n4) + fabs(n2 - 2 * n3 + n4);
        const double tau = n0 - 4.0 * n1 + 6.0 * n2 - 4.0 * n3 + n4;
        const double t2 = 2 * (tau * tau); // pow(x, 2.0) is x * x
#if WENOFV_STRICT
        f0 = 1.0 + t2 / (b0 * b0 + 1e-16);
        f1 = 1.0 + t2 / (b1 * b1 + 1e-16);
        f2 = 1.0 + t2 / (b2 * b2 + 1e-16);
#else
        // beta_k^2 + 1e-16 lies in [1e-16, ~40]: the product of the three stays far from
        // underflow and overflow
        const double a0 = b0 * b0 + 1e-16, a1 = b1 * b1 + 1e-16, a2 = b2 * b2 + 1e-16;
        const double a01 = a0 * a1, tq = t2 / (a01 * a2);
        f0 = 1.0 + a1 * a2 * tq;
        f1 = 1.0 + a0 * a2 * tq;
        f2 = 1.0 + a01 * tq;
#endif
    }

    // numerator and denominator of the value at GP
    template <int GP> __device__ __forceinline__ double num_den(double &S) const
    {
        const double l = lam[GP >= 2 ? 1 : 0], l2 = l * l, l3 = cube_rn(l);
        const double a = (GP == 0 || GP == 3) ? 0.3 - 0.057142858 * l + 0.0071428571 * l2 - 0.00077200577 * l3
                                               : 0.16108042 - 0.035187607 * l + 0.0049466098 * l2 - 0.00058211525 * l3;
        const double b = (GP == 0 || GP == 3) ? 0.6 + 0.078571429 * l - 0.0101190476 * l2 + 0.00112012987 * l3
                                               : 0.58636364 + 0.087692641 * l - 0.0120401515 * l2 + 0.00139436871 * l3;
        const double c = (GP == 0 || GP == 3) ? 0.1 - 0.021428571 * l + 0.0029761905 * l2 - 0.00034812410 * l3
                                               : 0.25255594 - 0.052505034 * l + 0.0070935417 * l2 - 0.00081225346 * l3;
        // gp 0, 1: (d0, d1, d2) = (a, b, c); gp 2, 3 mirror them
        const double d0 = GP < 2 ? a : c, d1 = b, d2 = GP < 2 ? c : a;
        double h0, h1, h2;
        weno_h<double, GP>(umm, um, u, up, upp, h0, h1, h2);
        double w0 = d0 * f0, w1 = d1 * f1, w2 = d2 * f2;
        S = w0 + w1 + w2;
#if WENOFV_STRICT
        w0 /= S; w1 /= S; w2 /= S;
        return w0 * h0 + w1 * h1 + w2 * h2;
#else
        return w0 * h0 + w1 * h1 + w2 * h2;
#endif
    }
    // S = sum of w_k lies in [~0.05, ~1e19]: products of four stay in range
    __device__ __forceinline__ void eval4(double *o) const
    {
        double q0, q1, q2, q3;
        const double n0 = num_den<0>(q0), n1 = num_den<1>(q1), n2 = num_den<2>(q2), n3 = num_den<3>(q3);
#if WENOFV_STRICT
        o[0] = n0; o[1] = n1; o[2] = n2; o[3] = n3;
#else
        const double q01 = q0 * q1, q23 = q2 * q3;
        const double inv = 1.0 / (q01 * q23);
        o[0] = n0 * (q1 * q23) * inv;
        o[1] = n1 * (q0 * q23) * inv;
        o[2] = n2 * (q01 * q3) * inv;
        o[3] = n3 * (q01 * q2) * inv;
#endif
    }
    __device__ __forceinline__ void eval03(double &o0, double &o3) const
    {
        double q0, q3;
        const double n0 = num_den<0>(q0), n3 = num_den<3>(q3);
#if WENOFV_STRICT
        o0 = n0; o3 = n3;
#else
        const double inv = 1.0 / (q0 * q3);
        o0 = n0 * q3 * inv;
        o3 = n3 * q0 * inv;
#endif
    }
};

// wenoExpWithThincReconstruction (include/Utility.hpp:473-688): PRIMITIVE3's reconstruction
// of z1 on a 7-point stencil.  A mixed centre (1e-6 < u < 1 - 1e-6) takes the THINC profile
// 0.5 Qmax (1 + theta tanh(1.5 ((x_gp + 1) / 2 - xcc))) + Qmin from its two neighbours (the
// cell value at a local extremum); any other cell WENOEXP's linear weights (lambda^2 h^2
// unclipped here) with WENO-Z's smoothness indicators on the normalised stencil and
// w_k = d_k (1 + |beta0 - beta2| / (beta_k + 1e-16)).  exp(1.5) and exp(-1.5), which gcc
// folds at compile time, are the correctly rounded constants; the exp, log and tanh of the
// profile are CUDA's, within an ulp or two of the C library's, so THINC cells do not agree
// with the reference bit for bit.  The profile itself amplifies such last-bit differences
// (xc = (e^beta - B) / (B - e^-beta) cancels as C nears 0 or 1): moving the C library's
// results by one ulp moves the reference's own RHS by up to ~1e-9 of max |U|.  FP64 only.
struct ExpThinc {
    double umm, um, u, up, upp;
    double f0, f1, f2, lam[2];    // WENO branch
    double qmin, qmax, theta, xcc; // THINC branch (contracted build: xcc holds xc)
    bool thinc, ext;

    __device__ __forceinline__ void init(const double *v, double dx4)
    {
        umm = v[1]; um = v[2]; u = v[3]; up = v[4]; upp = v[5];
        thinc = (1e-6 < u) & (u < 1 - 1e-6);
        if (thinc) {
            constexpr double beta = 1.5, e_beta = 0x1.1ed3fe64fc541p+2, e_mbeta = 0x1.c8f87724b5c1dp-3; // e^1.5, e^-1.5
            qmin = std_min(um, up);
            qmax = std_max(um, up) - qmin;
            theta = (up - u >= 0) ? 1.0 : -1.0; // sc_math::Sign, third_party/scTools/MyMath.h:47-50
            const double C = (u - qmin + 1e-20) / (qmax + 1e-20);
            const double arg = theta * beta * (2.0 * C - 1.0);
            // at exactly +-1.5 (C = 0 or 1) the reference's B is its compile-time exp(+-beta),
            // so that xc is exactly 0 or inf (the profile saturates) rather than +-tiny
            const double B = arg == beta ? e_beta : (arg == -beta ? e_mbeta : exp(arg));
            const double xc = (e_beta - B) / (B - e_mbeta);
#if WENOFV_STRICT
            xcc = log(xc) / (2.0 * beta);
#else
            xcc = xc; // the profile from xc itself (thinc_at)
#endif
            ext = (u - um) * (up - u) < 0;
            return;
        }
#if WENOFV_STRICT
        for (int s = 0; s < 2; s++) {
            const double *w = v + s;
            const double dif5 = (-w[0] + 5.0 * w[1] - 10.0 * w[2] + 10.0 * w[3] - 5.0 * w[4] + w[5]);
            const double dif3 = (w[0] - 11.0 * w[1] + 28.0 * w[2] - 28.0 * w[3] + 11.0 * w[4] - w[5]) / 6.0;
            lam[s] = fabs(dif3) < dx4 ? 0.0 : dif5 / dif3;
        }
#else
        const double a5 = -v[0] + 5.0 * v[1] - 10.0 * v[2] + 10.0 * v[3] - 5.0 * v[4] + v[5];
        const double a3 = v[0] - 11.0 * v[1] + 28.0 * v[2] - 28.0 * v[3] + 11.0 * v[4] - v[5];
        const double b5 = -v[1] + 5.0 * v[2] - 10.0 * v[3] + 10.0 * v[4] - 5.0 * v[5] + v[6];
        const double b3 = v[1] - 11.0 * v[2] + 28.0 * v[3] - 28.0 * v[4] + 11.0 * v[5] - v[6];
        const double th = 6.0 * dx4;
        const bool za = fabs(a3) < th, zb = fabs(b3) < th;
        const double qa = za ? 1.0 : a3, qb = zb ? 1.0 : b3;
        const double inv3 = 6.0 / (qa * qb);
        lam[0] = za ? 0.0 : a5 * qb * inv3;
        lam[1] = zb ? 0.0 : b5 * qa * inv3;
#endif
        const double umax = std_max(std_max(std_max(umm, um), std_max(u, up)), upp);
        const double umin = std_min(std_min(std_min(umm, um), std_min(u, up)), upp);
        double n0, n1, n2, n3, n4;
#if WENOFV_STRICT
        n0 = (umm - umin) / (umax - umin + 1e-20);
        n1 = (um - umin) / (umax - umin + 1e-20);
        n2 = (u - umin) / (umax - umin + 1e-20);
        n3 = (up - umin) / (umax - umin + 1e-20);
        n4 = (upp - umin) / (umax - umin + 1e-20);
#else
        const double inv = 1.0 / (umax - umin + 1e-20);
        n0 = (umm - umin) * inv; n1 = (um - umin) * inv; n2 = (u - umin) * inv;
        n3 = (up - umin) * inv; n4 = (upp - umin) * inv;
#endif
        double b0, b1, b2;
        weno_betas(n0, n1, n2, n3, n4, b0, b1, b2);
        const double tau = fabs(b0 - b2);
#if WENOFV_STRICT
        f0 = 1 + tau / (b0 + 1e-16);
        f1 = 1 + tau / (b1 + 1e-16);
        f2 = 1 + tau / (b2 + 1e-16);
#else
        // beta_k + 1e-16 in [1e-16, ~80]: the product of the three stays in range
        const double a0 = b0 + 1e-16, a1 = b1 + 1e-16, a2 = b2 + 1e-16;
        const double a01 = a0 * a1, tq = tau / (a01 * a2);
        f0 = 1 + a1 * a2 * tq;
        f1 = 1 + a0 * a2 * tq;
        f2 = 1 + a01 * tq;
#endif
    }

    template <int GP> __device__ __forceinline__ double thinc_at() const
    {
        if (ext) return u;
#if WENOFV_STRICT
        // (x + 1) / 2 of the reference-interval Gauss-Lobatto points (GaussLobatto_ref(4),
        // third_party/scTools/GaussQuadratureInRef.hpp:250-259)
        constexpr double x = GP == 0 ? -1.0 : GP == 1 ? -0.447213595499957939281834733746
                           : GP == 2 ? 0.447213595499957939281834733746 : 1.0;
        return 0.5 * qmax * (1 + theta * tanh(1.5 * ((x + 1) / 2 - xcc))) + qmin;
#else
        // with xcc = log(xc) / (2 beta): tanh(beta ((x + 1) / 2 - xcc)) = (K - xc) / (K + xc),
        // K = e^(beta (x + 1)), so the profile needs neither log nor tanh (xc = 0 gives 1;
        // xc = inf, the other saturated end, gives -1)
        constexpr double K = GP == 0 ? 1.0 : GP == 1 ? 0x1.254dd7e1a7f2ep+1 /* e^(1.5 (1 - 1/sqrt 5)) */
                           : GP == 2 ? 0x1.187ebf9c17648p+3 /* e^(1.5 (1 + 1/sqrt 5)) */ : 0x1.415e5bf6fb106p+4 /* e^3 */;
        const double xc = xcc;
        const double th = isinf(xc) ? -1.0 : (K - xc) / (K + xc);
        return 0.5 * qmax * (1 + theta * th) + qmin;
#endif
    }
    // numerator and denominator of the WENO value at GP (strict: the value, S unused)
    template <int GP> __device__ __forceinline__ double num_den(double &S) const
    {
        const double l = lam[GP >= 2 ? 1 : 0], l2 = l * l, l3 = cube_rn(l);
        const double a = (GP == 0 || GP == 3) ? 0.3 - 0.057142858 * l + 0.0071428571 * l2 - 0.00077200577 * l3
                                               : 0.16108042 - 0.035187607 * l + 0.0049466098 * l2 - 0.00058211525 * l3;
        const double b = (GP == 0 || GP == 3) ? 0.6 + 0.078571429 * l - 0.0101190476 * l2 + 0.00112012987 * l3
                                               : 0.58636364 + 0.087692641 * l - 0.0120401515 * l2 + 0.00139436871 * l3;
        const double c = (GP == 0 || GP == 3) ? 0.1 - 0.021428571 * l + 0.0029761905 * l2 - 0.00034812410 * l3
                                               : 0.25255594 - 0.052505034 * l + 0.0070935417 * l2 - 0.00081225346 * l3;
        const double d0 = GP < 2 ? a : c, d1 = b, d2 = GP < 2 ? c : a;
        double h0, h1, h2;
        weno_h<double, GP>(umm, um, u, up, upp, h0, h1, h2);
        double w0 = d0 * f0, w1 = d1 * f1, w2 = d2 * f2;
        S = w0 + w1 + w2;
#if WENOFV_STRICT
        w0 /= S; w1 /= S; w2 /= S;
#endif
        return w0 * h0 + w1 * h1 + w2 * h2;
    }
    __device__ __forceinline__ void eval4(double *o) const
    {
        if (thinc) {
            o[0] = thinc_at<0>(); o[1] = thinc_at<1>(); o[2] = thinc_at<2>(); o[3] = thinc_at<3>();
            return;
        }
        double q0, q1, q2, q3;
        const double n0 = num_den<0>(q0), n1 = num_den<1>(q1), n2 = num_den<2>(q2), n3 = num_den<3>(q3);
#if WENOFV_STRICT
        o[0] = n0; o[1] = n1; o[2] = n2; o[3] = n3;
#else
        const double q01 = q0 * q1, q23 = q2 * q3; // S in [~0.05, ~1e18]
        const double inv = 1.0 / (q01 * q23);
        o[0] = n0 * (q1 * q23) * inv;
        o[1] = n1 * (q0 * q23) * inv;
        o[2] = n2 * (q01 * q3) * inv;
        o[3] = n3 * (q01 * q2) * inv;
#endif
    }
    __device__ __forceinline__ void eval03(double &o0, double &o3) const
    {
        if (thinc) {
            o0 = thinc_at<0>(); o3 = thinc_at<3>();
            return;
        }
        double q0, q3;
        const double n0 = num_den<0>(q0), n3 = num_den<3>(q3);
#if WENOFV_STRICT
        o0 = n0; o3 = n3;
#else
        const double inv = 1.0 / (q0 * q3);
        o0 = n0 * q3 * inv;
        o3 = n3 * q0 * inv;
#endif
    }
};

// ------------------------------------------------------------------------------------
// equations
// ------------------------------------------------------------------------------------

// Two-phase 3-equation model with linear acoustic EOS (include/Equations.hpp:84-483).
// U = (z1 rho1, z2 rho2, rho u, rho v).  The volume fraction and pressure recovery always
// run in FP64 (also in the FP32-bulk form): the cancellation in q - qs and the division by
// z2 rho2 c2^2 near pure phases need it.
struct TwoPhaseK {
    static constexpr bool linear = true; // constant phase sound speeds
    double c1_2, c2_2, q, rho10, rho20;
    __device__ __forceinline__ explicit TwoPhaseK(const EqParams &p)
    {
        c1_2 = p.sound1 * p.sound1;
        c2_2 = p.sound2 * p.sound2;
        q = p.rho20 * c2_2 - p.rho10 * c1_2;
        rho10 = p.rho10;
        rho20 = p.rho20;
    }
    // getVolumeFrac, include/Equations.hpp:84-99
    __device__ __forceinline__ double volume_frac(double z1rho1, double z2rho2) const
    {
        const double qs = z2rho2 * c2_2 - z1rho1 * c1_2;
        const double r = ((q - qs) + sqrt((q - qs) * (q - qs) + 4.0 * z1rho1 * c1_2 * z2rho2 * c2_2)) / (2.0 * z2rho2 * c2_2);
        return r / (1.0 + r);
    }
    // getPressure, include/Equations.hpp:101-124 (dominant phase, g_preb dropped)
    __device__ __forceinline__ double pressure(double z1rho1, double z2rho2, double z1) const
    {
        const double z2 = 1.0 - z1;
        const double pre1 = c1_2 * (z1rho1 / z1 - rho10);
        const double pre2 = c2_2 * (z2rho2 / z2 - rho20);
        return (z1 < z2) ? pre2 : pre1;
    }
    // getSoundSpeed (Wood), include/Equations.hpp:126-146
    // getVolumeFrac + getPressure in one pass, contracted build: the same quadratic root with
    // z1 = r/(1+r) = N/(N+D) and the pressures rewritten with 1/z2 = 1+r, 1/z1 = 1+1/r
    // (r = N/D), i.e. one sqrt and two divisions instead of one sqrt and four
    __device__ __forceinline__ void recover(double z1rho1, double z2rho2, double &z1, double &p) const
    {
        const double qs = z2rho2 * c2_2 - z1rho1 * c1_2;
        const double N = (q - qs) + sqrt((q - qs) * (q - qs) + 4.0 * z1rho1 * c1_2 * z2rho2 * c2_2);
        const double Dn = 2.0 * z2rho2 * c2_2;
        const double ND = N + Dn;
        const double Ng = N > 0.0 ? N : 1.0; // N = 0: z1 = 0, pre1 unused
        const double inv = 1.0 / (ND * Ng);  // 1/(N + D) = Ng inv, 1/N = ND inv
        z1 = N * (Ng * inv);
        const double z2 = 1.0 - z1;
        const double pre2 = c2_2 * (z2rho2 - rho20) + 0.5 * N; // c2^2 (z2rho2 / z2 - rho20)
        const double pre1 = c1_2 * (z1rho1 + z1rho1 * Dn * (ND * inv) - rho10); // c1^2 (z1rho1 / z1 - rho10)
        p = (z1 < z2) ? pre2 : pre1;
    }
    // recover plus 1/rho of the same state with one division for 1/rho, 1/(N+D) and 1/N, in two
    // halves so that two states can share the division (recover_pair)
    struct Rec { double N, Dn, ND, Ng, X; };
    __device__ __forceinline__ Rec recover_a(double z1rho1, double z2rho2, double rho) const
    {
        Rec a;
        const double qs = z2rho2 * c2_2 - z1rho1 * c1_2;
        a.N = (q - qs) + sqrt((q - qs) * (q - qs) + 4.0 * z1rho1 * c1_2 * z2rho2 * c2_2);
        a.Dn = 2.0 * z2rho2 * c2_2;
        a.ND = a.N + a.Dn;
        a.Ng = a.N > 0.0 ? a.N : 1.0; // N = 0: z1 = 0, pre1 unused
        a.X = rho * a.ND * a.Ng;
        return a;
    }
    // inv = 1/X: 1/rho = ND Ng inv, 1/ND = rho Ng inv, 1/N = rho ND inv
    __device__ __forceinline__ void recover_b(const Rec &a, double inv, double z1rho1, double z2rho2, double rho, double &irho,
                                              double &z1, double &p) const
    {
        irho = a.ND * a.Ng * inv;
        z1 = a.N * (rho * a.Ng * inv);
        const double z2 = 1.0 - z1;
        const double pre2 = c2_2 * (z2rho2 - rho20) + 0.5 * a.N;
        const double pre1 = c1_2 * (z1rho1 + z1rho1 * a.Dn * (rho * a.ND * inv) - rho10);
        p = (z1 < z2) ? pre2 : pre1;
    }
    __device__ __forceinline__ void recover_rho(double z1rho1, double z2rho2, double rho, double &irho, double &z1,
                                                double &p) const
    {
        const Rec a = recover_a(z1rho1, z2rho2, rho);
        recover_b(a, 1.0 / a.X, z1rho1, z2rho2, rho, irho, z1, p);
    }
    // the strict order of tp_state: getVolumeFrac, then getPressure
    __device__ __forceinline__ void state(double z1rho1, double z2rho2, double &z1, double &p) const
    {
        z1 = volume_frac(z1rho1, z2rho2);
        p = pressure(z1rho1, z2rho2, z1);
    }
    // the volume fraction of the eigensystem (the pressure is not needed there)
    __device__ __forceinline__ void eigen_state(double z1rho1, double z2rho2, double &z1, double &p) const
    {
#if WENOFV_STRICT
        z1 = volume_frac(z1rho1, z2rho2);
        p = 0.0;
#else
        recover(z1rho1, z2rho2, z1, p);
#endif
    }
    template <class R> __device__ __forceinline__ R sound_p(R z1rho1, R z2rho2, R z1, R z2, double) const
    {
        return sound<R>(z1rho1, z2rho2, z1, z2);
    }
    template <class R> __device__ __forceinline__ void phase_c2(R, R, R, R, double, R &a, R &b) const
    {
        a = R(c1_2);
        b = R(c2_2);
    }
    // z2 comes in as 1 - z1 rounded from FP64: in FP32, 1 - (float)z1 loses z2 near pure phase 1
    template <class R> __device__ __forceinline__ R sound(R z1rho1, R z2rho2, R z1, R z2) const
    {
#if !WENOFV_STRICT
        if constexpr (sizeof(R) == sizeof(double)) {
            // 1/c^2 = rho (z1^2/(z1rho1 c1^2) + z2^2/(z2rho2 c2^2)) = T / P: c = sqrt(P/T) =
            // |P| / sqrt(P T), one reciprocal square root, for either sign of P and T (a
            // reconstructed partial density below 0 makes both negative); c = 0 where P = 0
            const double a1 = z1rho1 * c1_2, a2 = z2rho2 * c2_2;
            const double P = a1 * a2;
            const double T = (z1rho1 + z2rho2) * (z1 * z1 * a2 + z2 * z2 * a1);
            return P == 0.0 ? 0.0 : fabs(P) * rsqrt(P * T);
        }
#endif
        const R rho = z1rho1 + z2rho2;
        const R rho1 = z1rho1 / z1;
        const R rho2 = z2rho2 / z2;
        const R sc = sqrt(rho * (z1 / (rho1 * R(c1_2)) + z2 / (rho2 * R(c2_2))));
        return R(1.0) / sc;
    }
};

// Stiffened-gas phases on their isentropes (EQ_TWO_PHASE_SG; an extension, not in the
// reference): p_k(rho) = (pref + pi_k) (rho / rho_k0)^gamma_k - pi_k, whose expansion at pref
// is the linear model with c_k^2 = gamma_k (pref + pi_k) / rho_k0 (P.sound1/2 hold those).
// Pressure equilibrium z1rho1 / rho_1(p) + z2rho2 / rho_2(p) = 1 is solved for p by Newton
// steps from the linear model's state, kept above -min(pi_k) where both densities exist,
// until a step is below 1e-14 (|p| + max(pi_k) + |pref|), at most SG_NEWTON; then
// z1 = z1rho1 / rho_1(p).  The flux pressure is p - pref, as the linear model drops g_preb.
// The phase sound speeds are c_k^2 = gamma_k (p + pi_k) z_k / z_krho_k.  FP64 only; pow is
// CUDA's, so the results agree with the C library's to a few ulp, not bit for bit.
constexpr int SG_NEWTON = 12;
struct StiffK {
    static constexpr bool linear = false;
    TwoPhaseK lin;
    double g1, g2, pi1, pi2, pref, rho10, rho20, a1, a2, ig1, ig2, lo, scale;
    __device__ __forceinline__ explicit StiffK(const EqParams &p) : lin(p)
    {
        g1 = p.gamma1; g2 = p.gamma2; pi1 = p.pinf1; pi2 = p.pinf2; pref = p.preb;
        rho10 = p.rho10; rho20 = p.rho20;
        a1 = 1.0 / (pref + pi1); a2 = 1.0 / (pref + pi2);
        ig1 = 1.0 / g1; ig2 = 1.0 / g2;
        lo = -(pi1 < pi2 ? pi1 : pi2);
        scale = (pi1 > pi2 ? pi1 : pi2) + fabs(pref);
    }
    // x^(1/gamma) of the isentropes: pow in the strict build; exp(log(x) / gamma) in the
    // contracted one (x is near 1, so the error stays at a few ulp, without pow's extended
    // precision cost)
    static __device__ __forceinline__ double root(double x, double ig)
    {
#if WENOFV_STRICT
        return pow(x, ig);
#else
        return exp(ig * log(x));
#endif
    }
    // (z1, p - pref) of the state
    __device__ __forceinline__ void solve(double m1, double m2, double &z1, double &pg) const
    {
        double p = pref + lin.pressure(m1, m2, lin.volume_frac(m1, m2));
        if (!(p > lo)) p = 0.5 * (pref + lo);
        double r1 = 0.0;
        for (int it = 0; it < SG_NEWTON; it++) {
            r1 = rho10 * root((p + pi1) * a1, ig1);
            const double r2 = rho20 * root((p + pi2) * a2, ig2);
            const double h = m1 / r1 + m2 / r2 - 1.0;
            const double dh = -(m1 / (r1 * (g1 * (p + pi1))) + m2 / (r2 * (g2 * (p + pi2))));
            double pn = p - h / dh;
            if (!(pn > lo)) pn = 0.5 * (p + lo);
            const double dp = pn - p;
            p = pn;
            if (fabs(dp) <= 1e-14 * (fabs(p) + scale)) break;
        }
#if WENOFV_STRICT
        z1 = m1 / (rho10 * pow((p + pi1) * a1, ig1));
#else
        // rho_1 of the last step: its p moved by at most 1e-14 (|p| + max pi_k) since, which
        // changes rho_1 = rho10 x^(1/gamma_1) by at most that over gamma_1 (p + pi_1)
        z1 = m1 / r1;
#endif
        pg = p - pref;
    }
    __device__ __forceinline__ double volume_frac(double m1, double m2) const
    {
        double z1, pg;
        solve(m1, m2, z1, pg);
        return z1;
    }
    __device__ __forceinline__ void state(double m1, double m2, double &z1, double &pg) const { solve(m1, m2, z1, pg); }
    __device__ __forceinline__ void eigen_state(double m1, double m2, double &z1, double &pg) const { solve(m1, m2, z1, pg); }
    __device__ __forceinline__ void recover(double m1, double m2, double &z1, double &pg) const { solve(m1, m2, z1, pg); }
    __device__ __forceinline__ void recover_rho(double m1, double m2, double rho, double &irho, double &z1, double &pg) const
    {
        solve(m1, m2, z1, pg);
        irho = 1.0 / rho;
    }
    // Wood: 1 / (rho c^2) = z1 / (gamma_1 (p + pi_1)) + z2 / (gamma_2 (p + pi_2))
    template <class R> __device__ __forceinline__ R sound_p(R m1, R m2, R z1, R z2, double pg) const
    {
        static_assert(sizeof(R) == sizeof(double), "the stiffened-gas model runs in FP64");
        const double p = pg + pref;
        const double rho = m1 + m2;
        return 1.0 / sqrt(rho * (z1 / (g1 * (p + pi1)) + z2 / (g2 * (p + pi2))));
    }
    template <class R> __device__ __forceinline__ void phase_c2(R m1, R m2, R z1, R z2, double pg, R &c1_2, R &c2_2) const
    {
        const double p = pg + pref;
        c1_2 = g1 * (p + pi1) * z1 / m1;
        c2_2 = g2 * (p + pi2) * z2 / m2;
    }
};

// the two-phase equation kinds and their thermodynamics
template <int EQ> struct IsTwoPhase { static constexpr bool value = EQ == EQ_TWO_PHASE || EQ == EQ_TWO_PHASE_SG; };
template <int EQ> struct TPKOf { using type = TwoPhaseK; };
template <> struct TPKOf<EQ_TWO_PHASE_SG> { using type = StiffK; };

// Primitive quantities of one state, computed once and reused by every consumer (the
// reference recomputes getVolumeFrac per call; the values are identical).
template <class R> struct TPState {
    R z1rho1, z2rho2, rhou, rhov, rho, u, v, pre, c;
    double pd;   // the FP64 pressure (pre is pd rounded to R)
    double irho; // 1/rho (contracted FP64 build)
};

// The state comes in FP64 in every form: the volume fraction and the pressure are
// recovered from the FP64 values.
template <class R, class KT>
__device__ __forceinline__ void tp_state(const KT &K, const double *U, TPState<R> &s)
{
    s.z1rho1 = (R)U[0]; s.z2rho2 = (R)U[1]; s.rhou = (R)U[2]; s.rhov = (R)U[3];
    s.rho = s.z1rho1 + s.z2rho2;
#if WENOFV_STRICT
    s.u = s.rhou / s.rho;
    s.v = s.rhov / s.rho;
    double z1;
    K.state(U[0], U[1], z1, s.pd);
#else
    double z1;
    if constexpr (sizeof(R) == sizeof(double)) {
        K.recover_rho(U[0], U[1], s.rho, s.irho, z1, s.pd);
        s.u = s.rhou * s.irho;
        s.v = s.rhov * s.irho;
    } else {
        const R ir = R(1) / s.rho;
        s.u = s.rhou * ir;
        s.v = s.rhov * ir;
        K.recover(U[0], U[1], z1, s.pd);
    }
#endif
    s.pre = (R)s.pd;
    s.c = K.template sound_p<R>(s.z1rho1, s.z2rho2, (R)z1, (R)(1.0 - z1), s.pd);
}

// the two face states of a Riemann problem: in the contracted FP64 build of the linear model
// their recoveries share one division (1/(X_L X_R) gives 1/X_L and 1/X_R), otherwise tp_state
// twice
template <class R, class KT>
__device__ __forceinline__ void tp_state_pair(const KT &K, const double *UL, const double *UR, TPState<R> &l, TPState<R> &r)
{
#if !WENOFV_STRICT
    if constexpr (sizeof(R) == sizeof(double) && KT::linear) {
        l.z1rho1 = UL[0]; l.z2rho2 = UL[1]; l.rhou = UL[2]; l.rhov = UL[3];
        r.z1rho1 = UR[0]; r.z2rho2 = UR[1]; r.rhou = UR[2]; r.rhov = UR[3];
        l.rho = l.z1rho1 + l.z2rho2;
        r.rho = r.z1rho1 + r.z2rho2;
        const typename KT::Rec a = K.recover_a(UL[0], UL[1], l.rho), b = K.recover_a(UR[0], UR[1], r.rho);
        const double inv = 1.0 / (a.X * b.X);
        double z1l, z1r;
        K.recover_b(a, b.X * inv, UL[0], UL[1], l.rho, l.irho, z1l, l.pd);
        K.recover_b(b, a.X * inv, UR[0], UR[1], r.rho, r.irho, z1r, r.pd);
        l.u = l.rhou * l.irho; l.v = l.rhov * l.irho;
        r.u = r.rhou * r.irho; r.v = r.rhov * r.irho;
        l.pre = l.pd; r.pre = r.pd;
        l.c = K.template sound_p<R>(l.z1rho1, l.z2rho2, z1l, 1.0 - z1l, l.pd);
        r.c = K.template sound_p<R>(r.z1rho1, r.z2rho2, z1r, 1.0 - z1r, r.pd);
        return;
    }
    if constexpr (sizeof(R) < sizeof(double) && KT::linear) {
        // FP32-bulk: the FP64 recoveries (z1, p) share one division (rho = 1 in the halves:
        // 1/(N+D) and 1/N only), the rest as tp_state
        TPState<R> *s2[2] = {&l, &r};
        const double *U2[2] = {UL, UR};
        const typename KT::Rec a = K.recover_a(UL[0], UL[1], 1.0), b = K.recover_a(UR[0], UR[1], 1.0);
        const double inv = 1.0 / (a.X * b.X);
        double z1[2], dummy;
        K.recover_b(a, b.X * inv, UL[0], UL[1], 1.0, dummy, z1[0], l.pd);
        K.recover_b(b, a.X * inv, UR[0], UR[1], 1.0, dummy, z1[1], r.pd);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            TPState<R> &s = *s2[k];
            const double *U = U2[k];
            s.z1rho1 = (R)U[0]; s.z2rho2 = (R)U[1]; s.rhou = (R)U[2]; s.rhov = (R)U[3];
            s.rho = s.z1rho1 + s.z2rho2;
            const R ir = R(1) / s.rho;
            s.u = s.rhou * ir;
            s.v = s.rhov * ir;
            s.pre = (R)s.pd;
            s.c = K.template sound_p<R>(s.z1rho1, s.z2rho2, (R)z1[k], (R)(1.0 - z1[k]), s.pd);
        }
        return;
    }
#endif
    tp_state<R>(K, UL, l);
    tp_state<R>(K, UR, r);
}

// getMaxEigenValue, include/Equations.hpp:149-156 (u from U[2]/(U[0]+U[1]) as there)
template <class R> __device__ __forceinline__ R tp_max_eig(const TPState<R> &s, double nx, double ny)
{
    return fabs(s.u * R(nx) + s.v * R(ny)) + s.c;
}

// getPhyFlux, include/Equations.hpp:158-186
template <class R> __device__ __forceinline__ void tp_phy_flux(const TPState<R> &s, R *F, bool xdir)
{
    if (xdir) {
        F[0] = s.z1rho1 * s.u;
        F[1] = s.z2rho2 * s.u;
        F[2] = s.rho * (s.u * s.u) + s.pre;
        F[3] = s.rho * s.u * s.v;
    } else {
        F[0] = s.z1rho1 * s.v;
        F[1] = s.z2rho2 * s.v;
        F[2] = s.rho * s.v * s.u;
        F[3] = s.rho * (s.v * s.v) + s.pre;
    }
}

// getLLFRiemannFlux, include/Equations.hpp:363-378
template <class R>
__device__ __forceinline__ void tp_llf(const TPState<R> &L, const TPState<R> &Rs, const R *UL, const R *UR, R *F, bool xdir)
{
    const double nx = xdir ? 1.0 : 0.0, ny = xdir ? 0.0 : 1.0;
    const R ws = std_max(tp_max_eig(L, nx, ny), tp_max_eig(Rs, nx, ny));
    R FUL[4], FUR[4];
    tp_phy_flux(L, FUL, xdir);
    tp_phy_flux(Rs, FUR, xdir);
#pragma unroll
    for (int r = 0; r < 4; ++r) F[r] = R(0.5) * (FUL[r] + FUR[r] - ws * (UR[r] - UL[r]));
}

// getHLLCRiemannFlux (Zhang & Zhang 2025), include/Equations.hpp:381-483
template <class R>
__device__ __forceinline__ void tp_hllc(const TPState<R> &L, const TPState<R> &Rs, const R *UL, const R *UR, R *F, bool xdir)
{
    const R nx = xdir ? R(1.0) : R(0.0), ny = xdir ? R(0.0) : R(1.0);
    const R vn_L = L.u * nx + L.v * ny;
    const R vn_R = Rs.u * nx + Rs.v * ny;
    R FUL[4], FUR[4], U[4];
    FUL[0] = L.z1rho1 * vn_L;
    FUL[1] = L.z2rho2 * vn_L;
    FUL[2] = L.rhou * vn_L + L.pre * nx;
    FUL[3] = L.rhov * vn_L + L.pre * ny;
    FUR[0] = Rs.z1rho1 * vn_R;
    FUR[1] = Rs.z2rho2 * vn_R;
    FUR[2] = Rs.rhou * vn_R + Rs.pre * nx;
    FUR[3] = Rs.rhov * vn_R + Rs.pre * ny;
#if WENOFV_STRICT
    const R sL = sqrt(L.rho), sR = sqrt(Rs.rho);
    const R vn_roe = (vn_L * sL + vn_R * sR) / (sL + sR);
    R c2_roe = (L.c * L.c * sL + Rs.c * Rs.c * sR) / (sL + sR);
    c2_roe += R(0.5) * sL * sR / (sL + sR) / (sL + sR) * (vn_R - vn_L) * (vn_R - vn_L);
#else
    R vn_roe, c2_roe;
    if constexpr (sizeof(R) == sizeof(double)) {
        // Roe weights w_L = sL/(sL+sR) = 1/(1+t), w_R = t w_L with t = sqrt(rho_R/rho_L):
        // one square root and one division
        const R t = sqrt(Rs.rho * L.irho);
        const R wL = R(1) / (R(1) + t), wR = t * wL;
        vn_roe = vn_L * wL + vn_R * wR;
        c2_roe = L.c * L.c * wL + Rs.c * Rs.c * wR;
        c2_roe += R(0.5) * wL * wR * (vn_R - vn_L) * (vn_R - vn_L);
    } else {
        const R sL = sqrt(L.rho), sR = sqrt(Rs.rho);
        const R is = R(1) / (sL + sR);
        vn_roe = (vn_L * sL + vn_R * sR) * is;
        c2_roe = (L.c * L.c * sL + Rs.c * Rs.c * sR) * is;
        c2_roe += R(0.5) * sL * sR * is * is * (vn_R - vn_L) * (vn_R - vn_L);
    }
#endif
    const R c_roe = sqrt(c2_roe);
    const R S_L = std_min(vn_L - L.c, vn_roe - c_roe);
    const R S_R = std_max(vn_R + Rs.c, vn_roe + c_roe);
#if !WENOFV_STRICT
    if constexpr (sizeof(R) == sizeof(double)) {
        // S* = num/den and the star factor k = (S_K - vn_K)/(S_K - S*) = (S_K - vn_K) den /
        // (S_K den - num) from one division; the side is the sign of S* (num over den)
        const R num = (S_L - vn_L) * L.rho * vn_L - (S_R - vn_R) * Rs.rho * vn_R + Rs.pre - L.pre;
        const R den = (S_L - vn_L) * L.rho - (S_R - vn_R) * Rs.rho;
        const bool left = (den < R(0)) ? (num <= R(0)) : (num >= R(0));
        const bool super = left ? (S_L >= R(0.0)) : (S_R <= R(0));
        const TPState<R> &K = left ? L : Rs;
        const R *UK = left ? UL : UR;
        const R *FK = left ? FUL : FUR;
        if (super) {
#pragma unroll
            for (int r = 0; r < 4; r++) F[r] = FK[r];
            return;
        }
        const R S_K = left ? S_L : S_R, vn_K = left ? vn_L : vn_R;
        const R m = S_K * den - num;
        const R inv = R(1) / (den * m);
        const R S_star = num * m * inv;
        const R k = (S_K - vn_K) * den * den * inv;
        U[0] = K.z1rho1;
        U[1] = K.z2rho2;
        U[2] = K.rho * (K.u + (S_star - vn_K) * nx);
        U[3] = K.rho * (K.v + (S_star - vn_K) * ny);
#pragma unroll
        for (int r = 0; r < 4; r++) F[r] = S_K * (k * U[r] - UK[r]) + FK[r];
        return;
    }
#endif
    const R S_star = ((S_L - vn_L) * L.rho * vn_L - (S_R - vn_R) * Rs.rho * vn_R + Rs.pre - L.pre) /
                     ((S_L - vn_L) * L.rho - (S_R - vn_R) * Rs.rho);
    if (S_star >= R(0)) {
        if (S_L >= R(0.0)) {
#pragma unroll
            for (int r = 0; r < 4; r++) F[r] = FUL[r];
        } else {
            const R k = (S_L - vn_L) / (S_L - S_star);
            U[0] = L.z1rho1;
            U[1] = L.z2rho2;
            U[2] = L.rho * (L.u + (S_star - vn_L) * nx);
            U[3] = L.rho * (L.v + (S_star - vn_L) * ny);
#pragma unroll
            for (int r = 0; r < 4; r++) F[r] = S_L * (k * U[r] - UL[r]) + FUL[r];
        }
    } else {
        if (S_R <= R(0)) {
#pragma unroll
            for (int r = 0; r < 4; r++) F[r] = FUR[r];
        } else {
            const R k = (S_R - vn_R) / (S_R - S_star);
            U[0] = Rs.z1rho1;
            U[1] = Rs.z2rho2;
            U[2] = Rs.rho * (Rs.u + (S_star - vn_R) * nx);
            U[3] = Rs.rho * (Rs.v + (S_star - vn_R) * ny);
#pragma unroll
            for (int r = 0; r < 4; r++) F[r] = S_R * (k * U[r] - UR[r]) + FUR[r];
        }
    }
}

// FP32-bulk forms of the two fluxes.  The same fluxes, rearranged so that FP32 rounds only
// small quantities: the pressure terms of the momentum fluxes are added in FP64 (the
// pressure of a weakly compressible flow is a large constant plus small variations, and
// its FP32 rounding would not cancel between the two faces of a cell), the pressure jump of
// S* and the state jump of LLF are formed in FP64, and the HLLC star fluxes use the exact
// identities S_K (k U*_K - U_K) + F_K = k S* U_K + k rho_K S_K (S* - vn_K) n + p_K n
// (k = (S_K - vn_K) / (S_K - S*)), which need no difference of nearly equal terms.
__device__ __forceinline__ void tp_llf_f32(const TPState<float> &L, const TPState<float> &Rs, const double *ULd,
                                           const double *URd, double *F, bool xdir)
{
    const double nx = xdir ? 1.0 : 0.0, ny = xdir ? 0.0 : 1.0;
    const float ws = std_max(tp_max_eig(L, nx, ny), tp_max_eig(Rs, nx, ny));
    const float vn_L = xdir ? L.u : L.v, vn_R = xdir ? Rs.u : Rs.v;
    const float ut_L = xdir ? L.v : L.u, ut_R = xdir ? Rs.v : Rs.u;
    float FD[4]; // FUL + FUR without the pressure terms
    FD[0] = L.z1rho1 * vn_L + Rs.z1rho1 * vn_R;
    FD[1] = L.z2rho2 * vn_L + Rs.z2rho2 * vn_R;
    FD[2] = L.rho * vn_L * (xdir ? vn_L : ut_L) + Rs.rho * vn_R * (xdir ? vn_R : ut_R);
    FD[3] = L.rho * vn_L * (xdir ? ut_L : vn_L) + Rs.rho * vn_R * (xdir ? ut_R : vn_R);
    const double pm = 0.5 * (L.pd + Rs.pd);
#pragma unroll
    for (int r = 0; r < 4; ++r) F[r] = (double)(0.5f * (FD[r] - ws * (float)(URd[r] - ULd[r])));
    F[2] += pm * nx;
    F[3] += pm * ny;
}

__device__ __forceinline__ void tp_hllc_f32(const TPState<float> &L, const TPState<float> &Rs, double *F, bool xdir)
{
    const float vn_L = xdir ? L.u : L.v, vn_R = xdir ? Rs.u : Rs.v;
    const float sL = sqrtf(L.rho), sR = sqrtf(Rs.rho);
    const float is = 1.0f / (sL + sR);
    const float vn_roe = (vn_L * sL + vn_R * sR) * is;
    float c2_roe = (L.c * L.c * sL + Rs.c * Rs.c * sR) * is;
    c2_roe += 0.5f * sL * sR * is * is * (vn_R - vn_L) * (vn_R - vn_L);
    const float c_roe = sqrtf(c2_roe);
    const float S_L = std_min(vn_L - L.c, vn_roe - c_roe);
    const float S_R = std_max(vn_R + Rs.c, vn_roe + c_roe);
    const float dp = (float)(Rs.pd - L.pd);
    const float S_star = ((S_L - vn_L) * L.rho * vn_L - (S_R - vn_R) * Rs.rho * vn_R + dp) /
                         ((S_L - vn_L) * L.rho - (S_R - vn_R) * Rs.rho);
    const bool left = S_star >= 0.0f;
    const TPState<float> &K = left ? L : Rs;
    const float S_K = left ? S_L : S_R, vn_K = left ? vn_L : vn_R;
    const bool super = left ? (S_L >= 0.0f) : (S_R <= 0.0f);
    float a, b; // F = a U_K + b n (+ p_K n in FP64)
    if (super) {
        a = vn_K;
        b = 0.0f;
    } else {
        const float k = (S_K - vn_K) / (S_K - S_star);
        a = k * S_star;
        b = k * K.rho * S_K * (S_star - vn_K);
    }
    F[0] = (double)(a * K.z1rho1);
    F[1] = (double)(a * K.z2rho2);
    F[2] = (double)(a * K.rhou + (xdir ? b : 0.0f)) + (xdir ? K.pd : 0.0);
    F[3] = (double)(a * K.rhov + (xdir ? 0.0f : b)) + (xdir ? 0.0 : K.pd);
}

// Characteristic matrices of the two-phase system, include/Equations.hpp:189-327.
// Row k of L and row r of R in direction x (xdir) or y.
template <class R> struct TPEigen {
    R z1rho1, z2rho2, rho, u, v, c, c2, sc1_2, sc2_2;
    R i2c2, i2c, irc2, idsc, irho, pad; // reciprocals of the contracted build; pad: odd size in smem
};
#if !WENOFV_STRICT
// The linear model's eigensystem data in the contracted build, with two divisions and one
// square root besides the state recovery (the strict build keeps the reference's expressions).
// With A_k = z_k rho_k c_k^2 and S = z1^2 A2 + z2^2 A1 (the Wood sum of sound()):
//   c^2 = A1 A2 / (rho S),  1/(2c^2) = rho S / (2 A1 A2),  1/(rho c^2) = S / (A1 A2),
//   sc1^2 = c1^2 c2^2 z1 z2rho2 / S,  sc2^2 = c1^2 c2^2 z2 z1rho1 / S
// (sc_k^2 = c_k^2/z_k - c_k^2/z_k zrho_k / (zrho1 + zrho2), zrho_k = z_krho_k c_k^2 / z_k^2,
// multiplied through by z1^2 z2^2), and 1/(sc1^2 - sc2^2) = S / (c1^2 c2^2 (z1 z2rho2 - z2 z1rho1)).
// W = 1/(A1 A2 S) yields both 1/(A1 A2) and 1/S.
__device__ __forceinline__ void tp_eigen_prep_linear(const TwoPhaseK &K, const double *U, TPEigen<double> &e)
{
    const double m1 = U[0], m2 = U[1];
    e.z1rho1 = m1; e.z2rho2 = m2;
    e.rho = m1 + m2;
    double z1, pd;
    K.recover_rho(m1, m2, e.rho, e.irho, z1, pd);
    e.u = U[2] * e.irho;
    e.v = U[3] * e.irho;
    const double z2 = 1.0 - z1;
    const double A1 = m1 * K.c1_2, A2 = m2 * K.c2_2;
    const double Sw = z1 * z1 * A2 + z2 * z2 * A1;
    const double P = A1 * A2;
    const double W = 1.0 / (P * Sw);
    const double iS = P * W, iP = Sw * W;
    e.c2 = P * iS * e.irho;
    e.c = sqrt(e.c2);
    e.i2c2 = 0.5 * e.rho * Sw * iP;
    e.i2c = e.c * e.i2c2;
    e.irc2 = Sw * iP;
    const double B = K.c1_2 * K.c2_2;
    const double d1 = z1 * m2, d2 = z2 * m1;
    e.sc1_2 = B * d1 * iS;
    e.sc2_2 = B * d2 * iS;
    e.idsc = Sw / (B * (d1 - d2));
}
#endif
template <class R, class KT> __device__ __forceinline__ void tp_eigen_prep(const KT &K, const double *U, TPEigen<R> &e)
{
#if !WENOFV_STRICT
    if constexpr (sizeof(R) == sizeof(double) && KT::linear) {
        tp_eigen_prep_linear(K, U, e);
        return;
    }
#endif
    e.z1rho1 = (R)U[0]; e.z2rho2 = (R)U[1];
    e.rho = e.z1rho1 + e.z2rho2;
#if WENOFV_STRICT
    e.u = (R)U[2] / e.rho;
    e.v = (R)U[3] / e.rho;
#else
    e.irho = R(1) / e.rho;
    e.u = (R)U[2] * e.irho;
    e.v = (R)U[3] * e.irho;
#endif
    double z1d, pd;
    K.eigen_state(U[0], U[1], z1d, pd);
    const R z1 = (R)z1d;
    const R z2 = (R)(1.0 - z1d);
    e.c = K.template sound_p<R>(e.z1rho1, e.z2rho2, z1, z2, pd);
    e.c2 = e.c * e.c;
    R c1_2, c2_2;
    K.template phase_c2<R>(e.z1rho1, e.z2rho2, z1, z2, pd, c1_2, c2_2);
    if constexpr (sizeof(R) < sizeof(double)) {
        // FP32: the same quantities without the cancellation 1 - zrho1/(zrho1+zrho2) and
        // without dividing by z_k^2 (exact algebra: multiply zrho_k through by z1^2 z2^2)
        const R a = e.z1rho1 * c1_2 * (z2 * z2), b = e.z2rho2 * c2_2 * (z1 * z1);
        const R g = c1_2 * c2_2 / (a + b);
        e.sc1_2 = g * (z1 * e.z2rho2);
        e.sc2_2 = g * (z2 * e.z1rho1);
    } else {
        const R zrho1 = e.z1rho1 * c1_2 / (z1 * z1);
        const R zrho2 = e.z2rho2 * c2_2 / (z2 * z2);
        e.sc1_2 = c1_2 / z1 - c1_2 / z1 * zrho1 / (zrho1 + zrho2);
        e.sc2_2 = c2_2 / z2 - c2_2 / z2 * zrho2 / (zrho1 + zrho2);
    }
#if !WENOFV_STRICT
    e.i2c2 = R(1) / (R(2.0) * e.c2);
    e.i2c = e.c * e.i2c2; // c / (2 c^2) = 1/(2c)
    e.irc2 = R(1) / (e.rho * e.c2);
    e.idsc = R(1) / (e.sc1_2 - e.sc2_2);
#endif
}
template <class R> __device__ __forceinline__ void tp_L_row(const TPEigen<R> &e, bool xdir, int k, R *row)
{
    const R un = xdir ? e.u : e.v, ut = xdir ? e.v : e.u;
#if !WENOFV_STRICT // contracted build: multiplications by the prepared reciprocals
    switch (k) {
    case 0:
        row[0] = (e.sc1_2 + e.c * un) * e.i2c2;
        row[1] = (e.sc2_2 + e.c * un) * e.i2c2;
        row[2] = xdir ? -e.i2c : R(0);
        row[3] = xdir ? R(0) : -e.i2c;
        break;
    case 1:
        row[0] = -e.z2rho2 * (e.sc1_2 - e.sc2_2) * e.irc2;
        row[1] = e.z1rho1 * (e.sc1_2 - e.sc2_2) * e.irc2;
        row[2] = R(0);
        row[3] = R(0);
        break;
    case 2:
        row[0] = -ut;
        row[1] = -ut;
        row[2] = xdir ? R(0) : R(1.0);
        row[3] = xdir ? R(1.0) : R(0);
        break;
    default:
        row[0] = (e.sc1_2 - e.c * un) * e.i2c2;
        row[1] = (e.sc2_2 - e.c * un) * e.i2c2;
        row[2] = xdir ? e.i2c : R(0);
        row[3] = xdir ? R(0) : e.i2c;
        break;
    }
#else
    switch (k) {
    case 0:
        row[0] = (e.sc1_2 + e.c * un) / (R(2.0) * e.c2);
        row[1] = (e.sc2_2 + e.c * un) / (R(2.0) * e.c2);
        row[2] = xdir ? R(-1.0) / (R(2.0) * e.c) : R(0);
        row[3] = xdir ? R(0) : R(-1.0) / (R(2.0) * e.c);
        break;
    case 1:
        row[0] = -e.z2rho2 * (e.sc1_2 - e.sc2_2) / (e.rho * e.c2);
        row[1] = e.z1rho1 * (e.sc1_2 - e.sc2_2) / (e.rho * e.c2);
        row[2] = R(0);
        row[3] = R(0);
        break;
    case 2:
        row[0] = -ut;
        row[1] = -ut;
        row[2] = xdir ? R(0) : R(1.0);
        row[3] = xdir ? R(1.0) : R(0);
        break;
    default:
        row[0] = (e.sc1_2 - e.c * un) / (R(2.0) * e.c2);
        row[1] = (e.sc2_2 - e.c * un) / (R(2.0) * e.c2);
        row[2] = xdir ? R(1.0) / (R(2.0) * e.c) : R(0);
        row[3] = xdir ? R(0) : R(1.0) / (R(2.0) * e.c);
        break;
    }
#endif
}
template <class R> __device__ __forceinline__ void tp_R_row(const TPEigen<R> &e, bool xdir, int r, R *row)
{
    switch (r) {
    case 0:
#if WENOFV_STRICT
        row[0] = e.z1rho1 / e.rho;
        row[1] = -e.sc2_2 / (e.sc1_2 - e.sc2_2);
        row[3] = e.z1rho1 / e.rho;
#else
        row[0] = e.z1rho1 * e.irho;
        row[1] = -e.sc2_2 * e.idsc;
        row[3] = row[0];
#endif
        row[2] = R(0);
        break;
    case 1:
#if WENOFV_STRICT
        row[0] = e.z2rho2 / e.rho;
        row[1] = e.sc1_2 / (e.sc1_2 - e.sc2_2);
        row[3] = e.z2rho2 / e.rho;
#else
        row[0] = e.z2rho2 * e.irho;
        row[1] = e.sc1_2 * e.idsc;
        row[3] = row[0];
#endif
        row[2] = R(0);
        break;
    case 2:
        row[0] = xdir ? e.u - e.c : e.u;
        row[1] = e.u;
        row[2] = xdir ? R(0) : R(1);
        row[3] = xdir ? e.u + e.c : e.u;
        break;
    default:
        row[0] = xdir ? e.v : e.v - e.c;
        row[1] = e.v;
        row[2] = xdir ? R(1) : R(0);
        row[3] = xdir ? e.v : e.v + e.c;
        break;
    }
}

// ---- Euler, gamma-law gas, U = (rho, rho u, rho v, E).  No counterpart in the reference;
//      restated from the standard formulation (Toro, ch. 3 and 10) in the oracle's order.
template <class R> struct EUState {
    R rho, u, v, E, p, c, H;
    R ic, b1; // 1/c and (gamma-1)/c^2 of the contracted build (eigenvectors); odd size in smem
};
template <class R> __device__ __forceinline__ void eu_state(double gamma, const double *U, EUState<R> &s)
{
    // velocity and pressure recovered in FP64 in every form
    const double ud = U[1] / U[0], vd = U[2] / U[0];
    const double pd = (gamma - 1.0) * (U[3] - 0.5 * U[0] * (ud * ud + vd * vd));
    s.rho = (R)U[0];
    s.u = (R)ud;
    s.v = (R)vd;
    s.E = (R)U[3];
    s.p = (R)pd;
    s.c = sqrt(R(gamma) * s.p / s.rho);
    s.H = (s.E + s.p) / s.rho;
#if !WENOFV_STRICT
    s.ic = R(1.0) / s.c;
    s.b1 = R(gamma - 1.0) * s.ic * s.ic;
#endif
}
template <class R> __device__ __forceinline__ void eu_phy_flux(const EUState<R> &s, const R *U, R *F, R nx, R ny)
{
    const R vn = s.u * nx + s.v * ny;
    F[0] = U[0] * vn;
    F[1] = U[1] * vn + s.p * nx;
    F[2] = U[2] * vn + s.p * ny;
    F[3] = (U[3] + s.p) * vn;
}
template <class R>
__device__ __forceinline__ void eu_llf(const EUState<R> &L, const EUState<R> &Rs, const R *UL, const R *UR, R *F, bool xdir)
{
    const R nx = xdir ? R(1) : R(0), ny = xdir ? R(0) : R(1);
    const R wl = fabs(L.u * nx + L.v * ny) + L.c, wr = fabs(Rs.u * nx + Rs.v * ny) + Rs.c;
    const R ws = std_max(wl, wr);
    R FL[4], FR[4];
    eu_phy_flux(L, UL, FL, nx, ny);
    eu_phy_flux(Rs, UR, FR, nx, ny);
#pragma unroll
    for (int r = 0; r < 4; ++r) F[r] = R(0.5) * (FL[r] + FR[r] - ws * (UR[r] - UL[r]));
}
template <class R>
__device__ __forceinline__ void eu_hllc(double gamma, const EUState<R> &L, const EUState<R> &Rs, const R *UL, const R *UR, R *F, bool xdir)
{
    const R nx = xdir ? R(1) : R(0), ny = xdir ? R(0) : R(1);
    const R rL = L.rho, rR = Rs.rho;
    const R vnL = L.u * nx + L.v * ny, vnR = Rs.u * nx + Rs.v * ny;
    const R sL = sqrt(rL), sR = sqrt(rR);
    const R inv = R(1.0) / (sL + sR);
    const R ur = (sL * L.u + sR * Rs.u) * inv, vr = (sL * L.v + sR * Rs.v) * inv;
    const R Hr = (sL * L.H + sR * Rs.H) * inv;
    const R vnr = ur * nx + vr * ny;
    const R cr = sqrt(R(gamma - 1.0) * (Hr - R(0.5) * (ur * ur + vr * vr)));
    const R S_L = std_min(vnL - L.c, vnr - cr);
    const R S_R = std_max(vnR + Rs.c, vnr + cr);
    const R S_star = (Rs.p - L.p + rL * vnL * (S_L - vnL) - rR * vnR * (S_R - vnR)) / (rL * (S_L - vnL) - rR * (S_R - vnR));
    R FL[4], FR[4];
    eu_phy_flux(L, UL, FL, nx, ny);
    eu_phy_flux(Rs, UR, FR, nx, ny);
    if (S_L >= R(0.0)) {
#pragma unroll
        for (int r = 0; r < 4; r++) F[r] = FL[r];
    } else if (S_star >= R(0.0)) {
        const R k = rL * (S_L - vnL) / (S_L - S_star);
        R Us[4];
        Us[0] = k;
        Us[1] = k * (L.u + (S_star - vnL) * nx);
        Us[2] = k * (L.v + (S_star - vnL) * ny);
        Us[3] = k * (UL[3] / rL + (S_star - vnL) * (S_star + L.p / (rL * (S_L - vnL))));
#pragma unroll
        for (int r = 0; r < 4; r++) F[r] = FL[r] + S_L * (Us[r] - UL[r]);
    } else if (S_R > R(0.0)) {
        const R k = rR * (S_R - vnR) / (S_R - S_star);
        R Us[4];
        Us[0] = k;
        Us[1] = k * (Rs.u + (S_star - vnR) * nx);
        Us[2] = k * (Rs.v + (S_star - vnR) * ny);
        Us[3] = k * (UR[3] / rR + (S_star - vnR) * (S_star + Rs.p / (rR * (S_R - vnR))));
#pragma unroll
        for (int r = 0; r < 4; r++) F[r] = FR[r] + S_R * (Us[r] - UR[r]);
    } else {
#pragma unroll
        for (int r = 0; r < 4; r++) F[r] = FR[r];
    }
}
// Euler eigenvectors in direction n (columns of R: u-c, entropy, shear, u+c)
template <class R> __device__ __forceinline__ void eu_L_row(double gamma, const EUState<R> &s, bool xdir, int k, R *row)
{
    const R nx = xdir ? R(1) : R(0), ny = xdir ? R(0) : R(1);
    const R q2 = R(0.5) * (s.u * s.u + s.v * s.v);
    const R vn = s.u * nx + s.v * ny, vt = s.v * nx - s.u * ny;
#if WENOFV_STRICT
    const R b1 = R(gamma - 1.0) / (s.c * s.c), b2 = q2 * b1;
    const R vnc = vn / s.c, nxc = nx / s.c, nyc = ny / s.c;
#else
    const R b1 = s.b1, b2 = q2 * b1;
    const R vnc = vn * s.ic, nxc = nx * s.ic, nyc = ny * s.ic;
#endif
    switch (k) {
    case 0:
        row[0] = R(0.5) * (b2 + vnc); row[1] = R(0.5) * (-b1 * s.u - nxc);
        row[2] = R(0.5) * (-b1 * s.v - nyc); row[3] = R(0.5) * b1;
        break;
    case 1:
        row[0] = R(1.0) - b2; row[1] = b1 * s.u; row[2] = b1 * s.v; row[3] = -b1;
        break;
    case 2:
        row[0] = -vt; row[1] = -ny; row[2] = nx; row[3] = R(0.0);
        break;
    default:
        row[0] = R(0.5) * (b2 - vnc); row[1] = R(0.5) * (-b1 * s.u + nxc);
        row[2] = R(0.5) * (-b1 * s.v + nyc); row[3] = R(0.5) * b1;
        break;
    }
}
template <class R> __device__ __forceinline__ void eu_R_row(const EUState<R> &s, bool xdir, int r, R *row)
{
    const R nx = xdir ? R(1) : R(0), ny = xdir ? R(0) : R(1);
    const R q2 = R(0.5) * (s.u * s.u + s.v * s.v);
    const R vn = s.u * nx + s.v * ny, vt = s.v * nx - s.u * ny;
    switch (r) {
    case 0: row[0] = R(1.0); row[1] = R(1.0); row[2] = R(0.0); row[3] = R(1.0); break;
    case 1: row[0] = s.u - s.c * nx; row[1] = s.u; row[2] = -ny; row[3] = s.u + s.c * nx; break;
    case 2: row[0] = s.v - s.c * ny; row[1] = s.v; row[2] = nx; row[3] = s.v + s.c * ny; break;
    default: row[0] = s.H - s.c * vn; row[1] = q2; row[2] = vt; row[3] = s.H + s.c * vn; break;
    }
}

// ------------------------------------------------------------------------------------
// equation dispatch (the equation kind is a template parameter of every kernel)
// ------------------------------------------------------------------------------------
template <int EQ> struct EqTraits { static constexpr int NV = 4; };
template <> struct EqTraits<EQ_LINEAR_ADV> { static constexpr int NV = 1; };

// getMaxEigenValue (include/Equations.hpp:149-156) for the CFL and the limiter's mu
template <int EQ, class R> __device__ __forceinline__ void max_eigs(const EqParams &P, const double *U, R &ax, R &ay)
{
    if constexpr (IsTwoPhase<EQ>::value) {
        const typename TPKOf<EQ>::type K(P);
        TPState<R> s;
        tp_state<R>(K, U, s);
        ax = tp_max_eig(s, 1.0, 0.0);
        ay = tp_max_eig(s, 0.0, 1.0);
    } else if constexpr (EQ == EQ_EULER) {
        EUState<R> s;
        eu_state<R>(P.gamma, U, s);
        ax = fabs(s.u * R(1.0) + s.v * R(0.0)) + s.c;
        ay = fabs(s.u * R(0.0) + s.v * R(1.0)) + s.c;
    } else {
        ax = fabs(R(P.adv_u) * R(1.0) + R(P.adv_v) * R(0.0));
        ay = fabs(R(P.adv_u) * R(0.0) + R(P.adv_v) * R(1.0));
    }
}

// getRiemannFlux dispatch (include/Equations.hpp:329-343); flux 0 LLF, 1 HLLC.
// For scalar advection both are the upwind (LLF with |a.n|) flux.
// The face states come in FP64 and the flux goes out in FP64 in every form.
// FL: the flux as a compile-time constant (0 LLF, 1 HLLC) in the stage kernels, or -1 to take
// it from the argument (the pointwise probes)
template <int EQ, class R, int FL = -1>
__device__ __forceinline__ void riemann(const EqParams &P, int flux_arg, const double *ULd, const double *URd, double *F, bool xdir)
{
    const int flux = FL < 0 ? flux_arg : FL;
    constexpr int NV = EqTraits<EQ>::NV;
    constexpr bool F32 = sizeof(R) < sizeof(double);
    R UL[NV], UR[NV], Fr[NV];
#pragma unroll
    for (int v = 0; v < NV; v++) { UL[v] = (R)ULd[v]; UR[v] = (R)URd[v]; }
    if constexpr (IsTwoPhase<EQ>::value) {
        const typename TPKOf<EQ>::type K(P);
        TPState<R> l, r;
        tp_state_pair<R>(K, ULd, URd, l, r);
        if constexpr (F32) {
            if (flux == 1) tp_hllc_f32(l, r, F, xdir);
            else tp_llf_f32(l, r, ULd, URd, F, xdir);
        } else {
            if (flux == 1) tp_hllc<R>(l, r, UL, UR, Fr, xdir);
            else tp_llf<R>(l, r, UL, UR, Fr, xdir);
        }
    } else if constexpr (EQ == EQ_EULER) {
        if constexpr (F32) {
            // FP32-bulk: the Euler flux stays FP64.  In FP32 the star flux F_K + S_K (U* - U_K)
            // and the pressure terms round away the small flux differences between the two
            // faces of a cell, which moved shock solutions by ~1e-4 (relative L1) within
            // ~1000 steps; the reconstruction is the FP32 part of this equation's bulk form.
            EUState<double> l, r;
            eu_state<double>(P.gamma, ULd, l);
            eu_state<double>(P.gamma, URd, r);
            if (flux == 1) eu_hllc<double>(P.gamma, l, r, ULd, URd, F, xdir);
            else eu_llf<double>(l, r, ULd, URd, F, xdir);
        } else {
            EUState<R> l, r;
            eu_state<R>(P.gamma, ULd, l);
            eu_state<R>(P.gamma, URd, r);
            if (flux == 1) eu_hllc<R>(P.gamma, l, r, UL, UR, Fr, xdir);
            else eu_llf<R>(l, r, UL, UR, Fr, xdir);
        }
    } else {
        const R an = xdir ? (R(P.adv_u) * R(1.0) + R(P.adv_v) * R(0.0)) : (R(P.adv_u) * R(0.0) + R(P.adv_v) * R(1.0));
        const R ws = std_max(fabs(an), fabs(an));
        Fr[0] = R(0.5) * (an * UL[0] + an * UR[0] - ws * (UR[0] - UL[0]));
    }
    if constexpr (!(F32 && (IsTwoPhase<EQ>::value || EQ == EQ_EULER))) { // those FP32 forms write F themselves
#pragma unroll
        for (int v = 0; v < NV; v++) F[v] = (double)Fr[v];
    }
}

// Characteristic projection rows: row k of L and row k of R for the state U.
template <int EQ, class R>
__device__ __forceinline__ void eigen_rows(const EqParams &P, const double *U, bool xdir, int k, R *Lrow, R *Rrow)
{
    if constexpr (IsTwoPhase<EQ>::value) {
        const typename TPKOf<EQ>::type K(P);
        TPEigen<R> e;
        tp_eigen_prep<R>(K, U, e);
        tp_L_row<R>(e, xdir, k, Lrow);
        tp_R_row<R>(e, xdir, k, Rrow);
    } else if constexpr (EQ == EQ_EULER) {
        EUState<R> s;
        eu_state<R>(P.gamma, U, s);
        eu_L_row<R>(P.gamma, s, xdir, k, Lrow);
        eu_R_row<R>(s, xdir, k, Rrow);
    } else {
        Lrow[0] = R(1.0);
        Rrow[0] = R(1.0);
    }
}

// Primitive variables of the two-phase model (FP64 in every form) for RECONSTRUCTIONTYPE 2
// (PRIMITIVE: z1, rho1, u, v; src/WENOFV.cpp:944-959) and 3 (PRIMITIVE2: z1, p, u, v;
// :1102-1121), and back to conserved variables at the Gauss points (:1002-1025, :1178-1189).
__device__ __forceinline__ void tp_to_primitive(const EqParams &P, int recon, const double *U, double *W)
{
    const TwoPhaseK K(P);
    const double z1 = K.volume_frac(U[0], U[1]);
    W[0] = z1;
    if (recon == 2) W[1] = U[0] / z1;
    else if (z1 > 0.5) W[1] = P.preb + K.c1_2 * (U[0] / z1 - P.rho10);
    else W[1] = P.preb + K.c2_2 * (U[1] / (1.0 - z1) - P.rho20);
    W[2] = U[2] / (U[0] + U[1]);
    W[3] = U[3] / (U[0] + U[1]);
}
__device__ __forceinline__ void tp_from_primitive(const EqParams &P, int recon, const double *W, double *U)
{
    const TwoPhaseK K(P);
    const double z1 = W[0];
    double z1rho1, z2rho2;
    if (recon == 2) {
        z2rho2 = K.c1_2 / K.c2_2 * (W[1] - P.rho10) + P.rho20;
        z2rho2 = z2rho2 * (1.0 - z1);
        z1rho1 = z1 * W[1];
    } else {
        z1rho1 = ((W[1] - P.preb) / K.c1_2 + P.rho10) * z1;
        z2rho2 = ((W[1] - P.preb) / K.c2_2 + P.rho20) * (1.0 - z1);
    }
    const double rho = z1rho1 + z2rho2;
    U[0] = z1rho1;
    U[1] = z2rho2;
    U[2] = rho * W[2];
    U[3] = rho * W[3];
}

// Per-cell eigensystem data, computed once per cell and row in FP64 (every form) and shared
// by the lanes that build its rows of L and R and by the limiter's wave speeds.
template <int EQ> struct CellEigen { using type = TPEigen<double>; };
template <> struct CellEigen<EQ_EULER> { using type = EUState<double>; };

template <int EQ> __device__ __forceinline__ void cell_eigen(const EqParams &P, const double *U, typename CellEigen<EQ>::type &e)
{
    if constexpr (IsTwoPhase<EQ>::value) {
        const typename TPKOf<EQ>::type K(P);
        tp_eigen_prep<double>(K, U, e);
    } else if constexpr (EQ == EQ_EULER) {
        eu_state<double>(P.gamma, U, e);
    }
}
template <int EQ>
__device__ __forceinline__ void eigen_rows_of(const EqParams &P, const typename CellEigen<EQ>::type &e, bool xdir, int k,
                                              double *Lrow, double *Rrow)
{
    if constexpr (IsTwoPhase<EQ>::value) {
        tp_L_row<double>(e, xdir, k, Lrow);
        tp_R_row<double>(e, xdir, k, Rrow);
    } else if constexpr (EQ == EQ_EULER) {
        eu_L_row<double>(P.gamma, e, xdir, k, Lrow);
        eu_R_row<double>(e, xdir, k, Rrow);
    } else {
        Lrow[0] = 1.0;
        Rrow[0] = 1.0;
    }
}
// getMaxEigenValue in x and y from the cell data (the same expressions as max_eigs)
template <int EQ> __device__ __forceinline__ void max_eigs_of(const typename CellEigen<EQ>::type &e, double &ax, double &ay)
{
    ax = fabs(e.u * 1.0 + e.v * 0.0) + e.c;
    ay = fabs(e.u * 0.0 + e.v * 1.0) + e.c;
}

// number of leading variables the bound-preserving limiter acts on: the two partial
// densities of the two-phase model (src/WENOFV.cpp:1964), the density for Euler, none for
// scalar advection
template <int EQ> struct LimitedVars { static constexpr int N = IsTwoPhase<EQ>::value ? 2 : (EQ == EQ_EULER ? 1 : 0); };

// Gauss-Lobatto 4-point weights as written at third_party/scTools/GaussQuadratureInRef.hpp:252-262
__device__ __forceinline__ double gl_weight(int gp)
{
    return (gp == 0 || gp == 3) ? 0.166666666666666666666666666667 : 0.833333333333333333333333333333;
}

} // namespace strict / fast
} // namespace wenofv
