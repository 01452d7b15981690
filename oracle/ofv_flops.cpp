// ofv_flops.cpp -- algorithmic flop table per cell-stage, from the counting build of the
// oracle.  TEST INFRASTRUCTURE ONLY.
//
// For each option combination one RHS evaluation is counted on n x n periodic grids for
// n = 32, 64, 128; the counts fit C(n) = a n^2 + b n + c exactly (the one-cell halo ring
// scales with n), and a is the per-cell figure.  The RK combination adds 5 flops per
// variable ((a*Un + b*U) + (c*dt)*rhs) and the CFL reduction of the final stage adds its
// counted per-cell cost divided by the stage count (3 for SSP-RK3).
#include <cmath>
#include <cstdio>
#include <vector>

#include "ofv_count.hpp"
#include "wenofv_oracle.h"

static double smooth(double x, double y) { return std::sin(2 * M_PI * x) * std::cos(2 * M_PI * y); }

static void init_state(const ofv_problem &p, std::vector<double> &U)
{
    const int nx = p.nx, ny = p.ny, nv = ofv_nvar(&p.eq);
    U.assign((size_t)nv * nx * ny, 0.0);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double x = (i + 0.5) / nx, y = (j + 0.5) / ny, s = smooth(x, y);
            const size_t k = (size_t)j * nx + i, n = (size_t)nx * ny;
            if (p.eq.kind == OFV_EQ_LINEAR_ADV) {
                U[k] = s;
            } else if (p.eq.kind == OFV_EQ_EULER) {
                const double rho = 1.0 + 0.2 * s, u = 0.3, v = -0.2, pr = 1.0 + 0.1 * s;
                U[k] = rho; U[n + k] = rho * u; U[2 * n + k] = rho * v;
                U[3 * n + k] = pr / 0.4 + 0.5 * rho * (u * u + v * v);
            } else {
                const double z1 = 0.5 + 0.4 * s;
                U[k] = z1 * 1000.0; U[n + k] = (1 - z1) * 1.0;
                U[2 * n + k] = (U[k] + U[n + k]) * 0.1; U[3 * n + k] = (U[k] + U[n + k]) * -0.1;
            }
        }
}

static double total(const ofv_counters &c) { return (double)(c.add + c.mul + c.div + c.sqrt + c.tr); }

static double count_rhs(ofv_problem p, int n, ofv_counters *out)
{
    p.nx = p.ny = n;
    std::vector<double> U, R;
    init_state(p, U);
    R.assign(U.size(), 0.0);
    g_ofv_cnt = ofv_counters{};
    ofv_rhs(&p, U.data(), R.data(), nullptr);
    if (out) *out = g_ofv_cnt;
    return total(g_ofv_cnt);
}

int main()
{
    const char *eqn[] = {"two_phase", "linear_advection", "euler", "two_phase_sg"};
    for (int eqk = 0; eqk < 4; eqk++)
        for (int recon = 0; recon < 5; recon++)
            for (int scheme = 0; scheme < 3; scheme++)
                for (int flux = 0; flux < 2; flux++)
                    for (int lim = 0; lim < 2; lim++) {
                        if (eqk == OFV_EQ_LINEAR_ADV && (recon || flux || lim)) continue;
                        if (recon >= 2 && eqk != OFV_EQ_TWO_PHASE) continue; // primitive forms: two-phase only
                        if (recon == 4 && scheme != 1) continue;               // PRIMITIVE3 ignores SCHEME
                        ofv_problem p{};
                        p.xl = 0; p.xr = 1; p.yl = 0; p.yr = 1;
                        p.bc = OFV_BC_PERIOD; p.rk = 2; p.cfl = 0.5;
                        p.scheme = scheme; p.flux = flux; p.recon = recon; p.limiter = lim;
                        p.threads = 1;
                        p.eq.kind = eqk;
                        p.eq.rho10 = 1000; p.eq.rho20 = 1; p.eq.sound1 = 70; p.eq.sound2 = 70;
                        p.eq.gamma = 1.4; p.eq.adv_u = 1; p.eq.adv_v = 1;
                        if (eqk == OFV_EQ_TWO_PHASE_SG) { // at the reference pressure (rho_k = rho_k0)
                            p.eq.preb = 1.0;
                            p.eq.gamma1 = 4.4; p.eq.pinf1 = 6000; p.eq.gamma2 = 1.4; p.eq.pinf2 = 0;
                        }
                        const double c1 = count_rhs(p, 32, nullptr), c2 = count_rhs(p, 64, nullptr);
                        ofv_counters k3;
                        const double c3 = count_rhs(p, 128, &k3);
                        // C(n) = a n^2 + b n + c through n = 32, 64, 128
                        const double d1 = (c2 - c1) / 32.0, d2 = (c3 - c2) / 64.0;
                        const double a = (d2 - d1) / (128.0 - 32.0);
                        const int nv = ofv_nvar(&p.eq);
                        // CFL per cell, counted on a 64^2 grid
                        p.nx = p.ny = 64;
                        std::vector<double> U;
                        init_state(p, U);
                        g_ofv_cnt = ofv_counters{};
                        ofv_compute_dt(&p, U.data(), nullptr);
                        const double cfl = total(g_ofv_cnt) / (64.0 * 64.0);
                        const double rk = 5.0 * nv;
                        const double per_cs = a + rk + cfl / 3.0;
                        const double sq = (double)k3.sqrt / (128.0 * 128.0), dv = (double)k3.div / (128.0 * 128.0);
                        std::printf("{\"eq\": \"%s\", \"recon\": %d, \"scheme\": %d, \"flux\": %d, \"limiter\": %d, "
                                    "\"rhs_flops_per_cell\": %.1f, \"rk_flops\": %.0f, \"cfl_flops_per_cell\": %.1f, "
                                    "\"flops_per_cell_stage\": %.1f, \"div_per_cell\": %.1f, \"sqrt_per_cell\": %.1f}\n",
                                    eqn[eqk], recon, scheme, flux, lim, a, rk, cfl, per_cs, dv, sq);
                    }
    return 0;
}
