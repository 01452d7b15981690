// Equations.hpp -- TwoPhaseEquation on the host side of the CUDA backend.
//
// Keeps the reference's equation object (include/Equations.hpp:52-1044): the test-case
// enum and its numbers, the public parameters g_rho10, g_rho20, g_sound1, g_sound2, g_u0,
// g_v0, g_preb, g_epsa, the domain xL..yR, outputTimes, boundaryCondition, getVarNum,
// setEquationParameters and getU0.  The pointwise physics (volume fraction, pressure,
// sound speed, fluxes, eigenvectors) runs on the GPU inside libwenofv_b200; params()
// hands the parameters to it as the C-ABI POD.
//
// setEquationParameters covers the periodic test cases the reference can run
// (SMOOTH, VORTEX, SHARP: include/Equations.hpp:490-689).  The others need the
// reference's unimplemented non-periodic boundary conditions and a gravity source; they
// throw std::invalid_argument, like an unknown case does in the reference (:975).
#pragma once
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/wenofv.h"

enum RIEMANNFLUXTYPE { LLF = 0, HLLC = 1 };

enum TESTCASETYPE {
    SMOOTH = 0,
    VORTEX = 1,
    SHARP = 2,
    DAMBREAK = 3,
    DAMBREAK2 = 4,
    DAMBREAK3 = 5,
    RTI = 6,
    STANDING_WAVE = 7,
    ZALESAK = 8,
};

enum BOUNDARYTYPE { PERIOD = 0, NEUMANN = 1, NoSlip = 2, NEUMANN2 = 3, FREESLIP = 4 };

inline const char *const TESTCASETYPE_STRINGS[] = {"SMOOTH", "VORTEX", "SHARP", "DAMBREAK", "DAMBREAK2",
                                                    "DAMBREAK3", "RTI", "STANDING_WAVE", "ZALESAK"};

class TwoPhaseEquation
{
public:
    double xL = 0, xR = 1, yL = 0, yR = 1;
    std::vector<double> outputTimes;
    BOUNDARYTYPE boundaryCondition = PERIOD;
    TESTCASETYPE testcase = SMOOTH;

    double g_rho10 = 1.2, g_rho20 = 1.0;
    double g_sound1 = 1.0, g_sound2 = 1.0;
    double g_u0 = 1.0, g_v0 = 1.0, g_preb = 0.0;
    double g_epsa = 1e-8;

    int getVarNum() const { return 4; }

    // the parameter sets of the periodic cases (include/Equations.hpp:490-689)
    void setEquationParameters(TESTCASETYPE type)
    {
        testcase = type;
        boundaryCondition = PERIOD;
        switch (type) {
        case SMOOTH:
            set_box(0.0, 1.0, 0.0, 1.0);
            outputTimes = {0, 0.05};
            set_phase(1.2, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0e-8);
            break;
        case VORTEX:
            set_box(-1.0, 1.0, -1.0, 1.0);
            outputTimes = {0, 0.005, 0.01};
            set_phase(1000.0, 1.0, 30.0, 30.0, 2.0, 2.0, 1.0e-4);
            break;
        case SHARP:
            set_box(0.0, 1.0, 0.0, 1.0);
            outputTimes = {0, 1.0};
            set_phase(1000.0, 1.0, 70.0, 70.0, 1.0, 1.0, 1e-8);
            break;
        default:
            throw std::invalid_argument(std::string("test case ") + TESTCASETYPE_STRINGS[type] +
                                        " needs non-periodic boundaries and gravity, which the CUDA backend does not provide");
        }
    }

    // initial volume fraction of phase 1 at (x, y)
    double z1_0(double x, double y) const
    {
        switch (testcase) {
        case SMOOTH: // the active (x-only) profile of include/Equations.hpp:514-515
            return g_epsa + (1 - 2 * g_epsa) * std::pow(std::sin(2.0 * M_PI * x), 2);
        case VORTEX: { // Gaussian bump on the periodic [-1,1)^2 box (:538-549)
            x = wrap(x, -1.0, 1.0);
            y = wrap(y, -1.0, 1.0);
            const double r = std::sqrt(x * x + y * y);
            return (1 - 2 * g_epsa) * std::exp(-std::pow(r, 2) / std::pow(0.2, 2)) + g_epsa;
        }
        case SHARP: { // square of half-width (xR-xL)/10 at the centre (:651-660)
            const double r = (xR - xL) / 10.0;
            const double xc = (xL + xR) / 2.0, yc = (yL + yR) / 2.0;
            return (std::fabs(x - xc) < r && std::fabs(y - yc) < r) ? 1 - g_epsa : g_epsa;
        }
        default:
            return g_epsa;
        }
    }

    // getU0 (include/Equations.hpp:979-1002): partial densities from the phase pressures
    // (uniform g_preb in every periodic case) and momenta from the uniform velocity
    void getU0(double xP, double yP, double *U) const
    {
        const double z_1 = z1_0(xP, yP);
        const double z_2 = 1.0 - z_1;
        const double p_1 = g_preb, p_2 = g_preb;
        const double rho10 = (p_1 - g_preb) / std::pow(g_sound1, 2) + g_rho10;
        const double rho20 = (p_2 - g_preb) / std::pow(g_sound2, 2) + g_rho20;
        const double z1rho1 = rho10 * z_1;
        const double z2rho2 = rho20 * z_2;
        const double rho = z1rho1 + z2rho2;
        U[0] = z1rho1;
        U[1] = z2rho2;
        U[2] = rho * u_0(xP, yP);
        U[3] = rho * v_0(xP, yP);
    }

    double u_0(double x, double y) const
    {
        // VORTEX adds r*0 + theta*0 + L*0 to g_u0 (:589-604), which is g_u0 for finite r
        (void)x; (void)y;
        return g_u0;
    }
    double v_0(double x, double y) const
    {
        (void)x; (void)y;
        return g_v0;
    }

    wenofv_eq_params params() const
    {
        wenofv_eq_params p{};
        p.eq_kind = WENOFV_EQ_TWO_PHASE;
        p.rho10 = g_rho10;
        p.rho20 = g_rho20;
        p.sound1 = g_sound1;
        p.sound2 = g_sound2;
        p.preb = g_preb;
        p.gamma = 1.4;
        return p;
    }

private:
    void set_box(double xl, double xr, double yl, double yr) { xL = xl; xR = xr; yL = yl; yR = yr; }
    void set_phase(double rho10, double rho20, double c1, double c2, double u0, double v0, double epsa)
    {
        g_rho10 = rho10; g_rho20 = rho20; g_sound1 = c1; g_sound2 = c2;
        g_u0 = u0; g_v0 = v0; g_preb = 0.0; g_epsa = epsa;
    }
    static double wrap(double v, double lo, double hi)
    {
        while (v >= hi) v -= hi - lo;
        while (v < lo) v += hi - lo;
        return v;
    }
};
