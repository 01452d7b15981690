// Equations.hpp -- TwoPhaseEquation on the host side of the CUDA backend.
//
// Keeps the reference's equation object (include/Equations.hpp:52-1044): the test-case
// enum and its numbers, the public parameters g_rho10, g_rho20, g_sound1, g_sound2, g_u0,
// g_v0, g_preb, g_epsa, the domain xL..yR, outputTimes, boundaryCondition, getVarNum,
// setEquationParameters and getU0.  The pointwise physics (volume fraction, pressure,
// sound speed, fluxes, eigenvectors) runs on the GPU inside libwenofv_b200; params()
// hands the parameters to it as the C-ABI POD.
//
// setEquationParameters covers the periodic test cases the reference can run (SMOOTH,
// VORTEX, SHARP: include/Equations.hpp:490-689) and the wall cases it declares but cannot
// run, because it stops on their boundary kind (src/WENOFV.cpp:2286-2292): DAMBREAK,
// DAMBREAK2, DAMBREAK3, RTI and STANDING_WAVE (include/Equations.hpp:747-973), with the
// library's NEUMANN walls and the gravity of assembleSourceTerm (src/WENOFV.cpp:1831-1872).
// ZALESAK (:690-745), a disc of radius 0.15 in solid-body rotation about the centre, selects
// NEUMANN2 (boundary from the initial data): CWENOFV builds the fixed ghost frame from the
// initial averages of the 4 cell layers around the domain.  Other cases throw
// std::invalid_argument, like an unknown case does in the reference (:975).
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
    double g_g0 = 0.0; // assembleSourceTerm's gravity of the case

    int getVarNum() const { return 4; }

    // the parameter sets of the test cases (include/Equations.hpp:490-973)
    void setEquationParameters(TESTCASETYPE type)
    {
        testcase = type;
        boundaryCondition = PERIOD;
        g_g0 = 0.0;
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
        case STANDING_WAVE: // (:747-789)
            set_box(0.0, 0.5, 0.0, 0.5);
            outputTimes = {3.0};
            set_phase(1000.0, 1.0, 100.0, 100.0, 0.0, 0.0, 1e-6, 1e4);
            walls(2 * M_PI);
            break;
        case RTI: // (:791-829)
            set_box(0.0, 1.0, 0.0, 4.0);
            outputTimes = {0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.0};
            set_phase(1.225, 0.1694, 100.0, 100.0, 0.0, 0.0, 1.0e-8, 10000.0);
            walls(9.81);
            break;
        case DAMBREAK: // (:831-877)
            set_box(0.0, 1.61, 0.0, 0.805);
            outputTimes = {0.0, 0.1599, 0.2766, 0.3733, 0.4499, 0.5733, 0.8623, 1.0233, 1.1666};
            set_phase(1000.0, 1.0, 100.0, 100.0, 0.0, 0.0, 1e-6, 1e4);
            walls(9.81);
            break;
        case DAMBREAK2: // (:879-925)
            set_box(0.0, 1.61, 0.0, 0.6);
            outputTimes = {1.5};
            set_phase(1000.0, 1.0, 100.0, 100.0, 0.0, 0.0, 1e-5, 1e4);
            walls(9.81);
            break;
        case DAMBREAK3: // (:927-973)
            set_box(0.0, 0.8, 0.0, 0.6);
            outputTimes = {1.5};
            set_phase(1000.0, 1.0, 100.0, 100.0, 0.0, 0.0, 1e-5, 1e4);
            walls(9.81);
            break;
        case ZALESAK: // (:690-745)
            set_box(0.0, 1.0, 0.0, 1.0);
            outputTimes = {2};
            set_phase(1000.0, 1.0, 70.0, 70.0, 1.0, 1.0, 1e-8);
            boundaryCondition = NEUMANN2;
            break;
        default:
            throw std::invalid_argument(std::string("test case ") + std::to_string((int)type) + " is not supported");
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
        case STANDING_WAVE: { // liquid below y = 0.25 + 0.025 cos(2 pi x) (:764-773)
            const double hs = 0.25, A = 0.025, kn = 2 * M_PI;
            return (y <= hs + A * std::cos(kn * x)) ? 1.0 - g_epsa : g_epsa;
        }
        case RTI: { // the heavy phase above y = 2 + 0.05 cos(2 pi x) (:814-820)
            const double yi = 2.0 + 0.05 * std::cos(2.0 * M_PI * x);
            return (y >= yi) ? 1.0 - g_epsa : g_epsa;
        }
        case DAMBREAK:  // a water block of L0 x H0 at the right (:855-861)
        case DAMBREAK2: // (:903-909)
        case DAMBREAK3: { // at the left (:951-957)
            const double H0 = testcase == DAMBREAK ? 0.3 : (testcase == DAMBREAK2 ? 0.6 : 0.4);
            const double L0 = testcase == DAMBREAK3 ? 0.2 : 0.6;
            if (testcase == DAMBREAK3)
                return (x >= xL && x <= xL + L0 && y >= yL && y <= yL + H0) ? 1.0 - g_epsa : g_epsa;
            return (x >= xR - L0 && x <= xR && y >= yL && y <= yL + H0) ? 1.0 - g_epsa : g_epsa;
        }
        case ZALESAK: { // disc of radius 0.15 at (0.5, 0.5) (:717-723)
            const double x0 = 0.5, y0 = 0.5, r = 0.15;
            return (std::pow(x - x0, 2) + std::pow(y - y0, 2) < std::pow(r, 2)) ? 1 - g_epsa : g_epsa;
        }
        default:
            return g_epsa;
        }
    }

    // getU0 (include/Equations.hpp:979-1002): partial densities from the phase pressures
    // (uniform g_preb in every case built here) and momenta from the uniform velocity
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
        if (testcase == ZALESAK) return M_PI * (0.5 - y); // rotation at omega = pi (:729-733)
        (void)x;
        return g_u0;
    }
    double v_0(double x, double y) const
    {
        if (testcase == ZALESAK) return M_PI * (x - 0.5); // (:734-738)
        (void)y;
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
        p.gravity = g_g0;
        return p;
    }

private:
    void set_box(double xl, double xr, double yl, double yr) { xL = xl; xR = xr; yL = yl; yR = yr; }
    void set_phase(double rho10, double rho20, double c1, double c2, double u0, double v0, double epsa, double preb = 0.0)
    {
        g_rho10 = rho10; g_rho20 = rho20; g_sound1 = c1; g_sound2 = c2;
        g_u0 = u0; g_v0 = v0; g_preb = preb; g_epsa = epsa;
    }
    void walls(double g)
    {
        boundaryCondition = NEUMANN;
        g_g0 = g;
    }
    static double wrap(double v, double lo, double hi)
    {
        while (v >= hi) v -= hi - lo;
        while (v < lo) v += hi - lo;
        return v;
    }
};
