// WENOFV.cpp -- CWENOFV methods of the CUDA backend (the reference's src/WENOFV.cpp:16-566
// call structure; the per-cell work runs in libwenofv_b200).
#include "../include/WENOFV.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>

namespace {
// 4-point Gauss-Legendre rule on [-1, 1] (the reference's GaussLegendre_ref, case 4,
// third_party/scTools/GaussQuadratureInRef.hpp:64-75)
const double kGLegX[4] = {-0.861136311594052575223946488893, -0.339981043584856264802665759103,
                          0.339981043584856264802665759103, 0.861136311594052575223946488893};
const double kGLegW[4] = {0.347854845137453857373063949222, 0.652145154862546142626936050778,
                          0.652145154862546142626936050778, 0.347854845137453857373063949222};
} // namespace

CWENOFV::CWENOFV(TwoPhaseEquation *eq, std::map<std::string, std::string> opts) : equation(eq), option(std::move(opts)) {}

CWENOFV::~CWENOFV()
{
    if (m_ctx) wenofv_destroy(m_ctx);
}

std::string CWENOFV::opt(const std::string &key, const std::string &dflt) const
{
    const auto it = option.find(key);
    return it == option.end() || it->second.empty() ? dflt : it->second;
}

void CWENOFV::check(int rc, const char *what) const
{
    if (rc != WENOFV_OK)
        throw std::runtime_error(std::string(what) + ": " + wenofv_strerror(rc) + " -- " + wenofv_last_error());
}

// option parsing and the grid of initializeSolver (src/WENOFV.cpp:43-123)
void CWENOFV::initializeGrid()
{
    const std::string backend = opt("BACKEND", "CUDA");
    if (backend != "CUDA")
        throw std::invalid_argument("BACKEND = " + backend + ": this build runs the CUDA backend only");
    m_testcase = (TESTCASETYPE)std::stoi(opt("TESTCASE", "0"));
    m_rkMeth = (RKMETHOD)std::stoi(opt("RKMETH", "2"));
    m_riemannFluxType = (RIEMANNFLUXTYPE)std::stoi(opt("RIEMANNFLUX", "0"));
    m_reconstructionType = (RECONSTRUCTIONTYPE)std::stoi(opt("RECONSTRUCTIONTYPE", "1"));
    equation->setEquationParameters(m_testcase);
    m_timeMoments = equation->outputTimes;
    const std::string tend = opt("ENDTIME", "");
    if (!tend.empty()) m_timeMoments = {0.0, std::stod(tend)};
    m_varNum = equation->getVarNum();
    m_scheme = (SCHEMETYPE)std::stoi(opt("SCHEME", "1"));
    m_pplimiter = std::stoi(opt("PPlimiter", "0")) != 0;
    m_cfl = std::stod(opt("CFL", "0.5"));
    m_ghostCellNum = 3;
    m_worldElemNumX = std::stoi(opt("ELEMNUMX", "100"));
    m_worldElemNumY = std::stoi(opt("ELEMNUMY", "100"));
    m_elemNumX = m_worldElemNumX;
    m_elemNumY = m_worldElemNumY;
    m_globalXL = equation->xL;
    m_globalXR = equation->xR;
    m_globalYL = equation->yL;
    m_globalYR = equation->yR;
    m_deltaX = (equation->xR - equation->xL) / m_worldElemNumX;
    m_deltaY = (equation->yR - equation->yL) / m_worldElemNumY;

    const std::string prec = opt("PRECISION", "FP64");
    if (prec == "FP64") m_precision = WENOFV_FP64;
    else if (prec == "FP64_STRICT") m_precision = WENOFV_FP64_STRICT;
    else if (prec == "FP32BULK" || prec == "FP32_BULK") m_precision = WENOFV_FP32_BULK;
    else throw std::invalid_argument("PRECISION = " + prec + ": expected FP64, FP64_STRICT or FP32BULK");
    m_refSlabs = std::stoi(opt("REFSLABS", "4"));
    m_device = std::stoi(opt("DEVICE", "0"));
    m_maxSteps = std::stoll(opt("MAXSTEPS", "0"));
    if (m_refSlabs < 0 || (m_refSlabs > 0 && m_worldElemNumX % m_refSlabs != 0))
        throw std::invalid_argument("ELEMNUMX must be divisible by REFSLABS (the reference's slab count)");
    m_Uh.assign((size_t)m_worldElemNumX * m_worldElemNumY * m_varNum, 0.0);
}

// initializeAve (src/WENOFV.cpp:232-279): the 4x4 Gauss-Legendre average of getU0 over
// every cell, with each cell's bounds computed as the reference's slab grid generator
// computes them (src/WENOFV.cpp:89-123), so the averages match it bit for bit.
void CWENOFV::initializeAve()
{
    const int slabs = m_refSlabs > 0 ? m_refSlabs : 1;
    const int perSlab = m_worldElemNumX / slabs;
    const int G = m_ghostCellNum;
    const double procYLeft = equation->yL + 0 * m_worldElemNumY * m_deltaY;
    const double ghostYLeft = procYLeft - m_deltaY * G;
    double U0[4];
    for (int i = 0; i < m_worldElemNumX; i++) {
        const int slab = i / perSlab, ei = i - slab * perSlab + G;
        const double procXLeft = equation->xL + slab * perSlab * m_deltaX;
        const double ghostXLeft = procXLeft - m_deltaX * G;
        const double xl = ghostXLeft + ei * m_deltaX, xr = ghostXLeft + (ei + 1) * m_deltaX;
        const double xc = (xl + xr) / 2, xd = xr - xl;
        for (int j = 0; j < m_worldElemNumY; j++) {
            const int ej = j + G;
            const double yl = ghostYLeft + ej * m_deltaY, yr = ghostYLeft + (ej + 1) * m_deltaY;
            const double yc = (yl + yr) / 2, yd = yr - yl;
            const double area = xd * yd;
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    const double gx = xc + 0.5 * xd * kGLegX[a], gy = yc + 0.5 * yd * kGLegX[b];
                    const double wx = 0.5 * xd * kGLegW[a], wy = 0.5 * yd * kGLegW[b];
                    equation->getU0(gx, gy, U0);
                    for (int r = 0; r < m_varNum; r++) acc[r] += U0[r] * wx * wy;
                }
            for (int r = 0; r < m_varNum; r++) Uh(i, j, r) = acc[r] / area;
        }
    }
}

wenofv_config CWENOFV::config() const
{
    wenofv_config c;
    wenofv_default_config(&c);
    c.nx = m_worldElemNumX;
    c.ny = m_worldElemNumY;
    c.xl = equation->xL;
    c.xr = equation->xR;
    c.yl = equation->yL;
    c.yr = equation->yR;
    c.bc = WENOFV_BC_PERIOD;
    c.rk_method = (int)m_rkMeth;
    c.cfl = m_cfl;
    c.scheme = (int)m_scheme;
    c.pp_limiter = m_pplimiter ? 1 : 0;
    c.riemann_flux = (int)m_riemannFluxType;
    c.reconstruction = (int)m_reconstructionType;
    c.ref_slabs = m_refSlabs;
    c.precision = m_precision;
    c.device = m_device;
    return c;
}

void CWENOFV::initializeSolver()
{
    initializeGrid();
    initializeAve();
    const wenofv_config c = config();
    const wenofv_eq_params p = equation->params();
    if (m_ctx) {
        wenofv_destroy(m_ctx);
        m_ctx = nullptr;
    }
    check(wenofv_create(&c, &p, &m_ctx), "wenofv_create");
    uploadUh();
    m_now = 0.0;
    m_stepCount = 0;
}

void CWENOFV::uploadUh() { check(wenofv_upload(m_ctx, m_Uh.data(), WENOFV_LAYOUT_REF_AOS), "wenofv_upload"); }
void CWENOFV::downloadUh() { check(wenofv_download(m_ctx, m_Uh.data(), WENOFV_LAYOUT_REF_AOS), "wenofv_download"); }

// calculateDeltaT (src/WENOFV.cpp:474-540) of the device state
double CWENOFV::calculateDeltaT(double now)
{
    (void)now;
    double dt = 0.0;
    check(wenofv_compute_dt(m_ctx, &dt), "calculateDeltaT");
    return dt;
}

// performTimeIntegration (src/WENOFV.cpp:541-566): one SSP-RK step of the device state
void CWENOFV::performTimeIntegration(double timestep)
{
    check(wenofv_step(m_ctx, timestep), "performTimeIntegration");
    m_stepCount++;
}

// assembleRHS (src/WENOFV.cpp:568-615) of the device state, into m_rhs
void CWENOFV::assembleRHS()
{
    m_rhs.assign(m_Uh.size(), 0.0);
    check(wenofv_rhs(m_ctx, m_rhs.data(), WENOFV_LAYOUT_REF_AOS), "assembleRHS");
}

// run (src/WENOFV.cpp:281-374): advance through the output moments; each interval is the
// reference's inner loop `while |now - t| > 1e-10 { dt = min(calculateDeltaT, t - now);
// performTimeIntegration(dt); now += dt; }`, executed on the device.  The .plt output of
// the reference is replaced by an optional binary dump of the final state (key OUTPUT).
void CWENOFV::run()
{
    const auto t0 = std::chrono::steady_clock::now();
    initializeSolver();
    const auto t1 = std::chrono::steady_clock::now();
    const bool hostLoop = opt("STEPMODE", "0") == "1";
    for (size_t k = 1; k < m_timeMoments.size(); k++) {
        const double targetTime = m_timeMoments[k];
        if (hostLoop) {
            // the reference's loop on the host, one C-ABI call per method (src/WENOFV.cpp:318-331)
            int64_t n = 0;
            while (std::abs(m_now - targetTime) > 1e-10 && (m_maxSteps <= 0 || n < m_maxSteps)) {
                const double remainingTime = targetTime - m_now;
                double timestep = calculateDeltaT(m_now);
                timestep = std::min(timestep, remainingTime);
                performTimeIntegration(timestep);
                m_now += timestep;
                n++;
            }
        } else {
            double tout = m_now;
            int64_t n = 0;
            check(wenofv_advance(m_ctx, m_now, targetTime, m_maxSteps, &tout, &n), "run");
            m_now = tout;
            m_stepCount += n;
        }
        downloadUh();
    }
    const auto t2 = std::chrono::steady_clock::now();
    const double solve = std::chrono::duration<double>(t2 - t1).count();
    const double init = std::chrono::duration<double>(t1 - t0).count();
    const double updates = (double)m_worldElemNumX * m_worldElemNumY * (m_rkMeth + 1) * m_stepCount;
    std::printf("{\"testcase\": \"%s\", \"grid\": [%d, %d], \"steps\": %lld, \"time\": %.17g, \"init_s\": %.6f, "
                "\"solve_s\": %.6f, \"cell_stage_updates_per_s\": %.6g}\n",
                TESTCASETYPE_STRINGS[m_testcase], m_worldElemNumX, m_worldElemNumY, (long long)m_stepCount, m_now, init,
                solve, solve > 0 ? updates / solve : 0.0);
    const std::string out = opt("OUTPUT", "");
    if (!out.empty()) {
        std::ofstream f(out, std::ios::binary);
        f.write(reinterpret_cast<const char *>(m_Uh.data()), (std::streamsize)(m_Uh.size() * sizeof(double)));
        if (!f) throw std::runtime_error("cannot write " + out);
    }
}
