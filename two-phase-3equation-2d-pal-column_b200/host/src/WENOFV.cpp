// WENOFV.cpp -- CWENOFV methods of the CUDA backend (the reference's src/WENOFV.cpp:16-566
// call structure; the per-cell work runs in libwenofv_b200).
#include "../include/WENOFV.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <limits>
#include <iomanip>
#include <iostream>
#include <sstream>
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
    if (m_writer.joinable()) m_writer.join();
    if (m_ctx) wenofv_destroy(m_ctx);
}

// joins the previous series writer and rethrows its error, if any
void CWENOFV::finishSeriesOutput()
{
    if (m_writer.joinable()) m_writer.join();
    if (m_writerError) {
        std::exception_ptr e = m_writerError;
        m_writerError = nullptr;
        std::rethrow_exception(e);
    }
}

// snapshot of the device state now (a device-side copy, then a read-back on the library's
// copy stream) and a worker thread that waits for it and appends the time series, so that
// the read-back and the file writing overlap the next piece of the device loop
void CWENOFV::startSeriesOutput(double now)
{
    finishSeriesOutput();
    m_snapshot.resize(m_Uh.size());
    check(wenofv_snapshot_begin(m_ctx, m_snapshot.data(), WENOFV_LAYOUT_REF_AOS), "wenofv_snapshot_begin");
    m_writer = std::thread([this, now] {
        try {
            check(wenofv_snapshot_wait(m_ctx), "wenofv_snapshot_wait");
            outputSpecialTestCasebyTime(now, m_snapshot.data());
        } catch (...) {
            m_writerError = std::current_exception();
        }
    });
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
    m_frame.clear();
    if (equation->boundaryCondition != NEUMANN2) return;
    // NEUMANN2 ("boundary from the initial data"): the same 4x4 average over the 4 cell layers
    // around the domain, on the uniform grid extended past its edges; held fixed by the library
    const int fw = m_worldElemNumX + 8, fh = m_worldElemNumY + 8;
    m_frame.assign((size_t)m_varNum * fw * fh, 0.0);
    for (int fj = 0; fj < fh; fj++)
        for (int fi = 0; fi < fw; fi++) {
            const int i = fi - 4, j = fj - 4;
            if (i >= 0 && i < m_worldElemNumX && j >= 0 && j < m_worldElemNumY) continue;
            const double xl = equation->xL + i * m_deltaX, xr = xl + m_deltaX;
            const double yl = equation->yL + j * m_deltaY, yr = yl + m_deltaY;
            const double xc = (xl + xr) / 2, xd = xr - xl, yc = (yl + yr) / 2, yd = yr - yl;
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    const double gx = xc + 0.5 * xd * kGLegX[a], gy = yc + 0.5 * yd * kGLegX[b];
                    const double wx = 0.5 * xd * kGLegW[a], wy = 0.5 * yd * kGLegW[b];
                    equation->getU0(gx, gy, U0);
                    for (int r = 0; r < m_varNum; r++) acc[r] += U0[r] * wx * wy;
                }
            for (int r = 0; r < m_varNum; r++) m_frame[((size_t)r * fh + fj) * fw + fi] = acc[r] / (xd * yd);
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
    c.bc = (int)equation->boundaryCondition; // BOUNDARYTYPE and WENOFV_BC_* share their numbers
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
    if (!m_frame.empty()) check(wenofv_set_frame(m_ctx, m_frame.data()), "wenofv_set_frame");
    uploadUh();
    m_now = 0.0;
    m_stepCount = 0;
}

namespace {
// getVolumeFrac / getPressure (include/Equations.hpp:84-124) of the host-side output
double volume_frac(const TwoPhaseEquation &e, const double *U)
{
    const double c1_2 = e.g_sound1 * e.g_sound1, c2_2 = e.g_sound2 * e.g_sound2;
    const double q = e.g_rho20 * c2_2 - e.g_rho10 * c1_2;
    const double qs = U[1] * c2_2 - U[0] * c1_2;
    const double r = ((q - qs) + std::sqrt((q - qs) * (q - qs) + 4.0 * U[0] * c1_2 * U[1] * c2_2)) / (2.0 * U[1] * c2_2);
    return r / (1.0 + r);
}
double pressure(const TwoPhaseEquation &e, const double *U, double z1)
{
    const double z2 = 1.0 - z1;
    const double pre1 = e.g_sound1 * e.g_sound1 * (U[0] / z1 - e.g_rho10);
    const double pre2 = e.g_sound2 * e.g_sound2 * (U[1] / z2 - e.g_rho20);
    return (z1 < z2) ? pre2 : pre1;
}
std::string num_str(double v)
{
    std::ostringstream o;
    o << v;
    return o.str();
}
} // namespace

// outputResults (src/WENOFV.cpp:2447-2523) at the initial, intermediate and final moments
void CWENOFV::outputResults(int count, double now, const std::string &specialCase)
{
    (void)count;
    if (m_outputDir.empty()) return;
    const bool exact = m_testcase == SMOOTH || m_testcase == VORTEX;
    const bool slice = opt("SLICEOUTPUT", "0") == "1";
    if (specialCase == "initial") {
        outputAve("initial");
        if (slice) outputSliceAve("initial");
        if (exact) outputAccuracy("initial", now);
        if (m_testcase == SHARP) outputUPoscillation("initial");
    } else if (specialCase == "final") {
        outputAve("final");
        if (slice) outputSliceAve("final");
        if (exact) outputAccuracy("final", now);
        if (m_testcase == SHARP) outputUPoscillation("final"); // outputSpecialTestCasebyCell (:3381-3391)
    } else if (specialCase == "intermediate") {
        outputAve(num_str(now) + "_intermediate");
        if (slice) outputSliceAve(num_str(now) + "_intermediate");
    }
}

// the per-cell theta record of the limiter's last call (getWorldTheta, m_worldTotalTheta),
// in the [i][j] order of m_Uh
std::vector<uint8_t> CWENOFV::thetaFlags() const
{
    std::vector<uint8_t> th((size_t)m_worldElemNumX * m_worldElemNumY, 0);
    check(wenofv_theta_flags(m_ctx, th.data(), WENOFV_LAYOUT_REF_AOS), "wenofv_theta_flags");
    return th;
}

// outputAve (src/WENOFV.cpp:2525-2601): cell centres, the variables of getVitalVarVal
// (include/Equations.hpp:1005-1043), the limiter's per-cell theta record (1 where the last
// limiter call scaled the cell: theta < 1 - 1e-8) and the Pr column.  The reference's Pr is
// m_totalPr, which every getFlux_* sets to zero (src/WENOFV.cpp:637, :746, :904, :1063,
// :1219) and nothing writes, so it is 0 here too.
void CWENOFV::outputAve(const std::string &prefix)
{
    const std::string filename = m_outputDir + "average_" + prefix + ".plt";
    std::ofstream f(filename);
    if (!f) throw std::runtime_error("cannot write " + filename);
    const std::vector<uint8_t> th = thetaFlags();
    f << "TITLE=FvSolution" << std::endl;
    f << "VARIABLES=X Y RHO1Z1 RHO2Z2 Z1 RHO1 RHO2 RHO U V PRE theta Pr " << std::endl;
    f << "ZONE T=TA, I=" << m_worldElemNumY << ", J=" << m_worldElemNumX << ", DATAPACKING = POINT" << std::endl;
    const int G = m_ghostCellNum;
    for (int i = 0; i < m_worldElemNumX; i++) {
        const double xl = equation->xL - G * m_deltaX + (i + G) * m_deltaX, xr = equation->xL - G * m_deltaX + (i + G + 1) * m_deltaX;
        for (int j = 0; j < m_worldElemNumY; j++) {
            const double yl = equation->yL - G * m_deltaY + (j + G) * m_deltaY, yr = equation->yL - G * m_deltaY + (j + G + 1) * m_deltaY;
            const double *U = &m_Uh[((size_t)i * m_worldElemNumY + j) * m_varNum];
            const double z1 = volume_frac(*equation, U), rho = U[0] + U[1];
            f << (xl + xr) / 2 << " " << (yl + yr) / 2 << " " << U[0] << " " << U[1] << " " << z1 << " " << U[0] / z1
              << " " << U[1] / (1.0 - z1) << " " << rho << " " << U[2] / rho << " " << U[3] / rho << " "
              << pressure(*equation, U, z1) << " " << (int)th[(size_t)i * m_worldElemNumY + j] << " " << 0 << " "
              << std::endl;
        }
    }
}

// outputSliceAve (src/WENOFV.cpp:2668-2737): the row j = 1 (the reference's ej = ghost + 1)
// in the columns of outputAve without Y.  The reference's outputResults never calls it; here
// the key SLICEOUTPUT = 1 writes slice_<prefix>.plt beside every average_<prefix>.plt.
void CWENOFV::outputSliceAve(const std::string &prefix)
{
    const std::string filename = m_outputDir + "slice_" + prefix + ".plt";
    std::ofstream f(filename);
    if (!f) throw std::runtime_error("cannot write " + filename);
    const std::vector<uint8_t> th = thetaFlags();
    f << "TITLE=FvSolution_Slice" << std::endl;
    f << "VARIABLES=X RHO1Z1 RHO2Z2 Z1 RHO1 RHO2 RHO U V PRE theta Pr " << std::endl;
    f << "ZONE T=TA, I=" << m_worldElemNumX << ", DATAPACKING = POINT" << std::endl;
    const int G = m_ghostCellNum, j = std::min(1, m_worldElemNumY - 1);
    for (int i = 0; i < m_worldElemNumX; i++) {
        const double xl = equation->xL - G * m_deltaX + (i + G) * m_deltaX, xr = equation->xL - G * m_deltaX + (i + G + 1) * m_deltaX;
        const double *U = &m_Uh[((size_t)i * m_worldElemNumY + j) * m_varNum];
        const double z1 = volume_frac(*equation, U), rho = U[0] + U[1];
        f << (xl + xr) / 2 << " " << U[0] << " " << U[1] << " " << z1 << " " << U[0] / z1 << " " << U[1] / (1.0 - z1)
          << " " << rho << " " << U[2] / rho << " " << U[3] / rho << " " << pressure(*equation, U, z1) << " "
          << (int)th[(size_t)i * m_worldElemNumY + j] << " " << 0 << " " << std::endl;
    }
}

// outputUPoscillation (src/WENOFV.cpp:2739-2805): for the SHARP square advected at (1, 1), each
// cell's deviation from that uniform flow: |(u-1, v-1)| / c1, |p| / (rho10 c1^2), |u-1| / c1
// and |v-1| / c1, in the layout of outputAve
void CWENOFV::outputUPoscillation(const std::string &prefix)
{
    const std::string filename = m_outputDir + "UPoscillation_" + prefix + ".plt";
    std::ofstream f(filename);
    if (!f) throw std::runtime_error("cannot write " + filename);
    f << "TITLE=FvSolution" << std::endl;
    f << "VARIABLES=X Y Speed_oscillation P_oscillation U_oscillation V_oscillation " << std::endl;
    f << "ZONE T=TA, I=" << m_worldElemNumY << ", J=" << m_worldElemNumX << ", DATAPACKING = POINT" << std::endl;
    const int G = m_ghostCellNum;
    const double c1 = equation->g_sound1;
    for (int i = 0; i < m_worldElemNumX; i++) {
        const double xl = equation->xL - G * m_deltaX + (i + G) * m_deltaX, xr = equation->xL - G * m_deltaX + (i + G + 1) * m_deltaX;
        for (int j = 0; j < m_worldElemNumY; j++) {
            const double yl = equation->yL - G * m_deltaY + (j + G) * m_deltaY, yr = equation->yL - G * m_deltaY + (j + G + 1) * m_deltaY;
            const double *U = &m_Uh[((size_t)i * m_worldElemNumY + j) * m_varNum];
            const double rho = U[0] + U[1], u = U[2] / rho, v = U[3] / rho;
            const double p = pressure(*equation, U, volume_frac(*equation, U));
            f << (xl + xr) / 2 << " " << (yl + yr) / 2 << " " << std::fabs(std::sqrt(std::pow(u - 1, 2) + std::pow(v - 1, 2))) / c1
              << " " << std::fabs(p) / equation->g_rho10 / std::pow(c1, 2) << " " << std::fabs(u - 1) / c1 << " "
              << std::fabs(v - 1) / c1 << " " << std::endl;
        }
    }
}

// outputSpecialTestCasebyTime (src/WENOFV.cpp:3363-3379): DAMBREAK's pressure probes, RTI's
// symmetry error, and for SHARP the interface thickness and outputUPoscillationByTime
// (:2865-2941), which appends the maxima over the cells of the pressure, speed, u and v deviations
// to oscillationByTime_<nx>.plt.  The reference's header names the columns Speed, P, U, V
// but writes them in the order P, Speed, U, V, and takes the signed u and v deviations (maxima
// from 0); both are kept, so that files from the two programs read alike.
void CWENOFV::outputSpecialTestCasebyTime(double now, const double *Us)
{
    if (m_testcase == DAMBREAK) {
        outputPressureByTime(now, Us);
        return;
    }
    if (m_testcase == RTI) {
        outputSymmetryErr(now, Us);
        return;
    }
    if (m_testcase != SHARP) return;
    outputThicknessByTime(now, Us);
    const std::string filename = m_outputDir + "oscillationByTime_" + std::to_string(m_worldElemNumX) + ".plt";
    const bool exists = std::filesystem::exists(filename);
    std::ofstream f(filename, std::ios::app);
    if (!f) throw std::runtime_error("cannot write " + filename);
    if (!exists)
        f << "TITLE=FvSolution" << std::endl
          << "VARIABLES=Time Speed_oscillation P_oscillation U_oscillation V_oscillation " << std::endl
          << "ZONE T=TA" << std::endl;
    const double c1 = equation->g_sound1;
    double pmax = 0, smax = 0, umax = 0, vmax = 0;
    for (int i = 0; i < m_worldElemNumX; i++)
        for (int j = 0; j < m_worldElemNumY; j++) {
            const double *U = &Us[((size_t)i * m_worldElemNumY + j) * m_varNum];
            const double rho = U[0] + U[1], u = U[2] / rho, v = U[3] / rho;
            pmax = std::max(pmax, std::fabs(pressure(*equation, U, volume_frac(*equation, U))) / equation->g_rho10 / std::pow(c1, 2));
            smax = std::max(smax, std::sqrt(std::pow(u - 1, 2) + std::pow(v - 1, 2)) / c1);
            umax = std::max(umax, (u - 1) / c1);
            vmax = std::max(vmax, (v - 1) / c1);
        }
    f << now << " " << pmax << " " << smax << " " << umax << " " << vmax << std::endl;
}

// outputThincknessByTime (src/WENOFV.cpp:3049-3108) for SHARP: 1 / the largest jump of z1
// between neighbouring cells in x or y (the right and upper neighbours), an interface
// thickness in cells, appended to thincknessByTime.plt under the reference's file and column
// names.  The last column and row compare with the periodic wrap, a choice of this mirror:
// the reference gathers the state without filling the gathered array's ghost cells
// (getWorldUh, src/WENOFV.cpp:2059-2093), so its last column and row compare with unfilled
// entries.  On SHARP the two agree in practice, because z1 there is the background's ~1e-8
// on both sides of the periodic seam.
void CWENOFV::outputThicknessByTime(double now, const double *Us)
{
    const std::string filename = m_outputDir + "thincknessByTime.plt";
    const bool exists = std::filesystem::exists(filename);
    std::ofstream f(filename, std::ios::app);
    if (!f) throw std::runtime_error("cannot write " + filename);
    if (!exists) f << "TITLE=FvSolution" << std::endl << "VARIABLES=time thinckness\n" << std::endl << "ZONE T=TA" << std::endl;
    const int nx = m_worldElemNumX, ny = m_worldElemNumY;
    auto z1 = [&](int i, int j) { return volume_frac(*equation, &Us[((size_t)(i % nx) * ny + (j % ny)) * m_varNum]); };
    double maxDiff = 0;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            const double z = z1(i, j);
            maxDiff = std::max(maxDiff, std::max(std::fabs(z - z1(i + 1, j)), std::fabs(z - z1(i, j + 1))));
        }
    f << now << " " << 1.0 / maxDiff << std::endl;
}

// outputSymmetryErr (src/WENOFV.cpp:3109-3151) for RTI: the largest difference of z1 between
// each cell of the left half and its mirror image across x = (xL + xR) / 2, appended to
// symmetry_err.plt (no header, as the reference writes it; its running maximum starts
// uninitialised there and at 0 here)
void CWENOFV::outputSymmetryErr(double now, const double *Us)
{
    std::ofstream f(m_outputDir + "symmetry_err.plt", std::ios::app);
    if (!f) throw std::runtime_error("cannot write " + m_outputDir + "symmetry_err.plt");
    const int nx = m_worldElemNumX, ny = m_worldElemNumY;
    double maxErr = 0;
    for (int i = 0; i < nx / 2; i++)
        for (int j = 0; j < ny; j++) {
            const double a = volume_frac(*equation, &Us[((size_t)i * ny + j) * m_varNum]);
            const double b = volume_frac(*equation, &Us[((size_t)(nx - 1 - i) * ny + j) * m_varNum]);
            maxErr = std::max(maxErr, std::fabs(a - b));
        }
    f << now << " " << maxErr << std::endl;
}

// outputPressureByTime (src/WENOFV.cpp:2942-3048) for DAMBREAK: the pressure on the left wall
// at y = 3, 15, 30 and 80 mm over rho10 g H0 (g = 9.81, H0 = 0.3), against t sqrt(g / H0).  For
// each height, the cell pressures of a 5x5 block around (first column, row floor(y / dy)) are
// reconstructed by WENO-JS across x to the wall face (Gauss-Lobatto point 0), then across y
// to the 4 points of the row's cell; the point nearest y is taken.  Cells beyond the domain
// are the mirror images that the library's NEUMANN walls use (the pressure keeps its sign).
// The reconstructions run through the library's WENO probe, so they are the solver's own.
void CWENOFV::outputPressureByTime(double now, const double *Us)
{
    const std::string filename = m_outputDir + "pressureByTime.plt";
    const bool exists = std::filesystem::exists(filename);
    std::ofstream f(filename, std::ios::app);
    if (!f) throw std::runtime_error("cannot write " + filename);
    if (!exists) f << "TITLE=FvSolution" << std::endl << "VARIABLES=Time P_y3mm P_y15mm P_y30mm P_y80mm\n" << std::endl << "ZONE T=TA" << std::endl;
    auto mirror = [](int k, int n) {
        for (int it = 0; it < 64 && (k < 0 || k >= n); it++) k = k < 0 ? -1 - k : 2 * n - 1 - k;
        return std::min(std::max(k, 0), n - 1);
    };
    const double heights_mm[4] = {3.0, 15.0, 30.0, 80.0};
    const double gl[4] = {-1.0, -std::sqrt(0.2), std::sqrt(0.2), 1.0}; // Gauss-Lobatto points on [-1, 1]
    std::vector<double> xst(4 * 25), xout(4 * 20), yst(4 * 5), yout(4 * 4);
    int rows[4];
    for (int h = 0; h < 4; h++) {
        const double y_m = heights_mm[h] / 1000.0;
        rows[h] = (int)std::floor(y_m / m_deltaY);
        for (int b = 0; b < 5; b++)     // row offset b - 2: one x-stencil per row
            for (int a = 0; a < 5; a++) { // column offset a - 2 from the first column
                const int i = mirror(a - 2, m_worldElemNumX), j = mirror(rows[h] + b - 2, m_worldElemNumY);
                const double *U = &Us[((size_t)i * m_worldElemNumY + j) * m_varNum];
                xst[(h * 5 + b) * 5 + a] = pressure(*equation, U, volume_frac(*equation, U)) / equation->g_rho10 / 9.81 / 0.3;
            }
    }
    check(wenofv_probe_weno(0, WENOFV_FP64_STRICT, xst.data(), 20, xout.data(), m_device), "wenofv_probe_weno");
    for (int h = 0; h < 4; h++)
        for (int b = 0; b < 5; b++) yst[h * 5 + b] = xout[(h * 5 + b) * 4 + 0];
    check(wenofv_probe_weno(0, WENOFV_FP64_STRICT, yst.data(), 4, yout.data(), m_device), "wenofv_probe_weno");
    f << now * std::sqrt(9.81 / 0.3);
    for (int h = 0; h < 4; h++) {
        const double y_m = heights_mm[h] / 1000.0;
        const double yc = equation->yL + (rows[h] + 0.5) * m_deltaY;
        int best = 0;
        double diff = std::numeric_limits<double>::max();
        for (int k = 0; k < 4; k++) {
            const double d = std::fabs(yc + 0.5 * m_deltaY * gl[k] - y_m);
            if (d < diff) { diff = d; best = k; }
        }
        f << " " << yout[h * 4 + best];
    }
    f << std::endl;
}

// outputAccuracy (src/WENOFV.cpp:3152-3251): z1 against the 4x4 Gauss-Legendre average of
// the initial volume fraction translated by (u0, v0) t
void CWENOFV::outputAccuracy(const std::string &prefix, double now)
{
    const int G = m_ghostCellNum;
    double e1 = 0.0, e2 = 0.0, einf = 0.0;
    for (int i = 0; i < m_worldElemNumX; i++) {
        const double xl = equation->xL - G * m_deltaX + (i + G) * m_deltaX, xr = equation->xL - G * m_deltaX + (i + G + 1) * m_deltaX;
        const double xc = (xl + xr) / 2;
        for (int j = 0; j < m_worldElemNumY; j++) {
            const double yl = equation->yL - G * m_deltaY + (j + G) * m_deltaY, yr = equation->yL - G * m_deltaY + (j + G + 1) * m_deltaY;
            const double yc = (yl + yr) / 2;
            double ex = 0.0;
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    const double gx = xc + 0.5 * m_deltaX * kGLegX[a], gy = yc + 0.5 * m_deltaY * kGLegX[b];
                    const double wx = 0.5 * m_deltaX * kGLegW[a], wy = 0.5 * m_deltaY * kGLegW[b];
                    ex += equation->z1_0(gx - equation->g_u0 * now, gy - equation->g_v0 * now) * wx * wy / m_deltaX / m_deltaY;
                }
            const double err = std::fabs(ex - volume_frac(*equation, &m_Uh[((size_t)i * m_worldElemNumY + j) * m_varNum]));
            e1 += err;
            e2 += std::pow(err, 2);
            if (err > einf) einf = err;
        }
    }
    e1 = e1 / m_worldElemNumX / m_worldElemNumY;
    e2 = std::sqrt(e2 / m_worldElemNumX / m_worldElemNumY);
    const std::string filename = m_outputDir + "accuracy_" + prefix + ".csv";
    const bool exists = std::filesystem::exists(filename);
    std::ofstream f(filename, exists ? std::ios::app : std::ios::out);
    if (!f) throw std::runtime_error("cannot write " + filename);
    if (!exists) f << "Cell Number, Linf-norm, L1-norm, L2-norm" << std::endl;
    f << m_worldElemNumX << ", " << std::setprecision(15) << std::setw(20) << std::scientific << einf << ", "
      << std::setw(20) << e1 << ", " << std::setw(20) << e2 << std::endl;
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
    m_outputDir = opt("OUTPUTDIR", "");
    if (!m_outputDir.empty()) {
        if (m_outputDir.back() != '/') m_outputDir += '/';
        std::filesystem::create_directories(m_outputDir);
    }
    outputResults(0, m_now, "initial");
    const auto t1 = std::chrono::steady_clock::now();
    const bool hostLoop = opt("STEPMODE", "0") == "1";
    const bool byTime = !m_outputDir.empty() && (m_testcase == SHARP || m_testcase == DAMBREAK || m_testcase == RTI);
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
                if (byTime && (m_stepCount == 1 || m_stepCount % 200 == 0)) {
                    downloadUh();
                    outputSpecialTestCasebyTime(m_now, m_Uh.data());
                }
            }
        } else if (byTime) {
            // the device loop in pieces that end at the steps where the reference writes its
            // time series (step 1 and every 200th, src/WENOFV.cpp:2486-2497)
            int64_t done = 0;
            while (std::abs(m_now - targetTime) > 1e-10 && (m_maxSteps <= 0 || done < m_maxSteps)) {
                int64_t piece = m_stepCount < 1 ? 1 : 200 - m_stepCount % 200;
                if (m_maxSteps > 0) piece = std::min<int64_t>(piece, m_maxSteps - done);
                double tout = m_now;
                int64_t n = 0;
                check(wenofv_advance(m_ctx, m_now, targetTime, piece, &tout, &n), "run");
                m_now = tout;
                m_stepCount += n;
                done += n;
                if (n == 0) break;
                if (m_stepCount == 1 || m_stepCount % 200 == 0) startSeriesOutput(m_now);
            }
        } else {
            double tout = m_now;
            int64_t n = 0;
            check(wenofv_advance(m_ctx, m_now, targetTime, m_maxSteps, &tout, &n), "run");
            m_now = tout;
            m_stepCount += n;
        }
        finishSeriesOutput();
        downloadUh();
        outputResults((int)m_stepCount, m_now, "intermediate");
    }
    const auto t2 = std::chrono::steady_clock::now();
    outputResults((int)m_stepCount, m_now, "final");
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
