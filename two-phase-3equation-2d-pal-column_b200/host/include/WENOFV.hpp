// WENOFV.hpp -- CWENOFV with the CUDA backend: the reference's solver class
// (include/WENOFV.hpp:87-257) with its option keys, enums, public members and stepping
// methods, whose work runs in libwenofv_b200 (include/wenofv.h) on one GPU.
//
// What stays as in the reference: construction from (TwoPhaseEquation*, option map), the
// settings.cfg keys TESTCASE ELEMNUMX ELEMNUMY RKMETH CFL SCHEME PPlimiter RIEMANNFLUX
// RECONSTRUCTIONTYPE, initializeSolver / initializeAve / calculateDeltaT /
// performTimeIntegration / assembleRHS / run, and the members m_worldElemNumX/Y, m_cfl,
// m_deltaX/Y, m_varNum, m_ghostCellNum, m_gpNum, m_pplimiter, m_timeMoments, m_testcase,
// m_scheme, m_rkMeth, m_riemannFluxType, m_reconstructionType.
//
// What changes:
//  * the whole domain lives on one GPU; there is no MPI decomposition.  The grid metric
//    can still carry the reference's 4-slab rounding (key REFSLABS, default 4) so that
//    PRECISION = FP64_STRICT reproduces the reference's cell averages bit for bit;
//  * m_Uh / m_rhs are host copies of the interior cell averages in the reference's
//    m_Uh[ei][ej].vector[r] order, [i][j][r] (ghost cells are an index map on the GPU);
//    m_Uh is refreshed from the device by downloadUh() and at each output time of run();
//  * errors throw std::runtime_error with the library's status text instead of printing,
//    waiting on stdin and exiting.
// Added keys: BACKEND (CUDA, the only backend), PRECISION (FP64 | FP64_STRICT | FP32BULK),
// REFSLABS, DEVICE, ENDTIME (replaces the case's last output time), MAXSTEPS (bound on
// the steps of each output interval, 0 = none), OUTPUT (file for the final state, FP64 [i][j][r]),
// OUTPUTDIR (directory for the reference's .plt / .csv output; none by default),
// STEPMODE (1: run's time loop on the host through calculateDeltaT / performTimeIntegration,
// as the reference loops; 0, the default: the loop on the device).
#pragma once
#include <cstdint>
#include <exception>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "Equations.hpp"

enum RKMETHOD { RK1 = 0, RK2 = 1, RK3 = 2 };
enum SCHEMETYPE { WENO = 0, WENOZ = 1, WENOEXP = 2 };
enum RECONSTRUCTIONTYPE {
    CONVERVATIVE = 0,
    CHARACTERISTIC = 1,
    PRIMITIVE = 2,
    PRIMITIVE2 = 3,
    PRIMITIVE3 = 4,
    ThincOnlyForZ1 = 5,
};

class CWENOFV
{
public:
    CWENOFV(TwoPhaseEquation *equation, std::map<std::string, std::string> option);
    ~CWENOFV();
    CWENOFV(const CWENOFV &) = delete;
    CWENOFV &operator=(const CWENOFV &) = delete;

    TwoPhaseEquation *equation;
    std::map<std::string, std::string> option;

    int m_worldElemNumX = 0, m_worldElemNumY = 0;
    int m_elemNumX = 0, m_elemNumY = 0;
    int m_ghostCellNum = 3;
    int m_varNum = 4;
    int m_gpNum = 4;
    double m_globalXL = 0, m_globalXR = 1, m_globalYL = 0, m_globalYR = 1;
    double m_cfl = 0.5;
    double m_deltaX = 0, m_deltaY = 0;
    bool m_pplimiter = false;
    std::vector<double> m_timeMoments;

    TESTCASETYPE m_testcase = SMOOTH;
    SCHEMETYPE m_scheme = WENOZ;
    RKMETHOD m_rkMeth = RK3;
    RIEMANNFLUXTYPE m_riemannFluxType = LLF;
    RECONSTRUCTIONTYPE m_reconstructionType = CHARACTERISTIC;

    std::vector<double> m_Uh;  // interior cell averages, [i][j][r]
    std::vector<double> m_frame; // NEUMANN2: ghost averages, SoA [r][ny+8][nx+8] (wenofv_set_frame)
    std::vector<double> m_rhs; // the last assembleRHS result, [i][j][r]

    int m_precision = WENOFV_FP64;
    int m_refSlabs = 4;
    int m_device = 0;
    int64_t m_maxSteps = 0;
    int64_t m_stepCount = 0;
    double m_now = 0.0;

    void initializeSolver();            // options, grid, initial averages, device state
    void initializeGrid();              // options and grid only (no GPU)
    void initializeAve();               // cell averages of getU0 by 4x4 Gauss-Legendre
    double calculateDeltaT(double now); // the CFL time step of the device state
    void performTimeIntegration(double timestep);
    void assembleRHS();
    void run();

    void downloadUh();
    void uploadUh();

    // the reference's output files (src/WENOFV.cpp:2447-2601, :3152-3251), written when the
    // key OUTPUTDIR names a directory: average_<prefix>.plt (Tecplot point data of the
    // cell averages and the derived variables) and, for SMOOTH and VORTEX,
    // accuracy_<prefix>.csv (L_inf, L1, L2 of z1 against the translated initial data)
    void outputResults(int count, double now, const std::string &specialCase);
    void outputAve(const std::string &prefix);      // with the limiter's theta record and Pr (= 0)
    void outputSliceAve(const std::string &prefix); // the row j = 1 (key SLICEOUTPUT = 1)
    void outputAccuracy(const std::string &prefix, double now);
    void outputUPoscillation(const std::string &prefix); // SHARP's velocity/pressure deviation
    // the time series of SHARP, DAMBREAK and RTI from a state Us ([i][j][r], m_Uh or a snapshot)
    void outputSpecialTestCasebyTime(double now, const double *Us);
    void outputPressureByTime(double now, const double *Us);  // DAMBREAK's wall pressure probes
    void outputThicknessByTime(double now, const double *Us); // SHARP's interface thickness
    void outputSymmetryErr(double now, const double *Us);     // RTI's left-right symmetry error
    std::vector<uint8_t> thetaFlags() const;                  // the limiter's per-cell record, [i][j]
    std::string m_outputDir;
    double &Uh(int i, int j, int r) { return m_Uh[((size_t)i * m_worldElemNumY + j) * m_varNum + r]; }
    wenofv_config config() const;

private:
    wenofv_ctx *m_ctx = nullptr;
    // asynchronous time-series output of the device loop: a snapshot of the state is read back
    // on the library's copy stream and written by a worker thread while the next steps run
    std::thread m_writer;
    std::exception_ptr m_writerError;
    std::vector<double> m_snapshot;
    void startSeriesOutput(double now);
    void finishSeriesOutput();
    std::string opt(const std::string &key, const std::string &dflt) const;
    void check(int rc, const char *what) const;
};
