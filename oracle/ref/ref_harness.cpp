// ref_harness.cpp -- drives the UNMODIFIED reference solver (src/WENOFV.cpp) through its
// public CWENOFV members, replacing src/main.cpp so that state can be injected and dumped
// as binary FP64.  TEST INFRASTRUCTURE: the parity oracle and the CPU baseline.
//
// The reference hard-codes a 4-rank x-slab decomposition (src/WENOFV.cpp:24, :34-38); the
// 4 ranks run as threads over the in-process MPI shim (mpi.h).  The stepping loop is the
// inner loop of CWENOFV::run (src/WENOFV.cpp:323-332) without output.
//
// usage: wenofv_ref [--testcase N] [--nx N] [--ny N] [--rk N] [--cfl X] [--scheme N]
//                   [--limiter N] [--flux N] [--recon N]
//                   [--rho10 X --rho20 X --sound1 X --sound2 X]   equation overrides
//                   [--u0 FILE]        initial averages, SoA [v][j][i] FP64 (else the test case IC)
//                   [--dump-u0 FILE]   the initial averages actually used
//                   [--steps N | --tend T] [--warmup N]   (warm-up steps run untimed first)
//                   [--rhs FILE]       one assembleRHS of the initial state, SoA FP64
//                   [--faces FILE]     face states after that assembleRHS [cell][B,T,L,R][v][gp]
//                   [--out FILE] [--dts FILE] [--time]
//                   [--output-ave DIR] after the steps, the reference's own outputAve("final") and
//                                      outputSliceAve("final") into DIR (average_final.plt,
//                                      slice_final.plt), to compare the host mirror's files with
//                   [--source-case N]  after initialisation, the test case that assembleSourceTerm
//                                      sees (DAMBREAK/RTI: g = 9.81, STANDING_WAVE: 2 pi), so that
//                                      its gravity runs on a periodic case's grid and boundaries
//                                      (the walls of those cases are not implemented)
#include <mpi.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <map>
#include <string>
#include <thread>
#include <unistd.h>
#include <vector>

#include "../include/Equations.hpp"
#include "../include/ReadConfig.hpp"
#include "../include/WENOFV.hpp"

namespace {

struct Args {
    std::map<std::string, std::string> opt;
    double rho10 = -1, rho20 = -1, sound1 = -1, sound2 = -1;
    std::string u0, dump_u0, rhs, faces, out, dts, output_ave;
    long steps = -1, warmup = 0;
    double tend = -1;
    bool time = false;
    int source_case = -1;
};

struct Shared {
    int nx = 0, ny = 0;
    std::vector<double> U0, U, rhs, faces, dts;
    double seconds = 0;
    long nsteps = 0;
    double t_final = 0;
};

bool read_file(const std::string &path, std::vector<double> &v, size_t n)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    v.resize(n);
    const size_t got = std::fread(v.data(), sizeof(double), n, f);
    std::fclose(f);
    return got == n;
}

void write_file(const std::string &path, const std::vector<double> &v)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) { std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(2); }
    std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
}

void rank_main(int rank, const Args &a, Shared &sh, const std::vector<double> &u0in)
{
    wenofv_shim_set_rank(rank);
    TwoPhaseEquation *equation = new TwoPhaseEquation();
    CWENOFV solver(equation, a.opt);
    solver.initializeSolver();
    if (a.rho10 > 0) equation->g_rho10 = a.rho10;
    if (a.rho20 > 0) equation->g_rho20 = a.rho20;
    if (a.sound1 > 0) equation->g_sound1 = a.sound1;
    if (a.sound2 > 0) equation->g_sound2 = a.sound2;
    if (a.source_case >= 0) solver.m_testcase = (TESTCASETYPE)a.source_case;

    const int nx = sh.nx, ny = sh.ny, nv = solver.m_varNum;
    const int x0 = solver.m_procIndexX * solver.m_elemNumX;
    auto idx = [&](int v, int j, int g) { return (size_t)v * nx * ny + (size_t)j * nx + g; };

    if (!u0in.empty()) {
        for (int ei = solver.m_startElemX; ei != solver.m_endElemX; ++ei)
            for (int ej = solver.m_startElemY; ej != solver.m_endElemY; ++ej)
                for (int v = 0; v < nv; ++v)
                    solver.m_Uh[ei][ej].vector[v] = u0in[idx(v, ej - solver.m_startElemY, x0 + ei - solver.m_startElemX)];
    }
    for (int ei = solver.m_startElemX; ei != solver.m_endElemX; ++ei)
        for (int ej = solver.m_startElemY; ej != solver.m_endElemY; ++ej)
            for (int v = 0; v < nv; ++v)
                sh.U0[idx(v, ej - solver.m_startElemY, x0 + ei - solver.m_startElemX)] = solver.m_Uh[ei][ej].vector[v];
    solver.exchangeGhostCellsValue();

    if (!a.rhs.empty() || !a.faces.empty()) {
        solver.assembleRHS();
        for (int ei = solver.m_startElemX; ei != solver.m_endElemX; ++ei)
            for (int ej = solver.m_startElemY; ej != solver.m_endElemY; ++ej) {
                const int g = x0 + ei - solver.m_startElemX, j = ej - solver.m_startElemY;
                for (int v = 0; v < nv; ++v) sh.rhs[idx(v, j, g)] = solver.m_rhs[ei][ej].vector[v];
                double *fc = &sh.faces[((size_t)j * nx + g) * 16 * nv];
                const CgridFlux &gf = solver.m_gridFlux[ei][ej];
                for (int v = 0; v < nv; ++v)
                    for (int gp = 0; gp < 4; ++gp) {
                        fc[0 * 4 * nv + v * 4 + gp] = gf.bottomFlux[v][gp];
                        fc[1 * 4 * nv + v * 4 + gp] = gf.topFlux[v][gp];
                        fc[2 * 4 * nv + v * 4 + gp] = gf.leftFlux[v][gp];
                        fc[3 * 4 * nv + v * 4 + gp] = gf.rightFlux[v][gp];
                    }
            }
    }

    // untimed warm-up steps (the state they produce is the timed steps' input)
    for (long k = 0; k < a.warmup; k++) solver.performTimeIntegration(solver.calculateDeltaT(0.0));
    MPI_Barrier(MPI_COMM_WORLD);
    const auto t0 = std::chrono::steady_clock::now();
    double now = 0;
    long count = 0;
    const bool by_time = a.tend > 0;
    while (by_time ? std::abs(now - a.tend) > 1e-10 : count < a.steps) {
        double timestep = solver.calculateDeltaT(now);
        if (by_time) timestep = std::min(timestep, a.tend - now);
        solver.performTimeIntegration(timestep);
        if (rank == 0) sh.dts.push_back(timestep);
        now += timestep;
        count++;
    }
    MPI_Barrier(MPI_COMM_WORLD);
    const auto t1 = std::chrono::steady_clock::now();
    if (rank == 0) {
        sh.seconds = std::chrono::duration<double>(t1 - t0).count();
        sh.nsteps = count;
        sh.t_final = now;
    }
    for (int ei = solver.m_startElemX; ei != solver.m_endElemX; ++ei)
        for (int ej = solver.m_startElemY; ej != solver.m_endElemY; ++ej)
            for (int v = 0; v < nv; ++v)
                sh.U[idx(v, ej - solver.m_startElemY, x0 + ei - solver.m_startElemX)] = solver.m_Uh[ei][ej].vector[v];
    if (!a.output_ave.empty()) { // every rank takes part in the gathers; rank 0 writes
        solver.m_outputDir = a.output_ave + "/";
        solver.outputAve("final");
        solver.outputSliceAve("final");
    }
}

} // namespace

int main(int argc, char **argv)
{
    Args a;
    a.opt = {{"TESTCASE", "0"}, {"ELEMNUMX", "100"}, {"ELEMNUMY", "100"}, {"RKMETH", "2"},
             {"CFL", "0.5"},    {"SCHEME", "1"},     {"PPlimiter", "0"},  {"RIEMANNFLUX", "0"},
             {"RECONSTRUCTIONTYPE", "1"}};
    const std::map<std::string, std::string> keys = {
        {"--testcase", "TESTCASE"}, {"--nx", "ELEMNUMX"},  {"--ny", "ELEMNUMY"},
        {"--rk", "RKMETH"},         {"--cfl", "CFL"},      {"--scheme", "SCHEME"},
        {"--limiter", "PPlimiter"}, {"--flux", "RIEMANNFLUX"}, {"--recon", "RECONSTRUCTIONTYPE"}};
    for (int k = 1; k < argc; k++) {
        const std::string s = argv[k];
        const char *val = k + 1 < argc ? argv[k + 1] : "";
        if (keys.count(s)) { a.opt[keys.at(s)] = val; k++; }
        else if (s == "--rho10") { a.rho10 = std::atof(val); k++; }
        else if (s == "--rho20") { a.rho20 = std::atof(val); k++; }
        else if (s == "--sound1") { a.sound1 = std::atof(val); k++; }
        else if (s == "--sound2") { a.sound2 = std::atof(val); k++; }
        else if (s == "--u0") { a.u0 = val; k++; }
        else if (s == "--dump-u0") { a.dump_u0 = val; k++; }
        else if (s == "--rhs") { a.rhs = val; k++; }
        else if (s == "--faces") { a.faces = val; k++; }
        else if (s == "--out") { a.out = val; k++; }
        else if (s == "--dts") { a.dts = val; k++; }
        else if (s == "--steps") { a.steps = std::atol(val); k++; }
        else if (s == "--warmup") { a.warmup = std::atol(val); k++; }
        else if (s == "--tend") { a.tend = std::atof(val); k++; }
        else if (s == "--time") { a.time = true; }
        else if (s == "--source-case") { a.source_case = std::atoi(val); k++; }
        else if (s == "--output-ave") { a.output_ave = val; k++; }
        else { std::fprintf(stderr, "unknown argument %s\n", s.c_str()); return 2; }
    }
    if (a.steps < 0 && a.tend <= 0) a.steps = 0;

    // absolute paths before leaving the caller's directory
    auto absp = [](std::string &p) { if (!p.empty()) p = std::filesystem::absolute(p).string(); };
    absp(a.u0); absp(a.dump_u0); absp(a.rhs); absp(a.faces); absp(a.out); absp(a.dts); absp(a.output_ave);

    Shared sh;
    sh.nx = std::atoi(a.opt["ELEMNUMX"].c_str());
    sh.ny = std::atoi(a.opt["ELEMNUMY"].c_str());
    const size_t n = (size_t)4 * sh.nx * sh.ny;
    std::vector<double> u0in;
    if (!a.u0.empty() && !read_file(a.u0, u0in, n)) {
        std::fprintf(stderr, "cannot read %zu doubles from %s\n", n, a.u0.c_str());
        return 2;
    }
    sh.U0.assign(n, 0.0);
    sh.U.assign(n, 0.0);
    sh.rhs.assign(n, 0.0);
    sh.faces.assign(n * 16, 0.0);

    // the solver writes ./output/<timestamp>... and a source backup into the working
    // directory (src/WENOFV.cpp:100-105, :3392); keep that in a scratch directory.
    char tmpl[] = "/tmp/wenofv_ref_XXXXXX";
    const char *scratch = mkdtemp(tmpl);
    const std::string cwd = std::filesystem::current_path().string();
    if (scratch) std::filesystem::current_path(scratch);
    // the reference blocks on std::cin.get() in its error paths; make that return
    if (!std::freopen("/dev/null", "r", stdin)) return 2;
    fflush(stdout);
    const int saved_stdout = dup(1);
    if (!std::freopen("/dev/null", "w", stdout)) return 2;

    const int P = 4; // src/WENOFV.cpp:24
    wenofv_shim_set_size(P);
    std::vector<std::thread> th;
    for (int r = 0; r < P; r++) th.emplace_back(rank_main, r, std::cref(a), std::ref(sh), std::cref(u0in));
    for (auto &t : th) t.join();

    fflush(stdout);
    dup2(saved_stdout, 1);
    std::filesystem::current_path(cwd);
    if (scratch) std::filesystem::remove_all(scratch);

    if (!a.dump_u0.empty()) write_file(a.dump_u0, sh.U0);
    if (!a.out.empty()) write_file(a.out, sh.U);
    if (!a.rhs.empty()) write_file(a.rhs, sh.rhs);
    if (!a.faces.empty()) write_file(a.faces, sh.faces);
    if (!a.dts.empty()) write_file(a.dts, sh.dts);
    if (a.time)
        std::printf("{\"seconds\": %.9g, \"steps\": %ld, \"t_final\": %.17g, \"ranks\": %d}\n", sh.seconds, sh.nsteps, sh.t_final, P);
    return 0;
}
