// main.cpp -- the reference's driver (src/main.cpp:9-39) on the CUDA backend:
//
//     wenofv_host [settings.cfg] [KEY=VALUE ...] [--dump-ic FILE]
//
// reads the settings file (default ./config/settings.cfg), lets KEY=VALUE arguments
// override its keys, builds TwoPhaseEquation and CWENOFV and runs the solver on one GPU.
// --dump-ic FILE writes the initial cell averages ([i][j][r], FP64), and for NEUMANN2 the
// ghost frame to FILE.frame ([r][ny+8][nx+8]), and exits without touching the GPU.  No MPI: the whole domain is one GPU's.
#include <cstring>
#include <fstream>
#include <iostream>

#include "../include/ReadConfig.hpp"
#include "../include/WENOFV.hpp"

int main(int argc, char *argv[])
{
    std::string inputfile = "./config/settings.cfg", dump_ic;
    std::map<std::string, std::string> overrides;
    for (int a = 1; a < argc; a++) {
        const char *s = argv[a];
        if (!std::strcmp(s, "--dump-ic") && a + 1 < argc) dump_ic = argv[++a];
        else if (std::strchr(s, '=')) {
            const std::string kv(s);
            const size_t eq = kv.find('=');
            overrides[CConfig::trim(kv.substr(0, eq))] = CConfig::trim(kv.substr(eq + 1));
        } else inputfile = s;
    }
    TwoPhaseEquation *equation = new TwoPhaseEquation();
    CConfig config(inputfile);
    std::map<std::string, std::string> option;
    if (!config.read(option)) return 1;
    for (const auto &kv : overrides) option[kv.first] = kv.second;
    try {
        CWENOFV solver(equation, option);
        if (!dump_ic.empty()) {
            solver.initializeGrid();
            solver.initializeAve();
            std::ofstream f(dump_ic, std::ios::binary);
            f.write(reinterpret_cast<const char *>(solver.m_Uh.data()), (std::streamsize)(solver.m_Uh.size() * sizeof(double)));
            bool ok = (bool)f;
            if (!solver.m_frame.empty()) { // NEUMANN2: the ghost frame beside it, FILE.frame
                std::ofstream g(dump_ic + ".frame", std::ios::binary);
                g.write(reinterpret_cast<const char *>(solver.m_frame.data()), (std::streamsize)(solver.m_frame.size() * sizeof(double)));
                ok = ok && (bool)g;
            }
            delete equation;
            return ok ? 0 : 1;
        }
        solver.run();
    } catch (const std::exception &e) {
        std::cerr << "error: " << e.what() << std::endl;
        delete equation;
        return 1;
    }
    delete equation;
    return 0;
}
