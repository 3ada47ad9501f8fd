// quokka: drop-in command line for the GPU runner.
//
//   quokka -i x.ini -c circuit.txt
//
// Same flags, messages and exit codes as the reference's CLI (src/main.cpp:13-20,
// readargs at src/common.cpp:5-31) and the same stdout lines as
// Simulator::setupIni / Simulator::run (src/simulator.cpp:188-230, :671-706):
// a mode line, then the runner-only wall time "<sec>s".  runner_type=GPU (the
// slot the reference leaves unimplemented, src/simulator.cpp:225-228) and
// runner_type=MEM both run on the GPU; the state never leaves HBM until the
// optional dump.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include "quokka_gpu.h"

static void readargs(int argc, char *argv[], std::string &ini, std::string &circuit) {
    for (int i = 1; i < argc; ++i) {
        std::string arg(argv[i]);
        if (arg.length() > 1 && arg[0] == '-') {
            std::string option = arg.substr(1);
            if (option == "i" && i + 1 < argc) {
                ++i;
                std::cout << "[Config File]: " << argv[i] << std::endl;
                ini = argv[i];
            } else if (option == "c" && i + 1 < argc) {
                ++i;
                std::cout << "[Circuit File]: " << argv[i] << std::endl;
                circuit = argv[i];
            } else {
                std::cout << "[Unknown Option]: " << option << std::endl;
                std::exit(1);
            }
        } else {
            std::cout << "[Non-option Argument]: " << arg << std::endl;
            std::exit(1);
        }
    }
}

static int die(const char *what) {
    std::cerr << what << ": " << qk_last_error() << std::endl;
    return 1;
}

int main(int argc, char *argv[]) {
    std::string ini, cir;
    readargs(argc, argv, ini, cir);

    qk_config cfg;
    if (qk_config_load(ini.c_str(), &cfg)) {
        std::cerr << "Error parsing config.ini!" << std::endl;
        std::cerr << qk_last_error() << std::endl;
        return 1;
    }
    const std::string runner = cfg.runner_type;
    if (runner != "GPU" && runner != "MEM") {
        std::cerr << "[Config File]: " << runner << " runner not found." << std::endl;
        return 1;
    }
    if (cfg.mpi_qbit != 0) {
        std::cerr << "[Config File]: mpi_qbit > 0 is not supported by the GPU runner." << std::endl;
        return 1;
    }
    std::cout << "GPU Mode" << std::endl;

    qk_circuit *c = nullptr;
    if (qk_circuit_load(cir.c_str(), cfg.is_subcircuit, cfg.total_qbit, &c)) return die("[setGate]");
    std::cerr << "[Simulator]: Circuit setup." << std::endl;

    qk_sv *sv = nullptr;
    if (qk_sv_create(cfg.total_qbit, cfg.precision, &sv)) return die("[GPU_Runner]");
    if (cfg.init_file[0] && qk_sv_load(sv, cfg.init_file)) return die("[init_file]");
    std::cerr << "[Simulator]: Ready to go." << std::endl;

    double sec = 0;
    if (qk_run(&cfg, c, sv, &sec)) return die("[GPU_Runner]");
    std::cout << sec << "s" << std::endl;

    const std::string dump = cfg.dump_file;
    if (!dump.empty() && cfg.dump_binary) {
        if (qk_sv_save(sv, dump.c_str())) return die("[dump]");
    } else if (!dump.empty() && cfg.MPI_testing) {
        // the reference's text dump: name = dump_file[0:3] + rank + ".txt",
        // one "%.11f" line per real and imaginary part (src/simulator.cpp:696-704)
        std::vector<double> host((size_t)2 << cfg.total_qbit);
        if (qk_sv_download(sv, host.data())) return die("[dump]");
        std::ofstream res(dump.substr(0, 3) + "0.txt");
        for (size_t k = 0; k < host.size(); k += 2)
            res << std::fixed << std::setprecision(11) << host[k] << "\n" << host[k + 1] << "\n";
    }
    qk_sv_destroy(sv);
    qk_circuit_destroy(c);
    return 0;
}
