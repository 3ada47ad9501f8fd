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
// optional dump.  runner_type=IO or DirectIO (the reference's out-of-core
// runners, src/IO_Runner.cpp, src/DIO_Runner.cpp) keep the state in host
// memory instead of files and run it on the GPU chunk by chunk (qk_hsv_*);
// their state_paths key is not needed.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

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

// The reference's text dump of 2^n (re, im) pairs: name = dump_file[0:3] +
// rank + ".txt", one "%.11f" line per part (src/simulator.cpp:696-704).
template <typename T>
static void text_dump(const std::string &dump, const T *v, size_t n2) {
    std::ofstream res(dump.substr(0, 3) + "0.txt");
    for (size_t k = 0; k < n2; k += 2)
        res << std::fixed << std::setprecision(11) << (double)v[k] << "\n" << (double)v[k + 1] << "\n";
}

// runner_type=IO / DirectIO: the state in pinned host memory, chunks of
// 2^device_qbit amplitudes on the GPU.
static int run_host_state(const qk_config &cfg, const std::string &cir) {
    std::cout << (std::string(cfg.runner_type) == "IO" ? "IO Mode" : "DIO Mode") << std::endl;
    qk_circuit *c = nullptr;
    if (qk_circuit_load(cir.c_str(), cfg.is_subcircuit, cfg.total_qbit, &c)) return die("[setGate]");
    std::cerr << "[Simulator]: Circuit setup." << std::endl;
    const int n = cfg.total_qbit;
    const size_t es = cfg.precision == QK_C128 ? 16 : 8;
    int L = cfg.device_qbit;
    if (L == 0) {   // the largest chunk of which three fit in three quarters of the free HBM
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
        L = n;
        while (L > 1 && 3 * (es << L) > free_b / 4 * 3) --L;
    }
    qk_hsv *h = nullptr;
    if (qk_hsv_create(n, L, cfg.precision, &h)) return die("[IO_Runner]");
    if (cfg.init_file[0]) {
        // a state file holds raw complex128 (the dump_format=bin layout)
        FILE *f = std::fopen(cfg.init_file, "rb");
        if (!f) { std::cerr << "[init_file]: cannot open " << cfg.init_file << std::endl; return 1; }
        std::vector<double> buf((size_t)2 << 20);
        const size_t namp = (size_t)1 << n;
        for (size_t k = 0; k < namp; k += buf.size() / 2) {
            const size_t m = std::min(buf.size() / 2, namp - k);
            if (std::fread(buf.data(), 16, m, f) != m) { std::cerr << "[init_file]: short file" << std::endl; return 1; }
            if (cfg.precision == QK_C128) std::memcpy(static_cast<double *>(qk_hsv_data(h)) + 2 * k, buf.data(), 16 * m);
            else
                for (size_t j = 0; j < 2 * m; ++j) static_cast<float *>(qk_hsv_data(h))[2 * k + j] = (float)buf[j];
        }
        std::fclose(f);
    }
    std::cerr << "[Simulator]: Ready to go." << std::endl;
    // a subcircuit file's groups matter only to the reference's chunking: its
    // gates run as one list
    if (qk_hsv_apply_gates(h, qk_circuit_gates(c), qk_circuit_num_gates(c))) return die("[IO_Runner]");
    double ms = 0;
    qk_hsv_stats(h, nullptr, &ms, nullptr);
    std::cout << ms / 1e3 << "s" << std::endl;
    const std::string dump = cfg.dump_file;
    const size_t n2 = (size_t)2 << n;
    if (!dump.empty() && cfg.dump_binary) {
        FILE *f = std::fopen(dump.c_str(), "wb");
        if (!f) { std::cerr << "[dump]: cannot open " << dump << std::endl; return 1; }
        if (cfg.precision == QK_C128) {
            std::fwrite(qk_hsv_data(h), 8, n2, f);
        } else {
            const float *v = static_cast<const float *>(qk_hsv_data(h));
            std::vector<double> buf(1 << 20);
            for (size_t k = 0; k < n2; k += buf.size()) {
                const size_t m = std::min(buf.size(), n2 - k);
                for (size_t j = 0; j < m; ++j) buf[j] = v[k + j];
                std::fwrite(buf.data(), 8, m, f);
            }
        }
        std::fclose(f);
    } else if (!dump.empty() && cfg.MPI_testing) {
        if (cfg.precision == QK_C128) text_dump(dump, static_cast<const double *>(qk_hsv_data(h)), n2);
        else text_dump(dump, static_cast<const float *>(qk_hsv_data(h)), n2);
    }
    qk_hsv_destroy(h);
    qk_circuit_destroy(c);
    return 0;
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
    const bool host_state = runner == "IO" || runner == "DirectIO";
    if (runner != "GPU" && runner != "MEM" && !host_state) {
        std::cerr << "[Config File]: " << runner << " runner not found." << std::endl;
        return 1;
    }
    if (cfg.mpi_qbit != 0) {
        std::cerr << "[Config File]: mpi_qbit > 0 is not supported by the GPU runner." << std::endl;
        return 1;
    }
    if (host_state) return run_host_state(cfg, cir);
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
        std::vector<double> host((size_t)2 << cfg.total_qbit);
        if (qk_sv_download(sv, host.data())) return die("[dump]");
        text_dump(dump, host.data(), host.size());
    }
    qk_sv_destroy(sv);
    qk_circuit_destroy(c);
    return 0;
}
