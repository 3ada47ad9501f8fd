// Test-only driver around the UNMODIFIED reference simulator.
//
// Part of the oracle (test infrastructure): it is linked against the
// reference's own translation units (src/makefile:8, minus src/main.cpp) and
// never ships with the product.  It does what the reference's `main`
// (src/main.cpp:13-20) does -- readargs, Simulator(ini, cir), run() -- with
// two test hooks:
//   -s FILE  overwrite MEM_Runner::buffer (src/MEM_Runner.hpp:27, public) with
//            a raw little-endian complex<double> state before run(), so a
//            seeded random initial state can be used instead of |0...0>
//            (src/MEM_Runner.cpp:79-81);
//   -o FILE  write MEM_Runner::buffer as raw complex<double> after run().
// The reference's own dump (src/simulator.cpp:696-704) is 11-digit decimal
// text, too coarse for a 1e-12 parity check, hence the binary dump.
// Simulator::run prints the runner-only wall time "<sec>s"
// (src/simulator.cpp:679-689); callers parse that line.
#include <complex>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "circuit.hpp"
#include "simulator.hpp"
#include "MEM_Runner.hpp"

int main(int argc, char **argv) {
    std::string ini, cir, init_path, out_path;
    for (int i = 1; i < argc; ++i) {
        std::string a(argv[i]);
        if (i + 1 >= argc) { std::cerr << "missing value for " << a << "\n"; return 2; }
        if (a == "-i") ini = argv[++i];
        else if (a == "-c") cir = argv[++i];
        else if (a == "-s") init_path = argv[++i];
        else if (a == "-o") out_path = argv[++i];
        else { std::cerr << "unknown option " << a << "\n"; return 2; }
    }
    if (ini.empty() || cir.empty()) {
        std::cerr << "usage: quokka_ref -i x.ini -c circuit.txt [-s init.bin] [-o out.bin]\n";
        return 2;
    }
    Simulator sim(ini, cir);
    MEM_Runner *mem = dynamic_cast<MEM_Runner *>(sim.Runner);
    if (!mem) { std::cerr << "runner_type must be MEM\n"; return 3; }
    std::vector<std::complex<double>> &buf = mem->buffer;
    if (!init_path.empty()) {
        FILE *f = std::fopen(init_path.c_str(), "rb");
        if (!f) { std::cerr << "cannot open " << init_path << "\n"; return 4; }
        size_t got = std::fread(buf.data(), sizeof(std::complex<double>), buf.size(), f);
        std::fclose(f);
        if (got != buf.size()) { std::cerr << "short initial state\n"; return 4; }
    }
    sim.run();
    if (!out_path.empty()) {
        FILE *f = std::fopen(out_path.c_str(), "wb");
        if (!f) { std::cerr << "cannot open " << out_path << "\n"; return 5; }
        size_t put = std::fwrite(buf.data(), sizeof(std::complex<double>), buf.size(), f);
        std::fclose(f);
        if (put != buf.size()) { std::cerr << "short write\n"; return 5; }
    }
    return 0;
}
