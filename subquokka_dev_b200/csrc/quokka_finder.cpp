// quokka_finder: subcircuit files for the reference's subcircuit runner.
//
//   quokka_finder circuit.txt [mode] [sub.txt] [--chunk K] [--qubits N]
//
// The positional arguments are those of the reference's finder
// (subcircuitFinder/finder.cpp:771-784):
// - the flat circuit file;
// - a mode, 0 or 1 (the reference's two chunk-search principles); both
//   select the one search of qk_circuit_chunk_groups;
// - the output file, sub.txt by default.
// The chunk is 12 qubits as in the reference (finder.cpp:797) unless --chunk
// says otherwise.  The qubit count defaults to the highest qubit used + 1.
// The output runs with is_subcircuit=1 in the reference's MEM runner and in
// the GPU runner, and computes the flat file's state.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "quokka_gpu.h"

static int usage() {
    std::fprintf(stderr, "usage: quokka_finder circuit.txt [mode] [sub.txt] [--chunk K] [--qubits N]\n");
    return 1;
}

int main(int argc, char *argv[]) {
    std::string in, out = "sub.txt";
    int mode = 0, chunk = 12, qubits = 0, npos = 0;
    for (int i = 1; i < argc; ++i) {
        const std::string a(argv[i]);
        if ((a == "--chunk" || a == "--qubits") && i + 1 < argc) {
            (a == "--chunk" ? chunk : qubits) = std::atoi(argv[++i]);
        } else if (!a.empty() && a[0] == '-') {
            return usage();
        } else if (npos == 0) {
            in = a, ++npos;
        } else if (npos == 1) {
            mode = std::atoi(a.c_str()), ++npos;
        } else if (npos == 2) {
            out = a, ++npos;
        } else {
            return usage();
        }
    }
    if (in.empty() || (mode != 0 && mode != 1)) return usage();
    qk_circuit *c = nullptr;
    if (qk_circuit_load(in.c_str(), 0, 63, &c)) {
        std::fprintf(stderr, "quokka_finder: %s\n", qk_last_error());
        return 1;
    }
    const qk_gate *g = qk_circuit_gates(c);
    const size_t ng = qk_circuit_num_gates(c);
    int n = qubits;
    if (n <= 0)
        for (size_t i = 0; i < ng; ++i)
            for (int j = 0; j < g[i].nq; ++j) n = g[i].q[j] + 1 > n ? g[i].q[j] + 1 : n;
    if (chunk > n) chunk = n;
    qk_circuit *sub = nullptr;
    int rc = qk_circuit_chunk_groups(g, ng, n, chunk, &sub);
    if (!rc) rc = qk_circuit_write(sub, 1, out.c_str());
    if (rc) {
        std::fprintf(stderr, "quokka_finder: %s\n", qk_last_error());
        qk_circuit_destroy(c);
        qk_circuit_destroy(sub);
        return 1;
    }
    size_t vswaps = 0;
    const qk_gate *sg = qk_circuit_gates(sub);
    for (size_t i = 0; i < qk_circuit_num_gates(sub); ++i) vswaps += sg[i].kind == QK_GATE_VSWAP;
    std::printf("%s: %d qubits, chunk %d, %zu gates -> %zu groups (%zu VSWAP)\n", out.c_str(), n, chunk, ng,
                qk_circuit_num_groups(sub), vswaps);
    qk_circuit_destroy(c);
    qk_circuit_destroy(sub);
    return 0;
}
