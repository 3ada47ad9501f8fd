// GPU_Runner over libquokka_gpu.so; see GPU_Runner.hpp.
#include "GPU_Runner.hpp"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "circuit.hpp"

namespace {

[[noreturn]] void die(const char *where) {
    std::cerr << where << ": " << qk_last_error() << std::endl;
    std::exit(1);
}

qk_gate blank(int kind, const std::vector<int> &targs) {
    qk_gate q;
    std::memset(&q, 0, sizeof q);
    q.kind = kind;
    q.nq = (int)targs.size();
    for (size_t i = 0; i < targs.size() && i < QK_MAX_TARGETS; ++i) q.q[i] = targs[i];
    return q;
}

// The MEM gate objects keep the coefficients their constructors derived
// from the written angle (src/circuit.cpp:2655, :2706-2709, :2734-2737,
// :2762-2765, :2947-2949, :2988-2991); the angle is read back from them, and
// the engine derives the same coefficients again (to the last bit or one
// unit in the last place).
double angle(std::complex<double> e) { return std::atan2(e.imag(), e.real()); }

}  // namespace

qk_gate GPU_Runner::to_qk(const Gate *g) {
    const std::vector<int> &t = g->targs;
    if (dynamic_cast<const H_Gate_MEM *>(g)) return blank(QK_GATE_H, t);
    if (dynamic_cast<const X_Gate_MEM *>(g)) return blank(QK_GATE_X, t);
    if (dynamic_cast<const Y_Gate_MEM *>(g)) return blank(QK_GATE_Y, t);
    if (dynamic_cast<const Z_Gate_MEM *>(g)) return blank(QK_GATE_Z, t);
    if (auto p = dynamic_cast<const Phase_Gate_MEM *>(g)) {
        qk_gate q = blank(QK_GATE_P, t);
        q.param = angle(p->phi);
        return q;
    }
    if (auto p = dynamic_cast<const U1_Gate_MEM *>(g)) {
        qk_gate q = blank(QK_GATE_U1, t);
        for (int k = 0; k < 4; ++k) {
            q.coeff[2 * k] = p->coeff[k].real();
            q.coeff[2 * k + 1] = p->coeff[k].imag();
        }
        return q;
    }
    if (auto p = dynamic_cast<const RX_Gate_MEM *>(g)) {   // cos(phi/2), i sin(-phi/2)
        qk_gate q = blank(QK_GATE_RX, t);
        q.param = 2 * std::atan2(-p->i_sin_Phi_2.imag(), p->cos_Phi_2.real());
        return q;
    }
    if (auto p = dynamic_cast<const RY_Gate_MEM *>(g)) {   // cos(phi/2), sin(phi/2)
        qk_gate q = blank(QK_GATE_RY, t);
        q.param = 2 * std::atan2(p->sin_Phi_2.real(), p->cos_Phi_2.real());
        return q;
    }
    if (auto p = dynamic_cast<const RZ_Gate_MEM *>(g)) {   // e^{+i phi/2}
        qk_gate q = blank(QK_GATE_RZ, t);
        q.param = 2 * angle(p->exp_p_iPhi_2);
        return q;
    }
    if (auto p = dynamic_cast<const U2_Gate_MEM *>(g)) {
        // the constructor stored file entry res(i) at i (src/circuit.cpp:
        // 2811-2819); put each back at its file position
        qk_gate q = blank(QK_GATE_U2, t);
        for (int i = 0; i < 16; ++i) {
            const int b1 = i & 1, b2 = (i >> 1) & 1, b3 = (i >> 2) & 1, b4 = (i >> 3) & 1;
            const int res = (b3 << 3) | (b4 << 2) | (b1 << 1) | b2;
            q.coeff[2 * res] = p->coeff[i].real();
            q.coeff[2 * res + 1] = p->coeff[i].imag();
        }
        return q;
    }
    // VSWAP_1_1 and MPI_VSWAP_1_1 are SWAP_Gate_MEM subclasses: test them first
    if (dynamic_cast<const VSWAP_Gate_1_1_MEM *>(g)) return blank(QK_GATE_VSWAP, t);
    if (dynamic_cast<const MPI_VSWAP_Gate_1_1_MEM *>(g)) return blank(QK_GATE_MPI_VSWAP, t);
    if (dynamic_cast<const SWAP_Gate_MEM *>(g)) return blank(QK_GATE_SWAP, t);
    if (auto p = dynamic_cast<const CPhase_Gate_MEM *>(g)) {
        qk_gate q = blank(QK_GATE_CP, t);
        q.param = angle(p->exp_iPhi);
        return q;
    }
    if (auto p = dynamic_cast<const RZZ_Gate_MEM *>(g)) {
        qk_gate q = blank(QK_GATE_RZZ, t);
        q.param = 2 * angle(p->exp_p_iPhi_2);
        return q;
    }
    if (dynamic_cast<const VSWAP_Gate_2_2_MEM *>(g) || dynamic_cast<const VSWAP_Gate_3_3_MEM *>(g) ||
        dynamic_cast<const VSWAP_Gate_4_4_MEM *>(g) || dynamic_cast<const VSWAP_Gate_6_6_MEM *>(g))
        return blank(QK_GATE_VSWAP, t);
    if (dynamic_cast<const MPI_VSWAP_Gate_2_2_MEM *>(g)) return blank(QK_GATE_MPI_VSWAP, t);
    std::cerr << "[GPU_Runner]: gate " << g->name << " has no GPU form" << std::endl;
    std::exit(1);
}

GPU_Runner::GPU_Runner(const std::string &ini) {
    if (qk_config_load(ini.c_str(), &cfg) != QK_OK) die("[Config File]");
    if (cfg.mpi_qbit != 0) {
        std::cerr << "[Config File]: mpi_qbit > 0 is not supported by the GPU runner." << std::endl;
        std::exit(1);
    }
    if (qk_sv_create(seg.N, cfg.precision, &sv) != QK_OK) die("[GPU_Runner]");
    if (cfg.init_file[0] && qk_sv_load(sv, cfg.init_file) != QK_OK) die("[init_file]");
}

GPU_Runner::~GPU_Runner() {
    const std::string dump = cfg.dump_file;
    if (!dump.empty() && cfg.dump_binary) {
        if (qk_sv_save(sv, dump.c_str()) != QK_OK) die("[dump]");
    } else if (!dump.empty() && cfg.MPI_testing) {
        // the reference's text dump: dump_file[0:3] + rank + ".txt", one
        // "%.11f" line per real and imaginary part
        std::vector<double> host((size_t)2 << seg.N);
        if (qk_sv_download(sv, host.data()) != QK_OK) die("[dump]");
        std::ofstream res(dump.substr(0, 3) + std::to_string(env.rank) + ".txt");
        for (size_t k = 0; k < host.size(); k += 2)
            res << std::fixed << std::setprecision(11) << host[k] << "\n" << host[k + 1] << "\n";
    }
    qk_sv_destroy(sv);
}

static qk_plan_opts plan_opts(const qk_config &cfg) {
    qk_plan_opts o;
    std::memset(&o, 0, sizeof o);
    o.dtype = cfg.precision;
    o.fuse_width = (cfg.fuse_width == 5 || cfg.fuse_width == 6) && cfg.precision == QK_C64 ? cfg.fuse_width : 0;
    return o;
}

void GPU_Runner::run(std::vector<Gate *> &circuit) {
    std::vector<qk_gate> g;
    g.reserve(circuit.size());
    for (const Gate *x : circuit) g.push_back(to_qk(x));
    int rc;
    if (cfg.fuse_width > 0) {
        const qk_plan_opts o = plan_opts(cfg);
        qk_plan *p = nullptr;
        rc = qk_plan_create(g.data(), g.size(), seg.N, &o, &p);
        if (rc == QK_OK) rc = qk_plan_apply(sv, p);
        qk_plan_destroy(p);
    } else {
        rc = qk_apply_gates(sv, g.data(), g.size());
    }
    // Simulator::run times this call on the host clock: finish the device work
    if (rc == QK_OK) rc = qk_sv_synchronize(sv);
    if (rc != QK_OK) die("[GPU_Runner]");
}

void GPU_Runner::run(std::vector<std::vector<Gate *>> &subcircuits) {
    std::vector<qk_gate> g;
    std::vector<int32_t> sizes;
    for (const auto &group : subcircuits) {
        sizes.push_back((int32_t)group.size());
        for (const Gate *x : group) g.push_back(to_qk(x));
    }
    const qk_plan_opts o = plan_opts(cfg);
    qk_plan *p = nullptr;
    int rc = qk_plan_create_groups(g.data(), sizes.data(), sizes.size(), seg.N, &o, &p);
    if (rc == QK_OK) rc = qk_plan_apply(sv, p);
    qk_plan_destroy(p);
    if (rc == QK_OK) rc = qk_sv_synchronize(sv);
    if (rc != QK_OK) die("[GPU_Runner]");
}
