// CPU check of the op-list rewrites (subquokka_dev_b200/csrc/qk_rewrite.cpp).
//
// Random op lists built from parsed gates (every MEM gate kind, random U1 /
// U2 matrices, CNOT-shaped U2s, VSWAPs) are run on small dense states by an
// independent simulator below, once as generated and once after the
// rewrites the planners apply:
// - forward lists: merge_one_qubit_runs, absorb_into_two_qubit_ops,
//   asap_order, relabel_perms; the final states must agree;
// - backward lists with gradient ops (Im <lambda|G|psi>, G = X, Y, Z):
//   hoist_gradients, merge_one_qubit_runs, absorb_into_two_qubit_ops,
//   pair_gradients; the final states and every gradient must agree.
// Exit status 0 when every case agrees within 1e-12.  One exception, from
// the reference's H: its constant 0.70710678118 makes H = 2c^2 (1 - 1.1e-11)
// times a unitary, so a gradient op moved past an H on another qubit (which
// commutes with it) changes by 1.1e-11 relative per H.  Lists with H are
// checked at 1e-12 for the states and 1e-9 for the gradients; lists without
// H at 1e-12 for both.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "qk_internal.h"

using qk::Op;
using cd = std::complex<double>;
using State = std::vector<cd>;

namespace {

cd c(const double *m, int k) { return {m[2 * k], m[2 * k + 1]}; }

// apply a 2^k x 2^k matrix (row-major complex) on qubits qs (index bit i = qs[i])
void apply_matrix(State &s, int n, const std::vector<int> &qs, const std::vector<cd> &m) {
    const int k = (int)qs.size(), d = 1 << k;
    const size_t N = (size_t)1 << n;
    size_t mask = 0;
    for (int q : qs) mask |= (size_t)1 << q;
    std::vector<cd> in(d), out(d);
    for (size_t base = 0; base < N; ++base) {
        if (base & mask) continue;
        for (int j = 0; j < d; ++j) {
            size_t idx = base;
            for (int i = 0; i < k; ++i)
                if ((j >> i) & 1) idx |= (size_t)1 << qs[i];
            in[j] = s[idx];
        }
        for (int r = 0; r < d; ++r) {
            cd acc = 0;
            for (int j = 0; j < d; ++j) acc += m[r * d + j] * in[j];
            out[r] = acc;
        }
        for (int j = 0; j < d; ++j) {
            size_t idx = base;
            for (int i = 0; i < k; ++i)
                if ((j >> i) & 1) idx |= (size_t)1 << qs[i];
            s[idx] = out[j];
        }
    }
}

// the matrix of a non-gradient op over its qubits, written from the op
// definitions in qk_internal.h
std::vector<cd> matrix_of(const Op &op, std::vector<int> &qs) {
    qs.assign(op.q, op.q + op.nq);
    switch (op.kind) {
    case qk::OP_DENSE1: return {c(op.m, 0), c(op.m, 1), c(op.m, 2), c(op.m, 3)};
    case qk::OP_PHASE1: return {1, 0, 0, c(op.m, 0)};
    case qk::OP_DIAG1: return {c(op.m, 0), 0, 0, c(op.m, 1)};
    case qk::OP_DENSE2: {
        std::vector<cd> m(16);
        for (int k = 0; k < 16; ++k) m[k] = c(op.m, k);
        return m;
    }
    case qk::OP_PHASE2: {
        std::vector<cd> m(16, 0);
        m[0] = m[5] = m[10] = 1;
        m[15] = c(op.m, 0);
        return m;
    }
    case qk::OP_DIAG2: {
        std::vector<cd> m(16, 0);
        for (int k = 0; k < 4; ++k) m[5 * k] = c(op.m, k);
        return m;
    }
    case qk::OP_SWAP2: {
        std::vector<cd> m(16, 0);
        m[0] = m[15] = 1;
        m[4 * 1 + 2] = m[4 * 2 + 1] = 1;
        return m;
    }
    case qk::OP_CX: {
        std::vector<cd> m(16, 0);
        const int ctl = op.aux, tgt = 1 - op.aux;
        for (int j = 0; j < 4; ++j) m[4 * (((j >> ctl) & 1) ? j ^ (1 << tgt) : j) + j] = 1;
        return m;
    }
    case qk::OP_CDENSE1: {   // q[0] target (bit 0), q[1] condition (bit 1)
        std::vector<cd> m(16, 0);
        for (int bc = 0; bc < 2; ++bc)
            for (int r = 0; r < 2; ++r)
                for (int j = 0; j < 2; ++j) m[4 * (r + 2 * bc) + (j + 2 * bc)] = c(op.m + 8 * bc, 2 * r + j);
        return m;
    }
    case qk::OP_PERM: {   // swap bit q[i] with bit q[k+i]
        const int k = op.nq / 2, d = 1 << op.nq;
        std::vector<cd> m((size_t)d * d, 0);
        for (int j = 0; j < d; ++j) {
            int r = j;
            for (int i = 0; i < k; ++i) {
                const int a = (j >> i) & 1, b = (j >> (k + i)) & 1;
                r = (r & ~(1 << i) & ~(1 << (k + i))) | (b << i) | (a << (k + i));
            }
            m[(size_t)r * d + j] = 1;
        }
        return m;
    }
    default: break;
    }
    std::fprintf(stderr, "unexpected op kind %d\n", op.kind);
    std::exit(2);
}

// Im <lambda| G |psi> on qubit q, G = a X + b Y + c Z
double grad_term(const State &psi, const State &lam, int n, int q, double a, double b, double cz) {
    const cd g00 = cz, g01 = cd(a, -b), g10 = cd(a, b), g11 = -cz;
    double s = 0;
    for (size_t i = 0; i < ((size_t)1 << n); ++i) {
        if ((i >> q) & 1) continue;
        const size_t j = i | ((size_t)1 << q);
        const cd gp0 = g00 * psi[i] + g01 * psi[j], gp1 = g10 * psi[i] + g11 * psi[j];
        s += (std::conj(lam[i]) * gp0 + std::conj(lam[j]) * gp1).imag();
    }
    return s;
}

void gen_abc(const Op &op, int which, double &a, double &b, double &cz) {
    const int gen = (int)op.m[0];
    if (gen == 5) {
        a = op.m[2 + 3 * which];
        b = op.m[3 + 3 * which];
        cz = op.m[4 + 3 * which];
        return;
    }
    a = gen == 1 ? 1 : gen == 4 ? op.m[2] : 0;
    b = gen == 2 ? 1 : gen == 4 ? op.m[3] : 0;
    cz = gen == 3 ? 1 : gen == 4 ? op.m[4] : 0;
}

// run a list on psi and lambda; gradient ops add into g[parameter]
void run(const std::vector<Op> &ops, int n, State &psi, State &lam, std::vector<double> &g) {
    for (const Op &op : ops) {
        if (op.kind == qk::OP_GRAD) {
            double a, b, cz;
            gen_abc(op, 0, a, b, cz);
            g[op.aux] += grad_term(psi, lam, n, op.q[0], a, b, cz);
            if ((int)op.m[0] == 5) {
                gen_abc(op, 1, a, b, cz);
                g[(int)op.m[8]] += grad_term(psi, lam, n, op.q[0], a, b, cz);
            }
            continue;
        }
        std::vector<int> qs;
        const std::vector<cd> m = matrix_of(op, qs);
        apply_matrix(psi, n, qs, m);
        apply_matrix(lam, n, qs, m);
    }
}

struct Gen {
    std::mt19937_64 rng;
    int n;
    bool with_h;
    double u() { return std::uniform_real_distribution<double>(-3, 3)(rng); }
    int qubit() { return (int)(rng() % n); }
    void unitary(int d, double *out) {   // Gram-Schmidt on a random complex matrix
        std::vector<cd> m((size_t)d * d);
        for (auto &x : m) x = cd(u(), u());
        for (int r = 0; r < d; ++r) {
            for (int p = 0; p < r; ++p) {
                cd dot = 0;
                for (int k = 0; k < d; ++k) dot += std::conj(m[p * d + k]) * m[r * d + k];
                for (int k = 0; k < d; ++k) m[r * d + k] -= dot * m[p * d + k];
            }
            double nr = 0;
            for (int k = 0; k < d; ++k) nr += std::norm(m[r * d + k]);
            for (int k = 0; k < d; ++k) m[r * d + k] /= std::sqrt(nr);
        }
        for (int k = 0; k < d * d; ++k) {
            out[2 * k] = m[k].real();
            out[2 * k + 1] = m[k].imag();
        }
    }
    Op op() {
        qk_gate g;
        std::memset(&g, 0, sizeof g);
        const int r = (int)(rng() % 13);
        const int a = qubit();
        int b = qubit();
        while (b == a) b = qubit();
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        static const int one[] = {QK_GATE_H, QK_GATE_X, QK_GATE_Y, QK_GATE_Z, QK_GATE_P, QK_GATE_RX, QK_GATE_RY,
                                  QK_GATE_RZ, QK_GATE_U1};
        if (r < 9) {
            g.kind = one[r] == QK_GATE_H && !with_h ? QK_GATE_RX : one[r];
            g.nq = 1;
            g.q[0] = a;
            g.param = u();
            if (g.kind == QK_GATE_U1) unitary(2, g.coeff);
        } else {
            static const int two[] = {QK_GATE_U2, QK_GATE_CP, QK_GATE_RZZ, QK_GATE_SWAP};
            g.kind = two[r - 9];
            g.nq = 2;
            g.q[0] = lo;
            g.q[1] = hi;
            g.param = u();
            if (g.kind == QK_GATE_U2) {
                if (rng() % 2) {   // a CNOT either way (big-endian file order)
                    static const int p0[4] = {0, 1, 3, 2}, p1[4] = {0, 3, 2, 1};
                    const int *p = rng() % 2 ? p0 : p1;
                    for (int k = 0; k < 4; ++k) g.coeff[2 * (4 * k + p[k])] = 1;
                } else {
                    unitary(4, g.coeff);
                }
            }
        }
        Op o;
        if (qk::lower_gate(g, o)) {
            std::fprintf(stderr, "lower_gate failed\n");
            std::exit(2);
        }
        return o;
    }
    Op vswap() {
        Op o;
        std::memset(&o, 0, sizeof o);
        o.kind = qk::OP_PERM;
        o.nq = 4;
        std::vector<int> qs(n);
        for (int i = 0; i < n; ++i) qs[i] = i;
        std::shuffle(qs.begin(), qs.end(), rng);
        for (int i = 0; i < 4; ++i) o.q[i] = qs[i];
        return o;
    }
    State state() {
        State s((size_t)1 << n);
        double nr = 0;
        for (auto &x : s) {
            x = cd(u(), u());
            nr += std::norm(x);
        }
        for (auto &x : s) x /= std::sqrt(nr);
        return s;
    }
};

double max_diff(const State &a, const State &b) {
    double d = 0;
    for (size_t i = 0; i < a.size(); ++i) d = std::max(d, std::abs(a[i] - b[i]));
    return d;
}

}  // namespace

int main() {
    int bad = 0;
    for (int seed = 0; seed < 120; ++seed) {
        const bool with_h = seed >= 60;
        const double gtol = with_h ? 1e-9 : 1e-12;
        Gen G{std::mt19937_64(seed), 4 + seed % 4, with_h};
        const int n = G.n;
        // forward list
        std::vector<Op> ops;
        for (int i = 0; i < 60; ++i) ops.push_back(seed % 3 == 0 && i % 17 == 5 ? G.vswap() : G.op());
        std::vector<Op> rw = ops;
        qk::relabel_perms(rw, n, 2, 8, 2, seed % 2 == 0);
        qk::merge_one_qubit_runs(rw, n);
        qk::absorb_into_two_qubit_ops(rw, n);
        if (seed % 2) qk::asap_order(rw, n);
        State p0 = G.state(), l0 = p0, p1 = p0, l1 = p0;
        std::vector<double> g0(64, 0), g1(64, 0);
        run(ops, n, p0, l0, g0);
        run(rw, n, p1, l1, g1);
        const double df = max_diff(p0, p1);
        if (df > 1e-12) {
            std::printf("forward seed %d: max |d amp| %.3g (%zu -> %zu ops)\n", seed, df, ops.size(), rw.size());
            ++bad;
        }
        // backward list: gradient ops on random qubits between the ops
        std::vector<Op> back;
        int np = 0;
        for (int i = 0; i < 60; ++i) {
            Op o = G.op();
            if (o.nq == 1 && G.rng() % 2 && np < 64) {
                Op gr;
                std::memset(&gr, 0, sizeof gr);
                gr.kind = qk::OP_GRAD;
                gr.nq = 1;
                gr.q[0] = o.q[0];
                gr.m[0] = 1 + (int)(G.rng() % 3);
                gr.aux = np++;
                back.push_back(gr);
            }
            back.push_back(o);
        }
        std::vector<Op> bw = back;
        qk::hoist_gradients(bw, n);
        qk::merge_one_qubit_runs(bw, n);
        qk::absorb_into_two_qubit_ops(bw, n);
        qk::pair_gradients(bw);
        State psi = G.state(), lam = G.state(), psi2 = psi, lam2 = lam;
        std::vector<double> h0(64, 0), h1(64, 0);
        run(back, n, psi, lam, h0);
        run(bw, n, psi2, lam2, h1);
        double dg = 0;
        for (int k = 0; k < 64; ++k) dg = std::max(dg, std::fabs(h0[k] - h1[k]));
        const double ds = std::max(max_diff(psi, psi2), max_diff(lam, lam2));
        if (dg > gtol || ds > 1e-12) {
            std::printf("backward seed %d: max |d grad| %.3g, max |d amp| %.3g (%zu -> %zu ops)\n", seed, dg, ds,
                        back.size(), bw.size());
            ++bad;
        }
    }
    std::printf("%s\n", bad ? "FAIL" : "ok");
    return bad ? 1 : 0;
}
