// Dense simulation of lowered ops on small states, and random ops, for the
// CPU checks of the planner (rewrite_check.cpp, plan_check.cpp).  Written
// from the op definitions in qk_internal.h, independently of the planner.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "qk_internal.h"

namespace dense_sim {

using qk::Op;
using cd = std::complex<double>;
using State = std::vector<cd>;

inline cd c(const double *m, int k) { return {m[2 * k], m[2 * k + 1]}; }

// apply a 2^k x 2^k matrix (row-major complex) on qubits qs (index bit i = qs[i])
inline void apply_matrix(State &s, int n, const std::vector<int> &qs, const std::vector<cd> &m) {
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
inline std::vector<cd> matrix_of(const Op &op, std::vector<int> &qs) {
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
inline double grad_term(const State &psi, const State &lam, int n, int q, double a, double b, double cz) {
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

inline void gen_abc(const Op &op, int which, double &a, double &b, double &cz) {
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
inline void run(const std::vector<Op> &ops, int n, State &psi, State &lam, std::vector<double> &g) {
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

inline Op lower(const qk_gate &g) {
    Op o;
    if (qk::lower_gate(g, o)) {
        std::fprintf(stderr, "lower_gate failed\n");
        std::exit(2);
    }
    return o;
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
    qk_gate gate() {
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
        return g;
    }
    Op op() { return lower(gate()); }
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

inline double max_diff(const State &a, const State &b) {
    double d = 0;
    for (size_t i = 0; i < a.size(); ++i) d = std::max(d, std::abs(a[i] - b[i]));
    return d;
}

}  // namespace dense_sim
