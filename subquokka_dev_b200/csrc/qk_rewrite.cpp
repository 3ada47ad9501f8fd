// Op-list rewrites that run before planning.  Each keeps the state the list
// computes (up to rounding) and shortens the programs of fused passes:
// - asap_order: the list in ASAP layers (planners try both orders);
// - merge_one_qubit_runs, absorb_into_two_qubit_ops: fewer, heavier ops;
// - hoist_gradients, pair_gradients: backward sweeps with gradient ops that
//   no longer split runs of one-qubit ops;
// - relabel_perms: VSWAPs (and optionally SWAPs) as renamings of qubits.
#include <algorithm>
#include <array>
#include <cstring>
#include <utility>
#include <vector>

#include "qk_internal.h"

namespace qk {

// ASAP layers: level = 1 + the highest level on the op's qubits (a
// permutation op takes every qubit's level); a stable sort by level keeps
// each qubit's op order, so the list computes the same state.
void asap_order(std::vector<Op> &ops, int n) {
    std::vector<int> lvl(n, 0);
    std::vector<std::pair<int, size_t>> key(ops.size());
    for (size_t i = 0; i < ops.size(); ++i) {
        const Op &op = ops[i];
        const bool all = op.kind == OP_PERM;
        int l = 0;
        for (int k = 0; k < (all ? n : op.nq); ++k) l = std::max(l, lvl[all ? k : op.q[k]]);
        ++l;
        for (int k = 0; k < (all ? n : op.nq); ++k) lvl[all ? k : op.q[k]] = l;
        key[i] = {l, i};
    }
    std::stable_sort(key.begin(), key.end());
    std::vector<Op> sorted;
    sorted.reserve(ops.size());
    for (const auto &k : key) sorted.push_back(ops[k.second]);
    ops.swap(sorted);
}

// 2 x 2 complex products, row-major (re, im) pairs.
void mat2_mul(const double (&x)[8], const double (&y)[8], double (&z)[8]) {   // z = x y
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) {
            double re = 0, im = 0;
            for (int k = 0; k < 2; ++k) {
                const double xr = x[2 * (2 * r + k)], xi = x[2 * (2 * r + k) + 1];
                const double yr = y[2 * (2 * k + c)], yi = y[2 * (2 * k + c) + 1];
                re += xr * yr - xi * yi;
                im += xr * yi + xi * yr;
            }
            z[2 * (2 * r + c)] = re;
            z[2 * (2 * r + c) + 1] = im;
        }
}

// Consecutive one-qubit ops on the same qubit (no other op on that qubit
// between them) multiplied into one: the later op moves back past ops on
// other qubits, which commute with it.  Two diagonal ops give a diagonal op,
// anything else a dense one.  Gradient ops and multi-qubit ops end a run.
bool one_qubit(const Op &op) { return op.kind == OP_DENSE1 || op.kind == OP_PHASE1 || op.kind == OP_DIAG1; }

void as_matrix(const Op &op, double (&m)[8]) {
    std::memset(m, 0, sizeof m);
    if (op.kind == OP_DENSE1) {
        std::memcpy(m, op.m, sizeof m);
    } else if (op.kind == OP_PHASE1) {
        m[0] = 1;
        m[6] = op.m[0];
        m[7] = op.m[1];
    } else {   // OP_DIAG1
        m[0] = op.m[0];
        m[1] = op.m[1];
        m[6] = op.m[2];
        m[7] = op.m[3];
    }
}

void merge_one_qubit_runs(std::vector<Op> &ops, int n) {
    std::vector<long> last(n, -1);
    std::vector<Op> out;
    out.reserve(ops.size());
    for (const Op &op : ops) {
        if (one_qubit(op) && last[op.q[0]] >= 0) {
            Op &a = out[last[op.q[0]]];
            double x[8], y[8], z[8];
            as_matrix(a, x);
            as_matrix(op, y);
            mat2_mul(y, x, z);   // op after a
            if (a.kind != OP_DENSE1 && op.kind != OP_DENSE1) {
                a.kind = OP_DIAG1;
                a.m[0] = z[0]; a.m[1] = z[1]; a.m[2] = z[6]; a.m[3] = z[7];
            } else {
                a.kind = OP_DENSE1;
                std::memcpy(a.m, z, sizeof z);
            }
            continue;
        }
        for (int k = 0; k < op.nq; ++k) last[op.q[k]] = -1;
        out.push_back(op);
        if (one_qubit(op)) last[op.q[0]] = (long)out.size() - 1;
    }
    ops.swap(out);
}

// Real dense ops: a real 2 x 2 costs four multiply-adds an amplitude, a
// complex one eight.
bool op_is_real(const Op &op) {
    const int nc = op.kind == OP_DENSE1 ? 4 : (op.kind == OP_DENSE2 || op.kind == OP_CDENSE1) ? 16 : 0;
    if (!nc) return false;
    for (int k = 0; k < nc; ++k)
        if (op.m[2 * k + 1] != 0.0) return false;
    return true;
}

// 4 x 4 matrix of a two-qubit op, index b(q[0]) + 2 b(q[1]), row-major (re, im).
static void op_matrix4(const Op &op, double (&m)[32]) {
    std::memset(m, 0, sizeof m);
    auto set = [&](int r, int c, double re, double im) { m[2 * (4 * r + c)] = re; m[2 * (4 * r + c) + 1] = im; };
    switch (op.kind) {
    case OP_DENSE2: std::memcpy(m, op.m, sizeof m); break;
    case OP_PHASE2: set(0, 0, 1, 0); set(1, 1, 1, 0); set(2, 2, 1, 0); set(3, 3, op.m[0], op.m[1]); break;
    case OP_DIAG2: for (int k = 0; k < 4; ++k) set(k, k, op.m[2 * k], op.m[2 * k + 1]); break;
    case OP_SWAP2: set(0, 0, 1, 0); set(1, 2, 1, 0); set(2, 1, 1, 0); set(3, 3, 1, 0); break;
    case OP_CX: {
        const int c = op.aux, t = 1 - op.aux;
        for (int j = 0; j < 4; ++j) set(((j >> c) & 1) ? j ^ (1 << t) : j, j, 1, 0);
        break;
    }
    default: break;
    }
}

// A two-qubit op whose two qubits both end with a pending one-qubit op takes
// both in: O (U0 x U1) becomes one op (the one-qubit ops move forward past
// ops on other qubits only).  Two dense one-qubit ops and any two-qubit op
// give a dense 4 x 4 op, which costs the arithmetic of the two 2 x 2 ops it
// replaces; three diagonal ops give a diagonal one.  Other mixes are left
// alone, since they would add arithmetic; but a diagonal op or a CX with
// only one qubit's pending op dense takes that op in as OP_CDENSE1 (the
// 26-qubit HEA forward: 685 -> 375 program ops, 37 -> 30 ms c128; folding
// one of two pending ops this way instead of both was slower on the brick
// circuit, 689 against 679 ms).  On the brick circuits (U3 on
// every qubit, then CZ pairs) this removes two of every three ops: the
// 30-qubit 20-layer circuit has 407 program ops instead of 941 and, though a
// dense op needs both qubits in the tile (39 passes instead of 26), runs in
// 679 ms instead of 725 ms (c128).
//
// keep_real: no fold turns real one-qubit ops complex (the passes apply a
// real 2 x 2 or 4 x 4 with half the multiply-adds of a complex one).  Two real pending ops before a complex two-qubit op become one
// real 4 x 4 op (their tensor product) followed by that op; a real pending
// op is not folded into a complex conditioned op.
void absorb_into_two_qubit_ops(std::vector<Op> &ops, int n, bool keep_real) {
    std::vector<long> last(n, -1);
    std::vector<char> dead;
    std::vector<Op> out;
    out.reserve(ops.size());
    auto diag = [](const Op &o) { return o.kind == OP_PHASE1 || o.kind == OP_DIAG1; };
    for (const Op &op : ops) {
        const bool two = op.nq == 2 && (op.kind == OP_DENSE2 || op.kind == OP_PHASE2 || op.kind == OP_DIAG2 ||
                                        op.kind == OP_SWAP2 || op.kind == OP_CX);
        // with one qubit's pending op dense (not both), a diagonal op or a CX
        // takes it in as a one-qubit op conditioned on the other qubit, which
        // may then lie anywhere, as for the diagonal op itself
        const bool both = two && last[op.q[0]] >= 0 && last[op.q[1]] >= 0 && out[last[op.q[0]]].kind == OP_DENSE1 &&
                          out[last[op.q[1]]].kind == OP_DENSE1;
        if (!both && two && (op.kind == OP_PHASE2 || op.kind == OP_DIAG2 || op.kind == OP_CX)) {
            int x = -1;   // index in op.q of the target
            if (op.kind == OP_CX) x = last[op.q[1 - op.aux]] >= 0 && out[last[op.q[1 - op.aux]]].kind == OP_DENSE1 ? 1 - op.aux : -1;
            else if (last[op.q[0]] >= 0 && out[last[op.q[0]]].kind == OP_DENSE1) x = 0;
            else if (last[op.q[1]] >= 0 && out[last[op.q[1]]].kind == OP_DENSE1) x = 1;
            if (x >= 0) {
                const Op &u = out[last[op.q[x]]];
                double o4[32];
                op_matrix4(op, o4);
                Op f;
                std::memset(&f, 0, sizeof f);
                f.kind = OP_CDENSE1;
                f.nq = 2;
                f.q[0] = op.q[x];
                f.q[1] = op.q[1 - x];
                for (int bc = 0; bc < 2; ++bc) {
                    // the 2x2 block of o4 on the target for condition value bc
                    double blk[8], res[8];
                    for (int rt = 0; rt < 2; ++rt)
                        for (int ct = 0; ct < 2; ++ct) {
                            const int r = x == 0 ? rt + 2 * bc : bc + 2 * rt, c = x == 0 ? ct + 2 * bc : bc + 2 * ct;
                            blk[2 * (2 * rt + ct)] = o4[2 * (4 * r + c)];
                            blk[2 * (2 * rt + ct) + 1] = o4[2 * (4 * r + c) + 1];
                        }
                    double um[8];
                    as_matrix(u, um);
                    mat2_mul(blk, um, res);
                    for (int k = 0; k < 8; ++k) f.m[8 * bc + k] = res[k];
                }
                if (!(keep_real && op_is_real(u) && !op_is_real(f))) {
                    dead[last[op.q[x]]] = 1;
                    last[op.q[0]] = last[op.q[1]] = -1;
                    out.push_back(f);
                    dead.push_back(0);
                    continue;
                }
            }
        }
        if (two && last[op.q[0]] >= 0 && last[op.q[1]] >= 0) {
            const Op &u0 = out[last[op.q[0]]], &u1 = out[last[op.q[1]]];
            const bool dense = u0.kind == OP_DENSE1 && u1.kind == OP_DENSE1;
            const bool all_diag = diag(u0) && diag(u1) && (op.kind == OP_PHASE2 || op.kind == OP_DIAG2);
            if (dense || all_diag) {
                double a[8], b[8], o4[32], k4[32], m4[32];
                as_matrix(u0, a);
                as_matrix(u1, b);
                for (int r = 0; r < 4; ++r)   // k4 = U1 (x) U0 in index b0 + 2 b1
                    for (int c = 0; c < 4; ++c) {
                        const double ar = a[2 * (2 * (r & 1) + (c & 1))], ai = a[2 * (2 * (r & 1) + (c & 1)) + 1];
                        const double br = b[2 * (2 * (r >> 1) + (c >> 1))], bi = b[2 * (2 * (r >> 1) + (c >> 1)) + 1];
                        k4[2 * (4 * r + c)] = ar * br - ai * bi;
                        k4[2 * (4 * r + c) + 1] = ar * bi + ai * br;
                    }
                op_matrix4(op, o4);
                for (int r = 0; r < 4; ++r)   // m4 = o4 k4
                    for (int c = 0; c < 4; ++c) {
                        double re = 0, im = 0;
                        for (int k = 0; k < 4; ++k) {
                            const double xr = o4[2 * (4 * r + k)], xi = o4[2 * (4 * r + k) + 1];
                            const double yr = k4[2 * (4 * k + c)], yi = k4[2 * (4 * k + c) + 1];
                            re += xr * yr - xi * yi;
                            im += xr * yi + xi * yr;
                        }
                        m4[2 * (4 * r + c)] = re;
                        m4[2 * (4 * r + c) + 1] = im;
                    }
                Op f;
                std::memset(&f, 0, sizeof f);
                f.nq = 2;
                f.q[0] = op.q[0];
                f.q[1] = op.q[1];
                if (all_diag) {
                    f.kind = OP_DIAG2;
                    for (int k = 0; k < 4; ++k) {
                        f.m[2 * k] = m4[2 * (5 * k)];
                        f.m[2 * k + 1] = m4[2 * (5 * k) + 1];
                    }
                } else {
                    f.kind = OP_DENSE2;
                    std::memcpy(f.m, m4, sizeof m4);
                }
                if (keep_real && dense && op_is_real(u0) && op_is_real(u1) && !op_is_real(f)) {
                    // the real product of the two, then the op itself
                    std::memcpy(f.m, k4, sizeof k4);
                    dead[last[op.q[0]]] = dead[last[op.q[1]]] = 1;
                    last[op.q[0]] = last[op.q[1]] = -1;
                    out.push_back(f);
                    dead.push_back(0);
                    out.push_back(op);
                    dead.push_back(0);
                    continue;
                }
                dead[last[op.q[0]]] = dead[last[op.q[1]]] = 1;
                last[op.q[0]] = last[op.q[1]] = -1;
                out.push_back(f);
                dead.push_back(0);
                continue;
            }
        }
        for (int k = 0; k < op.nq; ++k) last[op.q[k]] = -1;
        out.push_back(op);
        dead.push_back(0);
        if (one_qubit(op)) last[op.q[0]] = (long)out.size() - 1;
    }
    std::vector<Op> kept;
    kept.reserve(out.size());
    for (size_t i = 0; i < out.size(); ++i)
        if (!dead[i]) kept.push_back(out[i]);
    ops.swap(kept);
}


// Gradient ops of a backward sweep move to the start of their qubit's run of
// one-qubit ops.  After ops U_1 .. U_k on that qubit (and any ops on other
// qubits, which commute with G), Im<lambda|G|psi> equals Im<lambda|G'|psi>
// before them with G' = P^dag G P, P = U_k ... U_1: a traceless Hermitian
// a X + b Y + c Z (gen 4, a, b, c in m[2..4]).  The run's ops then follow
// one another and merge_one_qubit_runs multiplies them into one.
void hoist_gradients(std::vector<Op> &ops, int n) {
    const size_t N = ops.size();
    std::vector<long> start(n, -1);
    std::vector<std::array<double, 8>> P(n);
    std::vector<long> target(N, -1);
    std::vector<Op> moved(ops);
    for (size_t i = 0; i < N; ++i) {
        const Op &op = ops[i];
        if (op.kind == OP_GRAD) {
            const int q = op.q[0];
            if (start[q] < 0) continue;
            target[i] = start[q];
            double g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            const int gen = (int)op.m[0];
            if (gen == 1) { g[2] = 1; g[4] = 1; }
            else if (gen == 2) { g[3] = -1; g[5] = 1; }
            else if (gen == 3) { g[0] = 1; g[6] = -1; }
            else { g[2] = op.m[2]; g[3] = -op.m[3]; g[4] = op.m[2]; g[5] = op.m[3]; g[0] = op.m[4]; g[6] = -op.m[4]; }
            double pd[8], t[8], gp[8];
            const auto &pm = P[q];
            for (int r = 0; r < 2; ++r)   // P^dag
                for (int c = 0; c < 2; ++c) {
                    pd[2 * (2 * r + c)] = pm[2 * (2 * c + r)];
                    pd[2 * (2 * r + c) + 1] = -pm[2 * (2 * c + r) + 1];
                }
            double pa[8];
            for (int k = 0; k < 8; ++k) pa[k] = pm[k];
            mat2_mul(pd, g, t);
            mat2_mul(t, pa, gp);
            Op &h = moved[i];
            h.m[0] = 4;
            h.m[2] = gp[4];   // a = Re G'10
            h.m[3] = gp[5];   // b = Im G'10
            h.m[4] = gp[0];   // c = Re G'00
            continue;
        }
        if (one_qubit(op)) {
            const int q = op.q[0];
            double u[8], z[8];
            as_matrix(op, u);
            if (start[q] < 0) {
                start[q] = (long)i;
                for (int k = 0; k < 8; ++k) P[q][k] = u[k];
            } else {
                double pm[8];
                for (int k = 0; k < 8; ++k) pm[k] = P[q][k];
                mat2_mul(u, pm, z);
                for (int k = 0; k < 8; ++k) P[q][k] = z[k];
            }
            continue;
        }
        const int nq = op.kind == OP_PERM ? n : op.nq;
        for (int k = 0; k < nq; ++k) start[op.kind == OP_PERM ? k : op.q[k]] = -1;
    }
    std::vector<Op> out;
    out.reserve(N);
    std::vector<std::vector<size_t>> before(N);
    for (size_t i = 0; i < N; ++i)
        if (target[i] >= 0) before[target[i]].push_back(i);
    for (size_t i = 0; i < N; ++i) {
        for (size_t j : before[i]) out.push_back(moved[j]);
        if (target[i] < 0) out.push_back(ops[i]);
    }
    ops.swap(out);
}

// Two gradient ops on the same qubit at the same point (next to each other
// after hoist_gradients) share one sweep over the register pairs: gen 5
// holds both generators, a1 b1 c1 in m[2..4] and a2 b2 c2 in m[5..7], the
// second parameter index in m[8].
void pair_gradients(std::vector<Op> &ops) {
    auto abc = [](const Op &g, double *o) {
        const int gen = (int)g.m[0];
        o[0] = gen == 1 ? 1 : gen == 4 ? g.m[2] : 0;
        o[1] = gen == 2 ? 1 : gen == 4 ? g.m[3] : 0;
        o[2] = gen == 3 ? 1 : gen == 4 ? g.m[4] : 0;
    };
    std::vector<Op> out;
    out.reserve(ops.size());
    for (size_t i = 0; i < ops.size(); ++i) {
        const Op &a = ops[i];
        if (a.kind == OP_GRAD && (int)a.m[0] <= 4 && i + 1 < ops.size()) {
            const Op &b = ops[i + 1];
            if (b.kind == OP_GRAD && (int)b.m[0] <= 4 && b.q[0] == a.q[0]) {
                Op p = a;
                double x[3], y[3];
                abc(a, x);
                abc(b, y);
                p.m[0] = 5;
                for (int k = 0; k < 3; ++k) {
                    p.m[2 + k] = x[k];
                    p.m[5 + k] = y[k];
                }
                p.m[8] = b.aux;
                out.push_back(p);
                ++i;
                continue;
            }
        }
        out.push_back(a);
    }
    ops.swap(out);
}

// VSWAP_k_k as a relabelling of qubits.  The reference moves amplitudes for
// every VSWAP (src/MEM_Runner.cpp:146-167).  Here a VSWAP (and, with swaps
// set, a SWAP gate too) only swaps entries of bit_of (bit position of the
// circuit -> bit of the stored state), and the ops after it are renamed
// through that map.  At the end the stored
// state is brought into the circuit's layout by at most two rounds of
// disjoint bit swaps: any permutation is the product of two involutions.
// The content of stored bit x_i moves to x_{i+1} around each cycle
// x_0 -> x_1 -> ... -> x_{m-1}; that is the reflection x_i <-> x_{1-i}
// applied after the reflection x_i <-> x_{-i} (indices mod m).  Each round
// becomes OP_PERM ops of at most max_pairs pairs whose bits, with the low L
// state bits, fit max_bits tile bits, so that they run as tile passes.
static bool renamable(const Op &op, bool swaps) {
    return op.kind == OP_PERM || (op.kind == OP_SWAP2 && (swaps || op.aux == 1));
}

void relabel_perms(std::vector<Op> &ops, int n, int L, int max_bits, int max_pairs, bool swaps) {
    bool any = false;
    for (const Op &op : ops) any = any || renamable(op, swaps);
    if (!any) return;
    std::vector<int> bit_of(n);
    for (int p = 0; p < n; ++p) bit_of[p] = p;
    std::vector<Op> out;
    out.reserve(ops.size() + 4);
    for (const Op &op : ops) {
        if (renamable(op, swaps)) {
            const int k = op.nq / 2;
            for (int i = 0; i < k; ++i) std::swap(bit_of[op.q[i]], bit_of[op.q[k + i]]);
            continue;
        }
        Op r = op;
        for (int j = 0; j < r.nq; ++j) r.q[j] = bit_of[r.q[j]];
        out.push_back(r);
    }
    std::vector<int> to(n);   // content of stored bit x moves to bit to[x]
    for (int p = 0; p < n; ++p) to[bit_of[p]] = p;
    std::vector<std::pair<int, int>> rounds[2];
    std::vector<char> seen(n, 0);
    for (int s = 0; s < n; ++s) {
        if (seen[s] || to[s] == s) continue;
        std::vector<int> x;
        for (int c = s; !seen[c]; c = to[c]) {
            seen[c] = 1;
            x.push_back(c);
        }
        const int m = (int)x.size();
        for (int i = 1; i < m - i; ++i) rounds[0].push_back({x[i], x[m - i]});
        for (int j = 0; j < m; ++j) {
            const int pj = (m + 1 - j) % m;
            if (j < pj) rounds[1].push_back({x[j], x[pj]});
        }
    }
    for (auto &pairs : rounds) {
        std::vector<char> used(pairs.size(), 0);
        size_t left = pairs.size();
        while (left) {
            std::vector<char> bits(n, 0);
            int nbits = 0;
            for (int q = 0; q < std::min(n, L); ++q) bits[q] = 1, ++nbits;
            Op op;
            std::memset(&op, 0, sizeof op);
            op.kind = OP_PERM;
            op.aux = 1;
            std::vector<std::pair<int, int>> take;
            for (size_t i = 0; i < pairs.size() && (int)take.size() < max_pairs; ++i) {
                if (used[i]) continue;
                const int add = !bits[pairs[i].first] + !bits[pairs[i].second];
                if (!take.empty() && nbits + add > max_bits) continue;
                bits[pairs[i].first] = bits[pairs[i].second] = 1;
                nbits += add;
                take.push_back(pairs[i]);
                used[i] = 1;
                --left;
            }
            const int k = (int)take.size();
            op.nq = 2 * k;
            for (int i = 0; i < k; ++i) {
                op.q[i] = take[i].first;
                op.q[k + i] = take[i].second;
            }
            out.push_back(op);
        }
    }
    ops.swap(out);
}

}  // namespace qk
