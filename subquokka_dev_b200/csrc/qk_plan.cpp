// Host planner for fused passes.
//
// The reference gets its speed from cache blocking: subcircuitFinder groups
// gates whose qubits all sit inside a 2^12-amplitude chunk and inserts VSWAPs
// to bring other qubits into the chunk (subcircuitFinder/finder.cpp:629-698),
// and MEM_Runner applies each group chunk by chunk while it is cache-resident
// (src/MEM_Runner.cpp:172-183).  Here the chunk is a tile of 2^T amplitudes
// whose index bits can be ANY T qubits (the low ones for coalescing plus the
// ones the gates need), so no VSWAP is needed: a pass gathers the strided
// amplitude sets of its tiles straight from HBM.  VSWAPs that a circuit (a
// subcircuit file) does contain become renamings (relabel_perms).
//
// build_plan: greedy passes.  Walk the remaining gates in order; a gate joins
// the current pass if none of its qubits is blocked (an earlier gate on that
// qubit was left out) and, unless it is diagonal, its qubits fit in the tile
// bit set; otherwise its qubits become blocked.  Diagonal gates (Z, P, RZ, CP,
// RZZ) join any pass: a qubit outside the tile is constant over a tile.
//
// compile_pass: each thread holds 2^r amplitudes indexed by r "register" tile
// bits.  Ready gates (all earlier gates on their qubits done) run while their
// qubits are register bits; diagonal gates run at any time; when no ready gate
// can run the tile is re-distributed through shared memory (TOP_REMAP) so that
// the qubits of the next ready gates become register bits.
#include <algorithm>
#include <complex>
#include <array>
#include <cstdint>
#include <cstring>
#include <vector>

#include "qk_internal.h"

namespace qk {

PlanOptions default_plan_options(int dtype, int n) {
    PlanOptions o;
    o.dtype = dtype;
    // 2048-amplitude tiles, 16 amplitudes a thread (128 threads).  complex128:
    // 0.75 s on the 30-qubit random circuit against 0.87 s for (12, 3), the
    // per-op program overhead spread over more FP64 work.  complex64: more
    // passes than with 8192-amplitude tiles (31 against 21 on that circuit)
    // but shorter ones: 355 against 389 ms there, 3.73 against 3.99 s on the
    // 33-qubit 24-layer circuit, 181 against 185 ms on the 30-qubit QFT
    o.tile_bits = std::min(n, 11);
    o.reg_bits = std::min(o.tile_bits, 4);
    return o;
}

// Two-state (adjoint) passes.  complex128: small tiles, 256 amplitudes with
// 8 a thread, so that many CTAs share an SM; on the 26-qubit HEA (12 layers,
// 624 parameters) 178 ms against 183 ms with 1024-amplitude tiles and 190 ms
// with 2048.  complex64: 2048-amplitude tiles with 16 amplitudes of each
// state a thread (254 registers), 106.5 ms there against 113 ms with 512-
// amplitude tiles and 8 a thread, 109 / 111 ms with 1024 / 4096 and 16.
PlanOptions default_adjoint_options(int dtype, int n) {
    PlanOptions o;
    o.dtype = dtype;
    o.tile_bits = std::min(n, dtype == QK_C128 ? 8 : 11);
    o.reg_bits = std::min(o.tile_bits, dtype == QK_C128 ? 3 : 4);
    return o;
}

namespace {

int low_bits(int dtype) { return dtype == QK_C128 ? 3 : 4; }  // 128-byte runs

// Most tile bits of a permutation pass (qk_pass.cu stages such a tile in
// shared memory in one buffer).
int perm_tile_bits(int dtype) { return dtype == QK_C128 ? 13 : 14; }
constexpr int kPermMinTileBits = 10;

void push_c(HostPlan &p, double re, double im) {
    p.coef.push_back(re);
    p.coef.push_back(im);
}

// Shared-memory bytes a pass program may use: the kernel keeps the program
// and its coefficients next to the (double-buffered) tile.
size_t program_budget(int dtype, int T, int nstates) {
    const size_t tile = ((size_t)(dtype == QK_C128 ? 16 : 8) << T) * nstates;
    const size_t tiles = 2 * tile <= (200u << 10) ? 2 * tile : tile;
    const size_t avail = (220u << 10) - tiles;
    return std::min<size_t>(64u << 10, avail - (8u << 10));
}

// Bytes of program and coefficients one op adds (remaps: 25 % headroom).
size_t op_cost(const Op &op, int dtype) {
    const size_t c = dtype == QK_C128 ? 16 : 8;
    size_t ncoef = 4;
    if (op.kind == OP_DENSE2 || op.kind == OP_SWAP2 || op.kind == OP_CDENSE1) ncoef = 16;
    else if (op.kind == OP_PHASE1 || op.kind == OP_PHASE2) ncoef = 1;
    else if (op.kind == OP_CX) ncoef = 0;
    else if (op.kind == OP_GRAD) {
        // one double accumulator per gradient; a general generator takes two
        // coefficients, a pair of gradients four
        const int gen = (int)op.m[0];
        return (16 + (gen == 5 ? 16 + 4 * c : gen == 4 ? 8 + 2 * c : 8)) * 5 / 4;
    }
    return (16 + ncoef * c) * 5 / 4;
}

struct PassBuilder {
    const std::vector<Op> &ops;
    int n, T, r, L;
    HostPlan &plan;
    int grad_base = 0;  // first gradient slot of the pass being compiled
    // tile bits of a pass: false, as the ops in order need them; true, grown
    // ahead by the qubit that lets the most pending ops join
    bool lookahead = false;
    // diagonal ops with a qubit in a register slot wait for a re-mapping that
    // takes it out (there they cost one multiply a thread, in a slot one
    // for half or all of the thread's amplitudes), unless the op after them
    // on one of their qubits could run now
    bool defer_diagonals = false;
    // no TOP_R1 / TOP_R2 and no pass marked xops
    bool plain_ops = false;

    // Emit a pass over tile bits B running ops[idx] (in order, dependencies
    // already satisfied with respect to everything outside idx).
    int compile(const std::vector<int> &idx, std::vector<int> B) {
        std::sort(B.begin(), B.end());
        PassDesc d;
        std::memset(&d, 0, sizeof d);
        d.T = (int)B.size();
        for (int k = 0; k < d.T; ++k) d.bpos[k] = B[k];
        d.L = 0;
        while (d.L < d.T && d.bpos[d.L] == d.L) ++d.L;
        std::vector<int> local(n, -1);
        for (int k = 0; k < d.T; ++k) local[B[k]] = k;
        d.prog0 = (int)plan.ops.size();
        d.coef0 = (int)(plan.coef.size() / 2);
        d.grad0 = (int)plan.grad_params.size();
        grad_base = d.grad0;

        // per-qubit queues of the pass's ops (positions in idx)
        std::vector<std::vector<int>> queue(n);
        for (size_t i = 0; i < idx.size(); ++i)
            for (int k = 0; k < ops[idx[i]].nq; ++k) queue[ops[idx[i]].q[k]].push_back((int)i);
        std::vector<size_t> head(n, 0);
        std::vector<char> done(idx.size(), 0);
        auto ready = [&](size_t i) {
            const Op &op = ops[idx[i]];
            for (int k = 0; k < op.nq; ++k)
                if (queue[op.q[k]][head[op.q[k]]] != (int)i) return false;
            return true;
        };
        std::vector<int> Q;  // register slot -> tile-local bit
        auto in_regs = [&](int lq) { return std::find(Q.begin(), Q.end(), lq) != Q.end(); };
        auto runnable = [&](const Op &op) {
            bool ok = true;
            for (int k = op_reg_first(op); k < op_reg_first(op) + op_reg_count(op); ++k)
                ok = ok && in_regs(local[op.q[k]]);
            return ok;
        };
        auto in_slot = [&](const Op &op) {
            for (int k = 0; k < op.nq; ++k)
                if (local[op.q[k]] >= 0 && in_regs(local[op.q[k]])) return true;
            return false;
        };
        auto unblocks = [&](size_t i) {
            const Op &op = ops[idx[i]];
            for (int k = 0; k < op.nq; ++k) {
                const std::vector<int> &qq = queue[op.q[k]];
                const size_t h = head[op.q[k]] + 1;
                if (h < qq.size() && !op_is_diagonal(ops[idx[qq[h]]]) && runnable(ops[idx[qq[h]]])) return true;
            }
            return false;
        };
        size_t ndone = 0;
        bool mapped = false, flush = false;
        size_t done_at_remap = (size_t)-1;
        while (ndone < idx.size()) {
            bool progress = true;
            while (progress) {
                progress = false;
                for (size_t i = 0; i < idx.size(); ++i) {
                    if (done[i] || !ready(i)) continue;
                    const Op &op = ops[idx[i]];
                    if (!mapped) continue;  // the first program op is always a TOP_REMAP
                    if (!runnable(op)) continue;
                    if (defer_diagonals && !flush && op_is_diagonal(op) && in_slot(op) && !unblocks(i)) continue;
                    emit(op, local, Q);
                    done[i] = 1;
                    ++ndone;
                    for (int k = 0; k < op.nq; ++k) ++head[op.q[k]];
                    progress = true;
                }
            }
            if (ndone == idx.size()) break;
            if (defer_diagonals && !flush && mapped) {
                // waiting diagonal ops run now when only diagonal ops are
                // left or the last re-mapping ran nothing
                bool other = false;
                for (size_t i = 0; i < idx.size() && !other; ++i) other = !done[i] && !op_is_diagonal(ops[idx[i]]);
                if (!other || ndone == done_at_remap) {
                    flush = true;
                    continue;
                }
            }
            flush = false;
            if (mapped && ndone == done_at_remap)
                return fail(QK_ERR_ARG, "planner: a gate cannot be made register-resident (reg_bits %d)", r);
            done_at_remap = ndone;
            // re-map: qubits of ready non-diagonal gates first, then of the
            // following non-diagonal gates in program order
            std::vector<int> nq;
            auto add = [&](const Op &op) {
                const int k0 = op_reg_first(op), k1 = k0 + op_reg_count(op);
                int need = 0;
                for (int k = k0; k < k1; ++k)
                    if (std::find(nq.begin(), nq.end(), local[op.q[k]]) == nq.end()) ++need;
                if ((int)nq.size() + need > r) return;
                for (int k = k0; k < k1; ++k)
                    if (std::find(nq.begin(), nq.end(), local[op.q[k]]) == nq.end()) nq.push_back(local[op.q[k]]);
            };
            for (size_t i = 0; i < idx.size() && (int)nq.size() < r; ++i)
                if (!done[i] && ready(i) && op_reg_count(ops[idx[i]])) add(ops[idx[i]]);
            for (size_t i = 0; i < idx.size() && (int)nq.size() < r; ++i)
                if (!done[i] && op_reg_count(ops[idx[i]])) add(ops[idx[i]]);
            for (int b = 0; b < d.T && (int)nq.size() < r; ++b)
                if (std::find(nq.begin(), nq.end(), b) == nq.end()) nq.push_back(b);
            if (nq.empty()) return fail(QK_ERR_ARG, "planner: no register qubits for a pass");
            Q = nq;
            TOp t;
            std::memset(&t, 0, sizeof t);
            t.kind = TOP_REMAP;
            t.nbits = (uint8_t)r;
            for (int s = 0; s < r; ++s) t.bits[s] = (uint8_t)Q[s];
            plan.ops.push_back(t);
            ++plan.nremaps;
            mapped = true;
        }
        d.nprog = (int)plan.ops.size() - d.prog0;
        d.ncoef = (int)(plan.coef.size() / 2) - d.coef0;
        for (int i = d.prog0; i < d.prog0 + d.nprog && !plain_ops; ++i) {
            const int k = plan.ops[i].kind;
            d.xops |= k == TOP_R1 || k == TOP_R2 || k == TOP_DIAG || k == TOP_PHASE;
        }
        d.ngrad = (int)plan.grad_params.size() - d.grad0;
        // program coefficient indices relative to the pass's slice
        for (int i = d.prog0; i < d.prog0 + d.nprog; ++i)
            if (plan.ops[i].kind != TOP_REMAP) plan.ops[i].coef -= (uint32_t)d.coef0;
        plan.passes.push_back(d);
        plan.ngates += idx.size();
        return QK_OK;
    }

    uint8_t code(int q, const std::vector<int> &local) {
        return local[q] >= 0 ? (uint8_t)local[q] : (uint8_t)(kOuterFlag | q);
    }

    void emit(const Op &op, const std::vector<int> &local, const std::vector<int> &Q) {
        TOp t;
        std::memset(&t, 0, sizeof t);
        t.coef = (uint32_t)(plan.coef.size() / 2);
        auto slot = [&](int q) { return (int)(std::find(Q.begin(), Q.end(), local[q]) - Q.begin()); };
        switch (op.kind) {
        case OP_DENSE1:
            t.a = (uint8_t)slot(op.q[0]);
            if (!plain_ops && op_is_real(op)) {
                t.kind = TOP_R1;
                push_c(plan, op.m[0], op.m[2]);
                push_c(plan, op.m[4], op.m[6]);
                break;
            }
            t.kind = TOP_G1;
            for (int k = 0; k < 4; ++k) push_c(plan, op.m[2 * k], op.m[2 * k + 1]);
            break;
        case OP_GRAD: {
            // gradient slot of the pass in bits[0..1]; a general generator
            // (gen 4) as coefficients (a, b), (c, 0)
            t.kind = TOP_GRAD;
            t.a = (uint8_t)slot(op.q[0]);
            t.b = (uint8_t)op.m[0];
            int k = grad_base;
            while (k < (int)plan.grad_params.size() && plan.grad_params[k] != op.aux) ++k;
            if (k == (int)plan.grad_params.size()) plan.grad_params.push_back(op.aux);
            t.bits[0] = (uint8_t)((k - grad_base) & 0xFF);
            t.bits[1] = (uint8_t)((k - grad_base) >> 8);
            if (t.b == 4 || t.b == 5) {
                push_c(plan, op.m[2], op.m[3]);
                push_c(plan, op.m[4], 0);
            }
            if (t.b == 5) {   // the second gradient of the pair
                const int32_t p2 = (int32_t)op.m[8];
                int k2 = grad_base;
                while (k2 < (int)plan.grad_params.size() && plan.grad_params[k2] != p2) ++k2;
                if (k2 == (int)plan.grad_params.size()) plan.grad_params.push_back(p2);
                t.bits[2] = (uint8_t)((k2 - grad_base) & 0xFF);
                t.bits[3] = (uint8_t)((k2 - grad_base) >> 8);
                push_c(plan, op.m[5], op.m[6]);
                push_c(plan, op.m[7], 0);
            }
            break;
        }
        case OP_DENSE2:
        case OP_SWAP2: {
            double m[32];
            if (op.kind == OP_DENSE2) std::memcpy(m, op.m, sizeof m);
            else {
                std::memset(m, 0, sizeof m);
                const int perm[4] = {0, 2, 1, 3};
                for (int i = 0; i < 4; ++i) m[2 * (4 * perm[i] + i)] = 1.0;
            }
            int sa = slot(op.q[0]), sb = slot(op.q[1]);
            bool real = !plain_ops;
            for (int k = 0; k < 16; ++k) real = real && m[2 * k + 1] == 0.0;
            t.kind = real ? TOP_R2 : TOP_G2;
            // index bit 0 must be the lower slot: swap the two index bits
            auto sw = [&](int i) { return sa < sb ? i : ((i & 1) << 1) | ((i >> 1) & 1); };
            t.a = (uint8_t)std::min(sa, sb);
            t.b = (uint8_t)std::max(sa, sb);
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; j += real ? 2 : 1) {
                    const int k = 4 * sw(i) + sw(j);
                    if (real) push_c(plan, m[2 * k], m[2 * (4 * sw(i) + sw(j + 1))]);
                    else push_c(plan, m[2 * k], m[2 * k + 1]);
                }
            break;
        }
        case OP_CX:
            t.kind = TOP_CX;
            t.a = (uint8_t)slot(op.q[1 - op.aux]);
            t.b = code(op.q[op.aux], local);
            break;
        case OP_CDENSE1: {
            // condition in a register slot here: the block-diagonal 4 x 4
            // (index b(target) + 2 b(condition)); otherwise the condition is
            // the same for all of a thread's amplitudes and TOP_CG1 picks one
            // of the two 2x2 matrices
            if (local[op.q[1]] >= 0 && slot(op.q[1]) < (int)Q.size()) {
                Op d;
                std::memset(&d, 0, sizeof d);
                d.kind = OP_DENSE2;
                d.nq = 2;
                d.q[0] = op.q[0];
                d.q[1] = op.q[1];
                for (int rc = 0; rc < 2; ++rc)
                    for (int rt = 0; rt < 2; ++rt)
                        for (int ct = 0; ct < 2; ++ct) {
                            const int k = 4 * (rt + 2 * rc) + (ct + 2 * rc);
                            d.m[2 * k] = op.m[8 * rc + 2 * (2 * rt + ct)];
                            d.m[2 * k + 1] = op.m[8 * rc + 2 * (2 * rt + ct) + 1];
                        }
                emit(d, local, Q);
                return;
            }
            t.kind = TOP_CG1;
            t.a = (uint8_t)slot(op.q[0]);
            t.b = code(op.q[1], local);
            for (int k = 0; k < 8; ++k) push_c(plan, op.m[2 * k], op.m[2 * k + 1]);
            break;
        }
        case OP_PHASE1:
            t.kind = TOP_PHASE;
            t.a = code(op.q[0], local);
            t.b = kNoQubit;
            push_c(plan, op.m[0], op.m[1]);
            break;
        case OP_DIAG1:
            t.kind = TOP_DIAG;
            t.a = code(op.q[0], local);
            t.b = kNoQubit;
            push_c(plan, op.m[0], op.m[1]); push_c(plan, op.m[2], op.m[3]); push_c(plan, 1, 0); push_c(plan, 1, 0);
            break;
        case OP_PHASE2:
            t.kind = TOP_PHASE;
            t.a = code(op.q[0], local);
            t.b = code(op.q[1], local);
            push_c(plan, op.m[0], op.m[1]);
            break;
        case OP_DIAG2:
            t.kind = TOP_DIAG;
            t.a = code(op.q[0], local);
            t.b = code(op.q[1], local);
            for (int k = 0; k < 4; ++k) push_c(plan, op.m[2 * k], op.m[2 * k + 1]);
            break;
        default:
            break;  // OP_PERM never reaches a compute pass
        }
        // condition qubits of DIAG / PHASE (a, b) and CX (b): their register
        // slot in bits[0] / bits[1] (kNoSlot when not register-resident), so
        // that the kernel need not search the current mapping
        if (t.kind == TOP_DIAG || t.kind == TOP_PHASE || t.kind == TOP_CX || t.kind == TOP_CG1) {
            auto slot_of = [&](uint8_t c) -> uint8_t {
                if (c == kNoQubit || (c & kOuterFlag)) return kNoSlot;
                const auto it = std::find(Q.begin(), Q.end(), (int)c);
                return it == Q.end() ? kNoSlot : (uint8_t)(it - Q.begin());
            };
            t.bits[0] = (t.kind == TOP_CX || t.kind == TOP_CG1) ? kNoSlot : slot_of(t.a);
            t.bits[1] = slot_of(t.b);
        }
        plan.ops.push_back(t);
    }

    // Permutation pass (VSWAP_k_k): tile bits = low bits + the swapped qubits.
    void perm_pass(const Op &op) {
        PassDesc d;
        std::memset(&d, 0, sizeof d);
        const int k = op.nq / 2;
        std::vector<char> in(n, 0);
        for (int i = 0; i < op.nq; ++i) in[op.q[i]] = 1;
        int cnt = op.nq;
        for (int q = 0; q < n && q < L; ++q)
            if (!in[q]) { in[q] = 1; ++cnt; }
        d.perm = 1;
        d.nperm = k;
        // a few more low bits than the swapped ones need: longer contiguous
        // runs per tile row (identity on those bits)
        for (int q = 0; q < n && cnt < kPermMinTileBits && cnt <= perm_tile_bits(plan.dtype); ++q)
            if (!in[q]) { in[q] = 1; ++cnt; }
        if (cnt > perm_tile_bits(plan.dtype)) {
            // too many qubits for one tile: flat in-place permutation sweep
            d.perm = 2;
            for (int i = 0; i < k; ++i) { d.perm_a[i] = op.q[i]; d.perm_b[i] = op.q[k + i]; }
            plan.passes.push_back(d);
            return;
        }
        std::vector<int> local(n, -1);
        int t = 0;
        for (int q = 0; q < n; ++q)
            if (in[q]) { local[q] = t; d.bpos[t++] = q; }
        d.T = t;
        while (d.L < d.T && d.bpos[d.L] == d.L) ++d.L;
        for (int i = 0; i < k; ++i) { d.perm_a[i] = local[op.q[i]]; d.perm_b[i] = local[op.q[k + i]]; }
        plan.passes.push_back(d);
        plan.ngates += 1;
    }

    // Fill B up to T bits: the low bits first, then the lowest unused qubits.
    void fill(std::vector<int> &B) {
        for (int q = 0; q < n && (int)B.size() < T; ++q)
            if (std::find(B.begin(), B.end(), q) == B.end()) B.push_back(q);
    }

    // Ops of `pending` that join a pass on tile bits inB (in order; an op
    // joins when no skipped op precedes it on a shared qubit, its register
    // qubits are tile bits and the program budget allows).
    size_t joins(const std::vector<size_t> &pending, const std::vector<char> &inB, size_t budget) const {
        std::vector<char> blocked(n, 0);
        size_t cnt = 0, used = 0;
        int nblocked = 0;
        for (size_t i : pending) {
            const Op &op = ops[i];
            bool ok = op.kind != OP_PERM && (cnt == 0 || used + op_cost(op, plan.dtype) <= budget);
            for (int k = 0; k < op.nq && ok; ++k) ok = !blocked[op.q[k]];
            for (int k = op_reg_first(op); k < op_reg_first(op) + op_reg_count(op) && ok; ++k) ok = inB[op.q[k]];
            if (ok) {
                ++cnt;
                used += op_cost(op, plan.dtype);
                continue;
            }
            for (int k = 0; k < op.nq; ++k)
                if (!blocked[op.q[k]]) blocked[op.q[k]] = 1, ++nblocked;
            if (nblocked == n) break;
        }
        return cnt;
    }

    // Tile bits grown ahead: the first pending op's register qubits, then one
    // at a time the qubit (of the next 64 pending ops) that lets the most
    // ops join; when none adds one, the lowest candidate.  The planners keep
    // it when it gives fewer passes: the 30-qubit brick circuit 26 passes
    // instead of 39 (643 against 679 ms c128, 411 against 441 ms c64).  On
    // the 26-qubit HEA forward pass (15 passes instead of 27) c128 took
    // 32 ms against 30 ms: fewer passes with more re-mappings each.
    void choose_tile(const std::vector<size_t> &pending, size_t budget, std::vector<int> &B) const {
        std::vector<char> inB(n, 0);
        for (int q : B) inB[q] = 1;
        const Op &first = ops[pending[0]];
        for (int k = op_reg_first(first); k < op_reg_first(first) + op_reg_count(first); ++k)
            if (!inB[first.q[k]] && (int)B.size() < T) inB[first.q[k]] = 1, B.push_back(first.q[k]);
        size_t base = joins(pending, inB, budget);
        while ((int)B.size() < T) {
            std::vector<int> cands;
            for (size_t j = 0; j < pending.size() && j < 64; ++j) {
                const Op &op = ops[pending[j]];
                for (int k = op_reg_first(op); k < op_reg_first(op) + op_reg_count(op); ++k)
                    if (!inB[op.q[k]]) cands.push_back(op.q[k]);
            }
            std::sort(cands.begin(), cands.end());
            cands.erase(std::unique(cands.begin(), cands.end()), cands.end());
            if (cands.empty()) break;
            int best = -1;
            size_t bestc = base;
            for (int q : cands) {
                inB[q] = 1;
                const size_t c = joins(pending, inB, budget);
                inB[q] = 0;
                if (c > bestc) best = q, bestc = c;
            }
            if (best < 0) best = cands[0], bestc = base;
            inB[best] = 1;
            B.push_back(best);
            base = bestc;
        }
    }

    // Greedy passes over ops[first..last).
    int greedy(size_t first, size_t last) {
        std::vector<size_t> pending;
        for (size_t i = first; i < last; ++i) pending.push_back(i);
        while (!pending.empty()) {
            if (ops[pending[0]].kind == OP_PERM) {
                perm_pass(ops[pending[0]]);
                pending.erase(pending.begin());
                continue;
            }
            std::vector<int> B;
            for (int q = 0; q < std::min(n, L); ++q) B.push_back(q);
            const size_t budget = program_budget(plan.dtype, T, plan.nstates);
            if (lookahead) choose_tile(pending, budget, B);
            std::vector<char> blocked(n, 0);
            std::vector<int> take;
            std::vector<size_t> rest;
            size_t used = 0;
            for (size_t i : pending) {
                const Op &op = ops[i];
                bool blk = false;
                for (int k = 0; k < op.nq; ++k) blk = blk || blocked[op.q[k]];
                bool ok = !blk && op.kind != OP_PERM && (take.empty() || used + op_cost(op, plan.dtype) <= budget);
                if (ok && op_reg_count(op)) {
                    const int k0 = op_reg_first(op), k1 = k0 + op_reg_count(op);
                    int need = 0;
                    for (int k = k0; k < k1; ++k)
                        if (std::find(B.begin(), B.end(), op.q[k]) == B.end()) ++need;
                    ok = (int)B.size() + need <= T;
                    if (ok)
                        for (int k = k0; k < k1; ++k)
                            if (std::find(B.begin(), B.end(), op.q[k]) == B.end()) B.push_back(op.q[k]);
                }
                if (ok) {
                    take.push_back((int)i);
                    used += op_cost(op, plan.dtype);
                } else {
                    for (int k = 0; k < op.nq; ++k) blocked[op.q[k]] = 1;
                    rest.push_back(i);
                }
            }
            fill(B);
            int rc = compile(take, B);
            if (rc) return rc;
            pending.swap(rest);
        }
        return QK_OK;
    }
};

int lower_all(const qk_gate *gates, size_t ng, int n, std::vector<Op> &ops) {
    ops.resize(ng);
    for (size_t i = 0; i < ng; ++i) {
        int rc = lower_gate(gates[i], ops[i]);
        if (rc) return rc;
        for (int k = 0; k < ops[i].nq; ++k)
            if (ops[i].q[k] < 0 || ops[i].q[k] >= n)
                return fail(QK_ERR_QUBIT, "gate %zu: qubit %d outside a %d-qubit state", i, ops[i].q[k], n);
    }
    return QK_OK;
}

// Leading state bits always in the tile; two tile bits stay free for the
// qubits of any single gate, so every pass takes at least one gate.
int pass_low_bits(const PlanOptions &o, int n) {
    if (o.tile_bits >= n) return std::min(n, low_bits(o.dtype));
    return std::max(0, std::min(low_bits(o.dtype), o.tile_bits - 2));
}

int check_options(const PlanOptions &o, int n) {
    if (o.dtype != QK_C128 && o.dtype != QK_C64) return fail(QK_ERR_ARG, "unknown dtype %d", o.dtype);
    if (o.tile_bits < 1 || o.tile_bits > std::min(n, kPassMaxBits))
        return fail(QK_ERR_ARG, "tile_bits must be in [1, min(n, %d)], got %d", kPassMaxBits, o.tile_bits);
    const int max_reg = 4;  // more register-resident amplitudes spill
    // two register bits at least: a two-qubit gate needs both of its qubits
    const int min_reg = std::min(2, o.tile_bits);
    if (o.reg_bits < min_reg || o.reg_bits > std::min(o.tile_bits, max_reg))
        return fail(QK_ERR_ARG, "reg_bits must be in [%d, min(tile_bits, %d)], got %d", min_reg, max_reg, o.reg_bits);
    if (o.tile_bits - o.reg_bits > 9)
        return fail(QK_ERR_ARG, "tile_bits - reg_bits must be <= 9 (512 threads), got %d", o.tile_bits - o.reg_bits);
    if (o.dtype == QK_C128 && o.reg_bits == 4 && o.tile_bits - o.reg_bits > 8)   // 241 registers a thread
        return fail(QK_ERR_ARG, "complex128 with reg_bits 4 needs tile_bits - reg_bits <= 8 (256 threads)");
    const size_t bytes = (o.dtype == QK_C128 ? 16 : 8) << o.tile_bits;
    if (bytes > (200u << 10)) return fail(QK_ERR_ARG, "tile of %zu bytes exceeds shared memory", bytes);
    return QK_OK;
}

}  // namespace

int build_plan(const qk_gate *gates, size_t ng, int n, const PlanOptions &o, HostPlan &plan) {
    int rc = check_options(o, n);
    if (rc) return rc;
    std::vector<Op> lowered;
    rc = lower_all(gates, ng, n, lowered);
    if (rc) return rc;
    // VSWAPs are always renamings.  SWAP gates are too when that gives fewer
    // passes: their renaming removes them from the compute passes but can
    // leave a longer permutation to restore at the end.
    // The greedy planner follows list order: the list as given and its ASAP
    // layering are both planned (2 ms for 900 gates), the one with fewer
    // passes is kept.
    bool swaps = false;
    for (const Op &op : lowered) swaps = swaps || (op.kind == OP_SWAP2 && op.aux != 1);
    for (int variant = 0; variant < (swaps ? 8 : 4); ++variant) {
        std::vector<Op> ops = lowered;
        relabel_perms(ops, n, pass_low_bits(o, n), perm_tile_bits(o.dtype), 6, variant >= 4);
        merge_one_qubit_runs(ops, n);
        // real one-qubit ops stay real (TOP_R1 / TOP_R2 take half the
        // multiply-adds of complex ones): the 30-qubit QFT 228 -> 219 ms
        // complex128, 166 -> 163 ms complex64
        absorb_into_two_qubit_ops(ops, n, !o.plain_ops);
        if (variant % 2) asap_order(ops, n);
        HostPlan hp;
        hp.n = n;
        hp.dtype = o.dtype;
        hp.T = o.tile_bits;
        hp.r = o.reg_bits;
        PassBuilder b{ops, n, o.tile_bits, o.reg_bits, pass_low_bits(o, n), hp};
        b.lookahead = (variant >> 1) & 1;
        // diagonal ops wait for their qubits to leave the register slots
        // where the kernel carries a pending scalar (the 30-qubit QFT 163 ->
        // 159 ms complex64; complex128 with 16 register amplitudes keeps
        // none, and the extra re-mappings cost 219 -> 224 ms)
        b.plain_ops = o.plain_ops != 0;
        b.defer_diagonals = !o.plain_ops && pending_scalar_ok(o.dtype == QK_C128 ? 16 : 8, 1 << o.reg_bits, 1);
        rc = b.greedy(0, ops.size());
        if (rc) return rc;
        if (variant == 0 || hp.passes.size() < plan.passes.size() ||
            (hp.passes.size() == plan.passes.size() && hp.ops.size() < plan.ops.size()))
            plan = std::move(hp);
    }
    return QK_OK;
}

int build_perm_plan(const Op &op, int n, const PlanOptions &o, HostPlan &plan) {
    if (op.kind != OP_PERM || op.nq < 2 || op.nq % 2 || op.nq > 12)
        return fail(QK_ERR_ARG, "not a permutation of 1 to 6 bit pairs");
    for (int i = 0; i < op.nq; ++i)
        if (op.q[i] < 0 || op.q[i] >= n) return fail(QK_ERR_QUBIT, "qubit %d outside a %d-qubit state", op.q[i], n);
    int rc = check_options(o, n);
    if (rc) return rc;
    std::vector<Op> ops{op};
    plan = HostPlan();
    plan.n = n;
    plan.dtype = o.dtype;
    plan.T = o.tile_bits;
    plan.r = o.reg_bits;
    PassBuilder b{ops, n, o.tile_bits, o.reg_bits, pass_low_bits(o, n), plan};
    b.perm_pass(op);
    return QK_OK;
}

int build_adjoint_plan(const qk_gate *gates, size_t ng, const int32_t *pidx, int n, const PlanOptions &o,
                       HostPlan &plan) {
    int rc = check_options(o, n);
    if (rc) return rc;
    if (o.reg_bits > (o.dtype == QK_C64 ? 4 : 3))
        return fail(QK_ERR_ARG, "adjoint passes take at most %d register bits (two states a thread)",
                    o.dtype == QK_C64 ? 4 : 3);
    if (o.dtype == QK_C128 && o.reg_bits == 3 && o.tile_bits - o.reg_bits > 8)
        return fail(QK_ERR_ARG, "complex128 adjoint passes with reg_bits 3 need tile_bits - reg_bits <= 8");
    std::vector<Op> fwd;
    rc = lower_all(gates, ng, n, fwd);
    if (rc) return rc;
    std::vector<Op> ops;
    ops.reserve(2 * ng);
    for (size_t i = ng; i-- > 0;) {
        Op op = fwd[i];
        if (pidx && pidx[i] >= 0) {
            const int gen = gates[i].kind == QK_GATE_RX ? 1 : gates[i].kind == QK_GATE_RY ? 2 : gates[i].kind == QK_GATE_RZ ? 3 : 0;
            if (!gen) return fail(QK_ERR_UNSUPPORTED, "gate %zu: only RX, RY, RZ are trainable", i);
            Op g;
            std::memset(&g, 0, sizeof g);
            g.kind = OP_GRAD;
            g.nq = 1;
            g.q[0] = op.q[0];
            g.m[0] = gen;
            g.aux = pidx[i];
            ops.push_back(g);
        }
        invert_op(op);
        ops.push_back(op);
    }
    hoist_gradients(ops, n);
    merge_one_qubit_runs(ops, n);
    absorb_into_two_qubit_ops(ops, n);
    pair_gradients(ops);
    // A gradient op only needs the ops on its own qubit in order: ops on
    // other qubits act on both states alike and commute with G.  So the
    // backward list may be layered too; the order with fewer passes is kept.
    for (int variant = 0; variant < 4; ++variant) {
        std::vector<Op> list = ops;
        if (variant % 2) asap_order(list, n);
        HostPlan hp;
        hp.n = n;
        hp.dtype = o.dtype;
        hp.T = o.tile_bits;
        hp.r = o.reg_bits;
        hp.nstates = 2;
        PassBuilder b{list, n, o.tile_bits, o.reg_bits, pass_low_bits(o, n), hp};
        b.lookahead = variant >= 2;
        b.plain_ops = o.plain_ops != 0;
        rc = b.greedy(0, list.size());
        if (rc) return rc;
        if (variant == 0 || hp.passes.size() < plan.passes.size() ||
            (hp.passes.size() == plan.passes.size() && hp.ops.size() < plan.ops.size()))
            plan = std::move(hp);
    }
    return QK_OK;
}

// Apply a lowered op (dense matrix over its targets, little-endian) to the
// 64 columns of a 6-qubit block unitary in place; loc[k] = local bit of op.q[k].
static void block_apply(std::vector<double> &u, const Op &op, const int *loc) {
    const int nq = op.nq, d = 1 << nq;
    double m[2 * 16 * 16];
    std::memset(m, 0, sizeof m);
    auto put = [&](int r, int c, double re, double im) { m[2 * (r * d + c)] = re; m[2 * (r * d + c) + 1] = im; };
    switch (op.kind) {
    case OP_DENSE1: case OP_DENSE2:
        for (int k = 0; k < d * d; ++k) put(k / d, k % d, op.m[2 * k], op.m[2 * k + 1]);
        break;
    case OP_PHASE1: put(0, 0, 1, 0); put(1, 1, op.m[0], op.m[1]); break;
    case OP_DIAG1: put(0, 0, op.m[0], op.m[1]); put(1, 1, op.m[2], op.m[3]); break;
    case OP_PHASE2: for (int k = 0; k < 3; ++k) put(k, k, 1, 0); put(3, 3, op.m[0], op.m[1]); break;
    case OP_DIAG2: for (int k = 0; k < 4; ++k) put(k, k, op.m[2 * k], op.m[2 * k + 1]); break;
    case OP_SWAP2: put(0, 0, 1, 0); put(1, 2, 1, 0); put(2, 1, 1, 0); put(3, 3, 1, 0); break;
    case OP_CX:
        if (op.aux == 0) { put(0, 0, 1, 0); put(3, 1, 1, 0); put(2, 2, 1, 0); put(1, 3, 1, 0); }
        else { put(0, 0, 1, 0); put(1, 1, 1, 0); put(3, 2, 1, 0); put(2, 3, 1, 0); }
        break;
    default: return;
    }
    int mask = 0;
    for (int k = 0; k < nq; ++k) mask |= 1 << loc[k];
    for (int col = 0; col < kDenseDim; ++col) {
        double *v = u.data() + 2 * col;  // column col: element (row r) at 2 * (r * 64 + col)
        for (int base = 0; base < kDenseDim; ++base) {
            if (base & mask) continue;
            int idx[16];
            double xr[16], xi[16];
            for (int s = 0; s < d; ++s) {
                int r = base;
                for (int k = 0; k < nq; ++k)
                    if ((s >> k) & 1) r |= 1 << loc[k];
                idx[s] = r;
                xr[s] = v[2 * r * kDenseDim];
                xi[s] = v[2 * r * kDenseDim + 1];
            }
            for (int r = 0; r < d; ++r) {
                double yr = 0, yi = 0;
                for (int c = 0; c < d; ++c) {
                    const double ar = m[2 * (r * d + c)], ai = m[2 * (r * d + c) + 1];
                    yr += ar * xr[c] - ai * xi[c];
                    yi += ar * xi[c] + ai * xr[c];
                }
                v[2 * idx[r] * kDenseDim] = yr;
                v[2 * idx[r] * kDenseDim + 1] = yi;
            }
        }
    }
}

// The block partition of an op list; with_u: also the blocks' unitaries.
static void dense_partition(const std::vector<Op> &ops, int n, int width, int nseeds, bool with_u,
                            std::vector<DenseBlock> &blocks) {
    blocks.clear();
    std::vector<size_t> pending(ops.size());
    for (size_t i = 0; i < ops.size(); ++i) pending[i] = i;
    while (!pending.empty()) {
        if (ops[pending[0]].kind == OP_PERM) {
            DenseBlock b;
            b.perm = 1;
            b.perm_op = ops[pending[0]];
            b.ngates = 1;
            blocks.push_back(std::move(b));
            pending.erase(pending.begin());
            continue;
        }
        // Block qubits: the first pending gate's, then, while fewer than
        // `width`, the qubit (among those of the next 64 pending gates,
        // ascending) that lets the most pending gates join.  A gate joins when
        // its qubits are block qubits and no earlier gate on them was left
        // out.  When no qubit adds a gate, the lowest candidate is taken
        // anyway (it can let a later two-qubit gate join).  On the random
        // circuits this gives about 40 % fewer blocks than taking gates in
        // order.
        std::vector<char> inQ(n, 0), blocked(n, 0);
        std::vector<int> Q;
        auto absorb = [&](int qsize, std::vector<size_t> *take, std::vector<size_t> *rest) {
            std::fill(blocked.begin(), blocked.end(), 0);
            size_t cnt = 0;
            int qblocked = 0;
            for (size_t i : pending) {
                const Op &op = ops[i];
                bool ok = op.kind != OP_PERM;
                for (int k = 0; k < op.nq && ok; ++k) ok = inQ[op.q[k]] && !blocked[op.q[k]];
                if (ok) {
                    ++cnt;
                    if (take) take->push_back(i);
                    continue;
                }
                for (int k = 0; k < op.nq; ++k)
                    if (!blocked[op.q[k]]) {
                        blocked[op.q[k]] = 1;
                        qblocked += inQ[op.q[k]];
                    }
                if (rest) rest->push_back(i);
                else if (qblocked == qsize) break;   // counting: nothing more can join
            }
            return cnt;
        };
        // grow a block from the qubits of seed op s
        auto grow = [&](const Op &s) {
            std::fill(inQ.begin(), inQ.end(), 0);
            Q.clear();
            for (int k = 0; k < s.nq; ++k)
                if (!inQ[s.q[k]]) {
                    inQ[s.q[k]] = 1;
                    Q.push_back(s.q[k]);
                }
            size_t base = absorb((int)Q.size(), nullptr, nullptr);
            while ((int)Q.size() < width) {
                std::vector<int> cands;
                for (size_t j = 0; j < pending.size() && j < 64; ++j)
                    for (int k = 0; k < ops[pending[j]].nq; ++k)
                        if (!inQ[ops[pending[j]].q[k]]) cands.push_back(ops[pending[j]].q[k]);
                std::sort(cands.begin(), cands.end());
                cands.erase(std::unique(cands.begin(), cands.end()), cands.end());
                if (cands.empty()) break;
                int best = -1;
                size_t bestc = base;
                for (int q : cands) {
                    inQ[q] = 1;
                    const size_t c = absorb((int)Q.size() + 1, nullptr, nullptr);
                    inQ[q] = 0;
                    if (c > bestc) { best = q; bestc = c; }
                }
                if (best < 0) {
                    best = cands[0];
                    inQ[best] = 1;
                    bestc = absorb((int)Q.size() + 1, nullptr, nullptr);
                    inQ[best] = 0;
                }
                inQ[best] = 1;
                Q.push_back(best);
                base = bestc;
            }
            return base;
        };
        // seeds: the first pending op, then up to nseeds - 1 more ready ops
        // (no earlier pending op on their qubits); the block that lets the
        // most ops join is kept
        size_t got = grow(ops[pending[0]]);
        if (nseeds > 1) {
            std::vector<int> bestQ = Q;
            std::vector<char> seen(n, 0);
            int tried = 1;
            for (int k = 0; k < ops[pending[0]].nq; ++k) seen[ops[pending[0]].q[k]] = 1;
            for (size_t j = 1; j < pending.size() && j < 256 && tried < nseeds; ++j) {
                const Op &op = ops[pending[j]];
                bool ready = op.kind != OP_PERM;
                for (int k = 0; k < op.nq; ++k) ready = ready && !seen[op.q[k]];
                for (int k = 0; k < op.nq; ++k) seen[op.q[k]] = 1;
                if (!ready) continue;
                ++tried;
                const size_t c = grow(op);
                if (c > got) {
                    got = c;
                    bestQ = Q;
                }
            }
            Q = bestQ;
            std::fill(inQ.begin(), inQ.end(), 0);
            for (int q : Q) inQ[q] = 1;
        }
        std::vector<size_t> take, rest;
        absorb((int)Q.size(), &take, &rest);
        // pad with the highest free qubits (identity on them): keeping the low
        // qubits out of a block keeps its tiles' other index contiguous
        for (int q = n - 1; q >= 0 && (int)Q.size() < kDenseQubits; --q)
            if (std::find(Q.begin(), Q.end(), q) == Q.end()) Q.push_back(q);
        std::sort(Q.begin(), Q.end());
        DenseBlock b;
        for (int k = 0; k < kDenseQubits; ++k) b.q[k] = Q[k];
        if (with_u) {
            b.u.assign(2 * kDenseDim * kDenseDim, 0.0);
            for (int k = 0; k < kDenseDim; ++k) b.u[2 * (k * kDenseDim + k)] = 1.0;
            for (size_t i : take) {
                int loc[QK_MAX_TARGETS];
                for (int k = 0; k < ops[i].nq; ++k)
                    loc[k] = (int)(std::find(Q.begin(), Q.end(), ops[i].q[k]) - Q.begin());
                block_apply(b.u, ops[i], loc);
            }
        }
        b.ngates = (int)take.size();
        blocks.push_back(std::move(b));
        pending.swap(rest);
    }
}

int build_dense_blocks(const qk_gate *gates, size_t ng, int n, int width, int dtype, std::vector<DenseBlock> &blocks) {
    if (n < kDenseQubits) return fail(QK_ERR_ARG, "dense blocks need at least %d qubits", kDenseQubits);
    if (width < 2 || width > kDenseQubits) return fail(QK_ERR_ARG, "block width must be in [2, %d], got %d", kDenseQubits, width);
    std::vector<Op> ops;
    int rc = lower_all(gates, ng, n, ops);
    if (rc) return rc;
    // at most three pairs per restoring permutation: a permutation block
    // lists its targets in kDenseQubits entries
    relabel_perms(ops, n, low_bits(dtype), perm_tile_bits(dtype), kDenseQubits / 2, false);
    // The fuser is greedy, and which greedy choice needs the fewest blocks
    // depends on the circuit: the list as given and its ASAP layering, each
    // with 1, 4 and 16 seed ops per block, are partitioned (block counts
    // only), and the best is built.  On the 30-qubit 20-layer random circuit
    // this gives 36 blocks instead of 39; on the 26-qubit HEA 35 instead of
    // 55 (the given order with one seed).
    std::vector<Op> layered = ops;
    asap_order(layered, n);
    const std::vector<Op> *best_list = &ops;
    int best_seeds = 1;
    size_t best = SIZE_MAX;
    std::vector<DenseBlock> trial;
    for (const std::vector<Op> *list : {&ops, &layered})
        for (int seeds : {1, 4, 16}) {
            dense_partition(*list, n, width, seeds, false, trial);
            if (trial.size() < best) {
                best = trial.size();
                best_list = list;
                best_seeds = seeds;
            }
        }
    dense_partition(*best_list, n, width, best_seeds, true, blocks);
    return QK_OK;
}

int build_group_plan(const qk_gate *gates, const int32_t *sizes, size_t ngroups, int n, const PlanOptions &o,
                     HostPlan &plan) {
    size_t ng = 0;
    for (size_t g = 0; g < ngroups; ++g) {
        if (sizes[g] < 0) return fail(QK_ERR_ARG, "group %zu has negative size", g);
        ng += (size_t)sizes[g];
    }
    // The groups bound nothing here: a tile can hold any qubits, and VSWAP
    // groups become renamings, so the gates of all groups are planned as one
    // gate list.
    return build_plan(gates, ng, n, o, plan);
}

}  // namespace qk
