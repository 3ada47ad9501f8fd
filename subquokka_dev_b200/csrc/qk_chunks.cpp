// Chunk grouping for the reference's subcircuit runner, and circuit files
// written back out.
//
// qk_circuit_chunk_groups does the job of subcircuitFinder
// (subcircuitFinder/finder.cpp:771-877) for any gate of the MEM grammar.  Its
// output is what MEM_Runner::run(vector<vector<Gate*>>&) needs
// (src/MEM_Runner.cpp:136-185):
// - a compute group is applied chunk by chunk, so every gate in it acts on
//   bit positions below chunk_qbit only;
// - a VSWAP group holds one `VSWAP_1_1 a c` or `VSWAP_2_2 a b c d` with
//   a < b < chunk_qbit <= c < d, exchanging position a with c and b with d.
//   These are the forms the finder writes (finder.cpp:239-260).
// Two-qubit gates keep ascending targets.  A U2 whose positions come out
// descending is written with its matrix in the swapped basis.
//
// Method: a layout pos[q] maps each qubit of the circuit to a bit position.
// Repeat:
// - One group takes, in order, every gate whose qubits all sit in the chunk
//   and which no skipped gate on a shared qubit precedes.
// - When the first remaining gate cannot run, the next chunk set is chosen
//   greedily: the qubits of that gate, then one qubit at a time the one that
//   lets the most remaining gates run, preferring qubits already in the
//   chunk.  The qubits of the new set outside the chunk are exchanged with
//   the chunk's qubits outside the set, in pairs as VSWAP_2_2 and an odd one
//   as VSWAP_1_1.  A qubit leaving the chunk goes, where it can, to the
//   outer position it must end at.  (On the 30-qubit QFT with 12-qubit
//   chunks: 45 VSWAPs with the final restore, against 52 without that
//   preference; the reference's own sub file for that circuit has 42 and
//   leaves the state in a permuted layout.)
// At the end the layout returns to the circuit's own: positions above the
// chunk by VSWAP exchanges, then positions inside it by SWAP gates.  VSWAP
// and SWAP gates of the input only rename the qubits of the gates after them.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "qk_internal.h"

namespace {

using qk::fail;

bool is_vswap(const qk_gate &g) { return g.kind == QK_GATE_VSWAP || g.kind == QK_GATE_MPI_VSWAP; }

struct Grouper {
    int n, c;
    std::vector<int> pos, at;   // qubit -> position, position -> qubit
    qk_circuit *out;
    std::vector<int> final_pos; // position each qubit must end at (empty: no preference)

    void put_vswap(int a, int b, int x, int y, int k) {
        qk_gate g;
        std::memset(&g, 0, sizeof g);
        g.kind = QK_GATE_VSWAP;
        g.nq = 2 * k;
        if (k == 1) {
            g.q[0] = a;
            g.q[1] = x;
        } else {
            g.q[0] = a; g.q[1] = b; g.q[2] = x; g.q[3] = y;
        }
        out->gates.push_back(g);
        out->group_sizes.push_back(1);
        for (int i = 0; i < k; ++i) {
            const int p = i ? b : a, r = i ? y : x;
            std::swap(at[p], at[r]);
            pos[at[p]] = p;
            pos[at[r]] = r;
        }
    }

    // Exchange the chunk positions `in` with the outer positions `ex` (same
    // count).  A qubit leaving the chunk goes, where it can, to the outer
    // position it must end at, so that the final restore has less to do;
    // a VSWAP_2_2 pairs its lower chunk position with its lower outer one.
    void exchange(std::vector<int> in, std::vector<int> ex) {
        std::sort(in.begin(), in.end());
        std::sort(ex.begin(), ex.end());
        std::vector<std::pair<int, int>> home;   // (chunk position, its qubit's final outer position)
        if (!final_pos.empty())
            for (int p : in) {
                const int t = final_pos[at[p]];
                const auto it = std::find(ex.begin(), ex.end(), t);
                if (it == ex.end()) continue;
                home.push_back({p, t});
                ex.erase(it);
            }
        for (const auto &h : home) in.erase(std::find(in.begin(), in.end(), h.first));
        // pairs of home moves in the same order share a VSWAP_2_2
        std::vector<std::pair<int, int>> single;
        for (size_t i = 0; i < home.size();) {
            if (i + 1 < home.size() && home[i + 1].second > home[i].second) {
                put_vswap(home[i].first, home[i + 1].first, home[i].second, home[i + 1].second, 2);
                i += 2;
            } else {
                single.push_back(home[i++]);
            }
        }
        // a single home move shares a VSWAP_2_2 with a free pair in the same order
        for (const auto &h : single) {
            bool done = false;
            for (size_t a = 0; a < in.size() && !done; ++a)
                for (size_t b = 0; b < ex.size() && !done; ++b)
                    if ((in[a] > h.first) == (ex[b] > h.second)) {
                        const bool lo = h.first < in[a];
                        put_vswap(lo ? h.first : in[a], lo ? in[a] : h.first, lo ? h.second : ex[b],
                                  lo ? ex[b] : h.second, 2);
                        in.erase(in.begin() + a);
                        ex.erase(ex.begin() + b);
                        done = true;
                    }
            if (!done) put_vswap(h.first, 0, h.second, 0, 1);
        }
        size_t i = 0;
        for (; i + 1 < in.size(); i += 2) put_vswap(in[i], in[i + 1], ex[i], ex[i + 1], 2);
        if (i < in.size()) put_vswap(in[i], 0, ex[i], 0, 1);
    }

    // A gate renamed to positions, targets ascending.
    qk_gate place(const qk_gate &g) const {
        qk_gate r = g;
        for (int j = 0; j < r.nq; ++j) r.q[j] = pos[g.q[j]];
        if (r.nq == 2 && r.q[0] > r.q[1]) {
            std::swap(r.q[0], r.q[1]);
            if (r.kind == QK_GATE_U2) {
                // basis index 2 * bit(first) + bit(second): swapping the
                // targets swaps the two index bits of rows and columns
                auto sw = [](int i) { return ((i & 1) << 1) | (i >> 1); };
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j) {
                        const int k = 4 * sw(i) + sw(j);
                        r.coeff[2 * (4 * i + j)] = g.coeff[2 * k];
                        r.coeff[2 * (4 * i + j) + 1] = g.coeff[2 * k + 1];
                    }
            }
        }
        return r;
    }
};

}  // namespace

extern "C" {

int qk_circuit_chunk_groups(const qk_gate *gates, size_t ng, int nqubits, int chunk_qbit, qk_circuit **out) {
    if (!out || (!gates && ng)) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 63) return fail(QK_ERR_ARG, "nqubits must be in [1, 63], got %d", nqubits);
    if (chunk_qbit < 1 || chunk_qbit > nqubits)
        return fail(QK_ERR_ARG, "chunk_qbit must be in [1, nqubits = %d], got %d", nqubits, chunk_qbit);
    const int n = nqubits, c = chunk_qbit;
    // rename through the circuit's own VSWAPs: bit_of[p] = qubit whose
    // content sits at position p of the circuit's state after them
    std::vector<int> bit_of(n);
    std::iota(bit_of.begin(), bit_of.end(), 0);
    std::vector<qk_gate> work;
    work.reserve(ng);
    for (size_t i = 0; i < ng; ++i) {
        const qk_gate &g = gates[i];
        if (g.nq < 1 || g.nq > QK_MAX_TARGETS) return fail(QK_ERR_ARG, "gate %zu: %d targets", i, g.nq);
        for (int j = 0; j < g.nq; ++j) {
            if (g.q[j] < 0 || g.q[j] >= n)
                return fail(QK_ERR_QUBIT, "gate %zu: qubit %d outside a %d-qubit state", i, g.q[j], n);
            for (int k = 0; k < j; ++k)
                if (g.q[k] == g.q[j]) return fail(QK_ERR_ORDER, "gate %zu: qubit %d repeated", i, g.q[j]);
        }
        if (is_vswap(g) || g.kind == QK_GATE_SWAP) {
            if (g.nq % 2) return fail(QK_ERR_ARG, "gate %zu: VSWAP with %d targets", i, g.nq);
            const int k = g.nq / 2;
            for (int j = 0; j < k; ++j) std::swap(bit_of[g.q[j]], bit_of[g.q[k + j]]);
            continue;
        }
        if (g.nq > c)
            return fail(QK_ERR_ARG, "gate %zu acts on %d qubits, more than chunk_qbit = %d", i, g.nq, c);
        qk_gate r = g;
        for (int j = 0; j < g.nq; ++j) r.q[j] = bit_of[g.q[j]];
        work.push_back(r);
    }

    auto *res = new qk_circuit();
    Grouper G{n, c, std::vector<int>(n), std::vector<int>(n), res, std::vector<int>(n)};
    for (int p = 0; p < n; ++p) G.final_pos[bit_of[p]] = p;
    std::iota(G.pos.begin(), G.pos.end(), 0);
    std::iota(G.at.begin(), G.at.end(), 0);

    std::vector<size_t> pending(work.size());
    std::iota(pending.begin(), pending.end(), 0);
    constexpr size_t kNever = std::numeric_limits<size_t>::max();
    while (!pending.empty()) {
        std::vector<char> blocked(n, 0);
        std::vector<size_t> rest;
        int32_t taken = 0;
        for (size_t idx : pending) {
            const qk_gate &g = work[idx];
            bool blk = false, in = true;
            for (int j = 0; j < g.nq; ++j) {
                blk = blk || blocked[g.q[j]];
                in = in && G.pos[g.q[j]] < c;
            }
            if (!blk && in) {
                res->gates.push_back(G.place(g));
                ++taken;
            } else {
                for (int j = 0; j < g.nq; ++j) blocked[g.q[j]] = 1;
                rest.push_back(idx);
            }
        }
        if (taken) {
            res->group_sizes.push_back(taken);
            pending.swap(rest);
            continue;
        }
        // The first remaining gate needs qubits from outside the chunk.  The
        // next chunk set S starts with its qubits and grows by the qubit that
        // lets the most remaining gates run (ties: a qubit already in the
        // chunk, which costs no exchange, then the one needed soonest).
        std::vector<size_t> next(n, kNever);
        for (size_t k = 0; k < pending.size(); ++k) {
            const qk_gate &g = work[pending[k]];
            for (int j = 0; j < g.nq; ++j)
                if (next[g.q[j]] == kNever) next[g.q[j]] = k;
        }
        std::vector<char> inS(n, 0), blk(n, 0);
        int size = 0;
        const qk_gate &g0 = work[pending[0]];
        for (int j = 0; j < g0.nq; ++j) inS[g0.q[j]] = 1, ++size;
        auto runnable = [&]() {
            std::fill(blk.begin(), blk.end(), 0);
            size_t cnt = 0;
            int nblk = 0;
            for (size_t idx : pending) {
                const qk_gate &g = work[idx];
                bool b = false, ok = true;
                for (int j = 0; j < g.nq; ++j) {
                    b = b || blk[g.q[j]];
                    ok = ok && inS[g.q[j]];
                }
                if (!b && ok) ++cnt;
                else
                    for (int j = 0; j < g.nq; ++j)
                        if (!blk[g.q[j]]) blk[g.q[j]] = 1, ++nblk;
                if (nblk == n) break;
            }
            return cnt;
        };
        while (size < c) {
            int best = -1;
            size_t bestc = 0;
            for (int q = 0; q < n; ++q) {
                if (inS[q] || next[q] == kNever) continue;
                inS[q] = 1;
                const size_t a = runnable();
                inS[q] = 0;
                bool better = best < 0 || a > bestc;
                if (!better && a == bestc) {
                    const bool qi = G.pos[q] < c, bi = G.pos[best] < c;
                    better = (qi && !bi) || (qi == bi && next[q] < next[best]);
                }
                if (better) best = q, bestc = a;
            }
            if (best < 0) break;
            inS[best] = 1, ++size;
        }
        for (int p = 0; p < c && size < c; ++p)   // room left: keep chunk qubits
            if (!inS[G.at[p]]) inS[G.at[p]] = 1, ++size;
        std::vector<int> in, ex;   // chunk positions that leave, outer positions that come in
        for (int p = 0; p < c; ++p)
            if (!inS[G.at[p]]) in.push_back(p);
        for (int p = c; p < n; ++p)
            if (inS[G.at[p]]) ex.push_back(p);
        if (in.empty()) {   // cannot happen: the first gate has <= c qubits
            delete res;
            return fail(QK_ERR_ARG, "chunk grouping made no progress");
        }
        G.exchange(in, ex);
    }

    // back to the circuit's layout (position p holds qubit bit_of[p]):
    // positions above the chunk first, two at a time where their qubits wait
    // in the chunk in the same order; qubits parked at other outer positions
    // come through the chunk, preferably replacing qubits bound outward
    const std::vector<int> &want_at = bit_of;
    for (;;) {
        std::vector<std::pair<int, int>> direct;   // (outer position, chunk position of its qubit)
        std::vector<int> parked;                   // outer positions of qubits bound elsewhere outward
        bool done = true;
        for (int p = c; p < n; ++p) {
            if (G.at[p] == want_at[p]) continue;
            done = false;
            const int from = G.pos[want_at[p]];
            if (from < c) direct.push_back({p, from});
            else parked.push_back(from);
        }
        if (done) break;
        if (!direct.empty()) {
            std::vector<int> in{direct[0].second}, ex{direct[0].first};
            for (size_t k = 1; k < direct.size(); ++k)
                if ((direct[k].second > in[0]) == (direct[k].first > ex[0])) {
                    in.push_back(direct[k].second);
                    ex.push_back(direct[k].first);
                    break;
                }
            G.exchange(in, ex);
            continue;
        }
        // bring up to two parked qubits into the chunk
        std::vector<int> slots;
        for (int a = 0; a < c && slots.size() < 2; ++a)
            if (std::find(want_at.begin() + c, want_at.end(), G.at[a]) != want_at.end()) slots.push_back(a);
        for (int a = 0; a < c && slots.size() < 2; ++a)
            if (std::find(slots.begin(), slots.end(), a) == slots.end()) slots.push_back(a);
        const size_t k = std::min(parked.size(), slots.size());
        G.exchange(std::vector<int>(slots.begin(), slots.begin() + k), std::vector<int>(parked.begin(), parked.begin() + k));
    }
    int32_t swaps = 0;
    for (int p = 0; p < c; ++p) {
        if (G.at[p] == want_at[p]) continue;
        const int p2 = G.pos[want_at[p]];
        qk_gate s;
        std::memset(&s, 0, sizeof s);
        s.kind = QK_GATE_SWAP;
        s.nq = 2;
        s.q[0] = std::min(p, p2);
        s.q[1] = std::max(p, p2);
        res->gates.push_back(s);
        ++swaps;
        std::swap(G.at[p], G.at[p2]);
        G.pos[G.at[p]] = p;
        G.pos[G.at[p2]] = p2;
    }
    if (swaps) res->group_sizes.push_back(swaps);
    *out = res;
    qk::clear_error();
    return QK_OK;
}

int qk_circuit_write(const qk_circuit *c, int is_subcircuit, const char *path) {
    if (!c || !path) return fail(QK_ERR_ARG, "null argument");
    std::string text;
    char buf[64];
    auto num = [&](double v) {
        std::snprintf(buf, sizeof buf, " %.17g", v);
        text += buf;
    };
    size_t k = 0;
    for (size_t gi = 0; gi < c->group_sizes.size(); ++gi) {
        const int32_t cnt = c->group_sizes[gi];
        if (is_subcircuit) text += std::to_string(cnt) + "\n";
        for (int32_t j = 0; j < cnt; ++j, ++k) {
            const qk_gate &g = c->gates[k];
            static const char *names[] = {"", "H", "X", "Y", "Z", "P", "RX", "RY", "RZ", "U1", "U2", "SWAP", "CP",
                                          "RZZ"};
            if (g.kind >= QK_GATE_H && g.kind <= QK_GATE_RZZ) text += names[g.kind];
            else if (is_vswap(g))
                text += std::string(g.kind == QK_GATE_MPI_VSWAP ? "MPI_VSWAP_" : "VSWAP_") +
                        std::to_string(g.nq / 2) + "_" + std::to_string(g.nq / 2);
            else return fail(QK_ERR_ARG, "gate %zu: unknown kind %d", k, g.kind);
            for (int i = 0; i < g.nq; ++i) text += " " + std::to_string(g.q[i]);
            switch (g.kind) {
            case QK_GATE_P: case QK_GATE_RX: case QK_GATE_RY: case QK_GATE_RZ: case QK_GATE_CP: case QK_GATE_RZZ:
                num(g.param);
                break;
            case QK_GATE_U1:
                for (int i = 0; i < 8; ++i) num(g.coeff[i]);
                break;
            case QK_GATE_U2:
                for (int i = 0; i < 32; ++i) num(g.coeff[i]);
                break;
            default:
                break;
            }
            text += "\n";
        }
    }
    FILE *f = std::fopen(path, "w");
    if (!f) return fail(QK_ERR_IO, "cannot open %s for writing", path);
    const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
    if (std::fclose(f) != 0 || !ok) return fail(QK_ERR_IO, "cannot write %s", path);
    qk::clear_error();
    return QK_OK;
}

}  // extern "C"
