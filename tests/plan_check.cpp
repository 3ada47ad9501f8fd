// CPU check of the fused-pass planner (subquokka_dev_b200/csrc/qk_plan.cpp).
//
// The pass programs of a HostPlan are run by an emulator written from their
// definitions in qk_internal.h: a pass gathers every tile (2^T amplitudes
// whose index bits are the pass's state bits bpos) and runs its program on
// it; register slot s stands for tile bit Q[s] as the last TOP_REMAP set it;
// condition codes name a tile bit, a state bit outside the tile (constant
// over the tile) or none.  The thread and register layout of the CUDA
// interpreter plays no part: what is checked is the plan itself (pass
// choice, slots, condition codes, coefficient order, gradient slots,
// permutation passes).  Random circuits (every MEM gate, random U1/U2,
// CNOT-shaped U2s, VSWAPs) with small tiles, so that each plan has many
// passes and re-mappings:
// - forward plans (build_plan, both dtypes' budgets) against the dense
//   simulation of the gate list;
// - tensor-core dense-block plans (build_dense_blocks, widths 5 and 6)
//   against the same dense simulation;
// - adjoint plans (build_adjoint_plan) against the direct backward sweep:
//   the inverse gates from last to first on psi and lambda, the gradient of
//   each trainable gate taken just before its inverse.
// States agree within 1e-12; gradients within 1e-12, or 1e-9 for circuits
// with H (the reference's H constant is 1.1e-11 off unitary, and gradient
// ops move past gates on other qubits).  Exit status 0 on success.
#include "dense_sim.h"
#include "qk_operand.h"

using namespace dense_sim;
using qk::HostPlan;
using qk::PassDesc;
using qk::TOp;

namespace {

float bf16_value(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// The tensor-core operands of block b against its unitary: the complex128
// digit planes rebuild every entry of the real embedding W to half a unit
// of its row's last digit, every digit is in range; the complex64 bf16 hi +
// lo pair rebuilds W to bf16 x bf16 rounding; the supertile layouts hold the
// block's qubits and the lowest others, ascending.
int check_operands(const qk::DenseBlock &b, int n) {
    int bad = 0;
    std::vector<uint32_t> w8;
    qk::dense_i8_operand(b, w8);
    const unsigned char *digits = reinterpret_cast<const unsigned char *>(w8.data());
    const double *scale = reinterpret_cast<const double *>(w8.data() + qk::kI8OperandWords);
    std::vector<uint16_t> w16;
    qk::dense_block_operand(b, w16);
    const unsigned char *hi = reinterpret_cast<const unsigned char *>(w16.data());
    const unsigned char *lo = hi + qk::kBf16OperandBytes;
    double e8 = 0, e16 = 0;
    for (int m = 0; m < 128; ++m)
        for (int k = 0; k < 128; ++k) {
            const int ip = m >> 1, a = m & 1, i = k >> 1, c = k & 1;
            const double ur = b.u[2 * (ip * 64 + i)], ui = b.u[2 * (ip * 64 + i) + 1];
            const double w = a == 0 ? (c == 0 ? ur : -ui) : (c == 0 ? ui : ur);
            double v = 0;
            for (int d = qk::kI8Digits - 1; d >= 0; --d) {
                const int dg = (int8_t)digits[qk::sw128_i8_off((uint32_t)d, (uint32_t)m, (uint32_t)k)];
                if (d < qk::kI8Digits - 1 ? (dg < -128 || dg > 127) : (dg < -65 || dg > 65)) ++bad;
                v = v * 256 + dg;
            }
            // scale[m] = 2^(e_m - 1028); one unit of v is 2^(e_m - 1076)
            const double unit = std::ldexp(scale[m], -48);
            e8 = std::max(e8, std::fabs(v * unit - w) / unit);
            uint16_t h, l;
            std::memcpy(&h, hi + qk::sw128_off((uint32_t)m, (uint32_t)k), 2);
            std::memcpy(&l, lo + qk::sw128_off((uint32_t)m, (uint32_t)k), 2);
            e16 = std::max(e16, std::fabs((double)bf16_value(h) + (double)bf16_value(l) - w));
        }
    if (e8 > 0.5 || e16 > 1e-4) {
        std::printf("operands: digit error %.3g units, bf16 error %.3g\n", e8, e16);
        ++bad;
    }
    for (int tb : {12, 13}) {
        const qk::DenseDesc dd = qk::dense_block_desc(b, n, tb);
        int blockbits = 0;
        for (int t = 0; t < dd.p.T; ++t) {
            if (t && dd.p.bpos[t] <= dd.p.bpos[t - 1]) ++bad;
            const bool inblock = std::find(b.q, b.q + qk::kDenseQubits, dd.p.bpos[t]) != b.q + qk::kDenseQubits;
            if (inblock != (((dd.blockmask >> t) & 1u) != 0)) ++bad;
            blockbits += inblock;
        }
        if (dd.p.T != std::min(n, tb) || blockbits != qk::kDenseQubits || dd.p.L < 1) ++bad;
    }
    return bad;
}

int bit_of(uint8_t code, uint64_t j, uint64_t base) {
    if (code == qk::kNoQubit) return -1;
    if (code & qk::kOuterFlag) return (int)((base >> (code & 0x7F)) & 1);
    return (int)((j >> code) & 1);
}

// run every pass of hp on psi (and lam when two-state); gradients into g
void emulate(const HostPlan &hp, State &psi, State *lam, std::vector<double> &g) {
    const int n = hp.n;
    for (const PassDesc &d : hp.passes) {
        State *states[2] = {&psi, lam};
        if (d.perm == 2) {   // flat permutation: state bits perm_a[i] <-> perm_b[i]
            Op p;
            std::memset(&p, 0, sizeof p);
            p.kind = qk::OP_PERM;
            p.nq = 2 * d.nperm;
            for (int i = 0; i < d.nperm; ++i) {
                p.q[i] = d.perm_a[i];
                p.q[d.nperm + i] = d.perm_b[i];
            }
            std::vector<int> qs;
            const auto m = matrix_of(p, qs);
            for (State *s : states)
                if (s) apply_matrix(*s, n, qs, m);
            continue;
        }
        const int T = d.T;
        const uint64_t tn = 1ull << T;
        std::vector<int> outer;
        std::vector<char> in_tile(n, 0);
        for (int k = 0; k < T; ++k) in_tile[d.bpos[k]] = 1;
        for (int q = 0; q < n; ++q)
            if (!in_tile[q]) outer.push_back(q);
        auto addr = [&](uint64_t base, uint64_t j) {
            uint64_t a = base;
            for (int k = 0; k < T; ++k)
                if ((j >> k) & 1) a |= 1ull << d.bpos[k];
            return a;
        };
        for (uint64_t t = 0; t < (1ull << outer.size()); ++t) {
            uint64_t base = 0;
            for (size_t k = 0; k < outer.size(); ++k)
                if ((t >> k) & 1) base |= 1ull << outer[k];
            std::vector<cd> x[2];
            for (int si = 0; si < 2; ++si)
                if (states[si]) {
                    x[si].resize(tn);
                    for (uint64_t j = 0; j < tn; ++j) x[si][j] = (*states[si])[addr(base, j)];
                }
            if (d.perm == 1) {   // tile-local bit pairs swapped on store
                for (int si = 0; si < 2; ++si)
                    if (states[si])
                        for (uint64_t j = 0; j < tn; ++j) {
                            uint64_t r = j;
                            for (int i = 0; i < d.nperm; ++i) {
                                const uint64_t a = (j >> d.perm_a[i]) & 1, b = (j >> d.perm_b[i]) & 1;
                                r = (r & ~(1ull << d.perm_a[i]) & ~(1ull << d.perm_b[i])) | (b << d.perm_a[i]) |
                                    (a << d.perm_b[i]);
                            }
                            (*states[si])[addr(base, r)] = x[si][j];
                        }
                continue;
            }
            std::vector<int> Q;
            auto coef = [&](const TOp &op, int k) {
                const size_t i = (size_t)(d.coef0 + op.coef + k);
                return cd(hp.coef[2 * i], hp.coef[2 * i + 1]);
            };
            auto pairs = [&](int tb, auto &&f) {
                for (uint64_t j = 0; j < tn; ++j)
                    if (!((j >> tb) & 1)) f(j, j | (1ull << tb));
            };
            for (int pi = d.prog0; pi < d.prog0 + d.nprog; ++pi) {
                const TOp &op = hp.ops[pi];
                switch (op.kind) {
                case qk::TOP_REMAP:
                    Q.assign(op.bits, op.bits + op.nbits);
                    break;
                case qk::TOP_G1:
                case qk::TOP_CG1:
                case qk::TOP_CX:
                    for (int si = 0; si < 2; ++si)
                        if (states[si])
                            pairs(Q.at(op.a), [&](uint64_t j0, uint64_t j1) {
                                const cd a = x[si][j0], b = x[si][j1];
                                if (op.kind == qk::TOP_CX) {
                                    if (bit_of(op.b, j0, base) == 1) std::swap(x[si][j0], x[si][j1]);
                                    return;
                                }
                                const int off = op.kind == qk::TOP_CG1 && bit_of(op.b, j0, base) == 1 ? 4 : 0;
                                x[si][j0] = coef(op, off) * a + coef(op, off + 1) * b;
                                x[si][j1] = coef(op, off + 2) * a + coef(op, off + 3) * b;
                            });
                    break;
                case qk::TOP_R1:
                    for (int si = 0; si < 2; ++si)
                        if (states[si])
                            pairs(Q.at(op.a), [&](uint64_t j0, uint64_t j1) {
                                const cd a = x[si][j0], b = x[si][j1];
                                x[si][j0] = coef(op, 0).real() * a + coef(op, 0).imag() * b;
                                x[si][j1] = coef(op, 1).real() * a + coef(op, 1).imag() * b;
                            });
                    break;
                case qk::TOP_R2:
                case qk::TOP_G2: {
                    const int ta = Q.at(op.a), tb = Q.at(op.b);
                    for (int si = 0; si < 2; ++si)
                        if (states[si])
                            for (uint64_t j = 0; j < tn; ++j) {
                                if (((j >> ta) & 1) || ((j >> tb) & 1)) continue;
                                const uint64_t idx[4] = {j, j | (1ull << ta), j | (1ull << tb),
                                                         j | (1ull << ta) | (1ull << tb)};
                                cd in[4], out[4];
                                for (int k = 0; k < 4; ++k) in[k] = x[si][idx[k]];
                                for (int r = 0; r < 4; ++r) {
                                    out[r] = 0;
                                    for (int k = 0; k < 4; ++k) {
                                        const cd c = coef(op, op.kind == qk::TOP_R2 ? 2 * r + k / 2 : 4 * r + k);
                                        const double re = k % 2 ? c.imag() : c.real();
                                        out[r] += op.kind == qk::TOP_R2 ? cd(re) * in[k] : c * in[k];
                                    }
                                }
                                for (int k = 0; k < 4; ++k) x[si][idx[k]] = out[k];
                            }
                    break;
                }
                case qk::TOP_DIAG:
                case qk::TOP_PHASE:
                    for (int si = 0; si < 2; ++si)
                        if (states[si])
                            for (uint64_t j = 0; j < tn; ++j) {
                                const int ba = bit_of(op.a, j, base), bb = bit_of(op.b, j, base);
                                if (op.kind == qk::TOP_DIAG)
                                    x[si][j] *= coef(op, (ba < 0 ? 0 : ba) + 2 * (bb < 0 ? 0 : bb));
                                else if (ba != 0 && bb != 0)
                                    x[si][j] *= coef(op, 0);
                            }
                    break;
                case qk::TOP_GRAD: {
                    const int gen = op.b;
                    const int tb = Q.at(op.a);
                    for (int w = 0; w < (gen == 5 ? 2 : 1); ++w) {
                        double a = gen == 1, b = gen == 2, cz = gen == 3;
                        if (gen >= 4) {
                            a = coef(op, 2 * w).real();
                            b = coef(op, 2 * w).imag();
                            cz = coef(op, 2 * w + 1).real();
                        }
                        const int slot = w ? (op.bits[2] | (op.bits[3] << 8)) : (op.bits[0] | (op.bits[1] << 8));
                        const int param = hp.grad_params.at((size_t)(d.grad0 + slot));
                        const cd g00 = cz, g01 = cd(a, -b), g10 = cd(a, b), g11 = -cz;
                        double s = 0;
                        pairs(tb, [&](uint64_t j0, uint64_t j1) {
                            const cd p0 = x[0][j0], p1 = x[0][j1], l0 = x[1][j0], l1 = x[1][j1];
                            s += (std::conj(l0) * (g00 * p0 + g01 * p1) + std::conj(l1) * (g10 * p0 + g11 * p1)).imag();
                        });
                        g.at(param) += s;
                    }
                    break;
                }
                default:
                    std::fprintf(stderr, "unknown program op %d\n", op.kind);
                    std::exit(2);
                }
            }
            for (int si = 0; si < 2; ++si)
                if (states[si])
                    for (uint64_t j = 0; j < tn; ++j) (*states[si])[addr(base, j)] = x[si][j];
        }
    }
}

}  // namespace

int main() {
    int bad = 0, plans = 0;
    for (int seed = 0; seed < 80; ++seed) {
        const bool with_h = seed % 2;
        Gen G{std::mt19937_64(1000 + seed), 6 + seed % 3, with_h};
        const int n = G.n;
        const int T = 4 + seed % 3, r = 2 + (seed / 3) % 2;
        qk::PlanOptions o{seed % 4 < 2 ? QK_C128 : QK_C64, T, r};
        // forward
        std::vector<qk_gate> gates;
        for (int i = 0; i < 70; ++i) {
            if (i % 23 == 7) {
                qk_gate v;
                std::memset(&v, 0, sizeof v);
                const Op p = G.vswap();
                v.kind = QK_GATE_VSWAP;
                v.nq = 4;
                for (int k = 0; k < 4; ++k) v.q[k] = p.q[k];
                gates.push_back(v);
            } else {
                gates.push_back(G.gate());
            }
        }
        const State init = G.state();
        State ref = init;
        std::vector<double> none(1, 0);
        for (const qk_gate &g : gates) {
            std::vector<int> qs;
            const Op op = lower(g);
            const auto m = matrix_of(op, qs);
            apply_matrix(ref, n, qs, m);
        }
        // default programs (real ops, deferred diagonal ops) and those of
        // the batched kernel (plain ops)
        bool failed = false;
        for (int plain : {0, 1}) {
            o.plain_ops = plain;
            HostPlan hp;
            if (qk::build_plan(gates.data(), gates.size(), n, o, hp)) {
                std::printf("seed %d: build_plan failed: %s\n", seed, qk_last_error());
                ++bad;
                failed = true;
                break;
            }
            ++plans;
            State got = init;
            emulate(hp, got, nullptr, none);
            const double df = max_diff(ref, got);
            if (df > 1e-12) {
                std::printf("forward seed %d plain %d (n %d, T %d, r %d): max |d amp| %.3g, %zu passes\n", seed, plain,
                            n, T, r, df, hp.passes.size());
                ++bad;
            }
        }
        if (failed) continue;
        // tensor-core dense blocks (64 x 64 unitaries on six qubits, block
        // index bit b = qubit q[b]; permutation blocks for the restore)
        // (both dtypes: their permutation blocks have different tile limits)
        for (int form = 0; form < 4; ++form) {
            const int width = 5 + (form & 1), dtype = form < 2 ? QK_C64 : QK_C128;
            std::vector<qk::DenseBlock> blocks;
            if (qk::build_dense_blocks(gates.data(), gates.size(), n, width, dtype, blocks)) {
                std::printf("seed %d: build_dense_blocks failed: %s\n", seed, qk_last_error());
                ++bad;
                continue;
            }
            ++plans;
            State want = G.state(), have = want;
            for (const qk_gate &g : gates) {
                std::vector<int> qs;
                const auto m = matrix_of(lower(g), qs);
                apply_matrix(want, n, qs, m);
            }
            for (const qk::DenseBlock &b : blocks) {
                std::vector<int> qs;
                if (!b.perm) bad += check_operands(b, 14);   // layouts of these qubits in a 14-qubit state
                if (b.perm) {
                    const auto m = matrix_of(b.perm_op, qs);
                    apply_matrix(have, n, qs, m);
                    continue;
                }
                qs.assign(b.q, b.q + qk::kDenseQubits);
                std::vector<cd> u((size_t)qk::kDenseDim * qk::kDenseDim);
                for (size_t k = 0; k < u.size(); ++k) u[k] = cd(b.u[2 * k], b.u[2 * k + 1]);
                apply_matrix(have, n, qs, u);
            }
            const double dd = max_diff(want, have);
            if (dd > 1e-12) {
                std::printf("dense seed %d width %d dtype %d: max |d amp| %.3g, %zu blocks\n", seed, width, dtype, dd,
                            blocks.size());
                ++bad;
            }
        }
        // adjoint: trainable RX / RY / RZ, some sharing a parameter
        std::vector<qk_gate> circ;
        std::vector<int32_t> pidx;
        int np = 0;
        for (int i = 0; i < 70; ++i) {
            const qk_gate g = G.gate();
            circ.push_back(g);
            const bool rot = g.kind == QK_GATE_RX || g.kind == QK_GATE_RY || g.kind == QK_GATE_RZ;
            pidx.push_back(rot ? (np > 2 && G.rng() % 4 == 0 ? (int)(G.rng() % np) : np++) : -1);
        }
        qk::PlanOptions ao{o.dtype, std::min(T, 6), 2 + seed % 2, seed % 5 == 0};
        HostPlan ap;
        if (qk::build_adjoint_plan(circ.data(), circ.size(), pidx.data(), n, ao, ap)) {
            std::printf("seed %d: build_adjoint_plan failed: %s\n", seed, qk_last_error());
            ++bad;
            continue;
        }
        ++plans;
        std::vector<Op> back;
        for (size_t i = circ.size(); i-- > 0;) {
            Op op = lower(circ[i]);
            if (pidx[i] >= 0) {
                Op gr;
                std::memset(&gr, 0, sizeof gr);
                gr.kind = qk::OP_GRAD;
                gr.nq = 1;
                gr.q[0] = op.q[0];
                gr.m[0] = circ[i].kind == QK_GATE_RX ? 1 : circ[i].kind == QK_GATE_RY ? 2 : 3;
                gr.aux = pidx[i];
                back.push_back(gr);
            }
            qk::invert_op(op);
            back.push_back(op);
        }
        State psi = G.state(), lam = G.state(), psi2 = psi, lam2 = lam;
        std::vector<double> g0(np + 1, 0), g1(np + 1, 0);
        run(back, n, psi, lam, g0);
        emulate(ap, psi2, &lam2, g1);
        double dg = 0;
        for (int k = 0; k <= np; ++k) dg = std::max(dg, std::fabs(g0[k] - g1[k]));
        const double ds = std::max(max_diff(psi, psi2), max_diff(lam, lam2));
        if (dg > (with_h ? 1e-9 : 1e-12) || ds > 1e-12) {
            std::printf("adjoint seed %d (n %d, T %d): max |d grad| %.3g, max |d amp| %.3g, %zu passes\n", seed, n,
                        ao.tile_bits, dg, ds, ap.passes.size());
            ++bad;
        }
    }
    std::printf("%d plans, %s\n", plans, bad ? "FAIL" : "ok");
    return bad ? 1 : 0;
}
