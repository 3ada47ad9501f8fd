// CPU check of the op-list rewrites (subquokka_dev_b200/csrc/qk_rewrite.cpp).
//
// Random op lists built from parsed gates (every MEM gate kind, random U1 /
// U2 matrices, CNOT-shaped U2s, VSWAPs) are run on small dense states by an
// independent simulator below, once as generated and once after the
// rewrites the planners apply:
// - forward lists: merge_one_qubit_runs, absorb_into_two_qubit_ops (with
//   and without keep_real, which leaves real one-qubit ops real and may
//   emit a real 4 x 4 op before a complex two-qubit op), asap_order,
//   relabel_perms; the final states must agree;
// - backward lists with gradient ops (Im <lambda|G|psi>, G = X, Y, Z):
//   hoist_gradients, merge_one_qubit_runs, absorb_into_two_qubit_ops,
//   pair_gradients; the final states and every gradient must agree.
// Exit status 0 when every case agrees within 1e-12.  One exception, from
// the reference's H: its constant 0.70710678118 makes H = 2c^2 (1 - 1.1e-11)
// times a unitary, so a gradient op moved past an H on another qubit (which
// commutes with it) changes by 1.1e-11 relative per H.  Lists with H are
// checked at 1e-12 for the states and 1e-9 for the gradients; lists without
// H at 1e-12 for both.
#include "dense_sim.h"

using namespace dense_sim;

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
        const bool keep_real = seed % 4 >= 2;
        qk::absorb_into_two_qubit_ops(rw, n, keep_real);
        if (seed % 2) qk::asap_order(rw, n);
        State p0 = G.state(), l0 = p0, p1 = p0, l1 = p0;
        std::vector<double> g0(64, 0), g1(64, 0);
        run(ops, n, p0, l0, g0);
        run(rw, n, p1, l1, g1);
        const double df = max_diff(p0, p1);
        if (df > 1e-12) {
            std::printf("forward seed %d (keep_real %d): max |d amp| %.3g (%zu -> %zu ops)\n", seed, (int)keep_real, df,
                        ops.size(), rw.size());
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
