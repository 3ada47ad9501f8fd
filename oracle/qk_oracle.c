/*
 * ORACLE -- test infrastructure only (see qk_oracle.h).
 *
 * Restatement of the reference's MEM gate bodies (src/circuit.cpp:245-375)
 * and coefficient construction (src/circuit.cpp:2550-3041, :3457-3556).  The
 * reference walks each gate's amplitude tuples chunk by chunk with the loop
 * macros of src/circuit.cpp:143-242 and bit_string (src/MEM_Runner.cpp:90-99);
 * for ascending targets that visits every tuple (i, i + 2^t0, ...) exactly
 * once, which is what the loops below do directly.
 */
#include "qk_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cx;

static inline cx ld(const double *s, uint64_t i) { cx r = {s[2 * i], s[2 * i + 1]}; return r; }
static inline void st(double *s, uint64_t i, cx v) { s[2 * i] = v.re; s[2 * i + 1] = v.im; }
static inline cx mul(cx a, cx b) { cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cx add(cx a, cx b) { cx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cx C(double re, double im) { cx r = {re, im}; return r; }

/* insert a zero bit at position t (bit_string, src/MEM_Runner.cpp:90-99) */
static inline uint64_t ins0(uint64_t p, int t) {
    uint64_t lo = (1ull << t) - 1;
    return ((p & ~lo) << 1) | (p & lo);
}

/* [a0', a1'] = [[m0, m1], [m2, m3]] [a0, a1] -- U1GATE, RXGATE, RYGATE shape */
static void dense1(double *s, int n, int t, cx m0, cx m1, cx m2, cx m3) {
    const uint64_t np = 1ull << (n - 1), h = 1ull << t;
#pragma omp parallel for schedule(static)
    for (uint64_t p = 0; p < np; ++p) {
        uint64_t i = ins0(p, t);
        cx q0 = ld(s, i), q1 = ld(s, i + h);
        st(s, i, add(mul(m0, q0), mul(m1, q1)));
        st(s, i + h, add(mul(m2, q0), mul(m3, q1)));
    }
}

/* amplitudes with bit t set *= ph -- ZGATE, PGATE */
static void phase1(double *s, int n, int t, cx ph) {
    const uint64_t np = 1ull << (n - 1), h = 1ull << t;
#pragma omp parallel for schedule(static)
    for (uint64_t p = 0; p < np; ++p) {
        uint64_t i = ins0(p, t) | h;
        st(s, i, mul(ld(s, i), ph));
    }
}

int qko_apply(double *s, int n, const qk_gate *g) {
    const int a = g->q[0], b = g->q[1];
    const double phi = g->param;
    switch (g->kind) {
    case QK_GATE_H: { /* HGATE: c (q0 + q1), c (q0 - q1), c = 0.70710678118 (:245-248) */
        const double c = 0.70710678118;
        const uint64_t np = 1ull << (n - 1), h = 1ull << a;
#pragma omp parallel for schedule(static)
        for (uint64_t p = 0; p < np; ++p) {
            uint64_t i = ins0(p, a);
            cx q0 = ld(s, i), q1 = ld(s, i + h);
            st(s, i, C(c * (q0.re + q1.re), c * (q0.im + q1.im)));
            st(s, i + h, C(c * (q0.re - q1.re), c * (q0.im - q1.im)));
        }
        return 0;
    }
    case QK_GATE_X: /* XGATE (:255-257) */
        dense1(s, n, a, C(0, 0), C(1, 0), C(1, 0), C(0, 0));
        return 0;
    case QK_GATE_Y: /* YGATE: q1 * (-1i), q0 * 1i (:263-265) */
        dense1(s, n, a, C(0, 0), C(0, -1), C(0, 1), C(0, 0));
        return 0;
    case QK_GATE_Z: /* ZGATE (:271-272) */
        phase1(s, n, a, C(-1, 0));
        return 0;
    case QK_GATE_P: /* Phase_Gate_MEM phi(cos, sin) (:2655), PGATE (:284-285) */
        phase1(s, n, a, C(cos(phi), sin(phi)));
        return 0;
    case QK_GATE_U1: /* U1GATE (:274-277) */
        dense1(s, n, a, C(g->coeff[0], g->coeff[1]), C(g->coeff[2], g->coeff[3]), C(g->coeff[4], g->coeff[5]),
               C(g->coeff[6], g->coeff[7]));
        return 0;
    case QK_GATE_RX: { /* (:2706-2709), RXGATE (:287-290) */
        cx c = C(cos(phi / 2), 0), is = C(0, sin(-phi / 2));
        dense1(s, n, a, c, is, is, c);
        return 0;
    }
    case QK_GATE_RY: { /* (:2734-2737), RYGATE (:297-300) */
        cx c = C(cos(phi / 2), 0), sn = C(sin(phi / 2), 0), msn = C(-sin(phi / 2), 0);
        dense1(s, n, a, c, msn, sn, c);
        return 0;
    }
    case QK_GATE_RZ: { /* (:2762-2765), RZGATE (:307-309) */
        cx ep = C(cos(phi / 2), sin(phi / 2)), en = C(cos(-phi / 2), sin(-phi / 2));
        const uint64_t np = 1ull << (n - 1), h = 1ull << a;
#pragma omp parallel for schedule(static)
        for (uint64_t p = 0; p < np; ++p) {
            uint64_t i = ins0(p, a);
            st(s, i, mul(ld(s, i), en));
            st(s, i + h, mul(ld(s, i + h), ep));
        }
        return 0;
    }
    case QK_GATE_U2: { /* U2_Gate_MEM coefficient permutation (:2811-2819), U2Gate (:321-329) */
        cx m[16];
        for (int i = 0; i < 16; ++i) {
            int b1 = i & 1, b2 = (i >> 1) & 1, b3 = (i >> 2) & 1, b4 = (i >> 3) & 1;
            int res = (b3 << 3) | (b4 << 2) | (b1 << 1) | b2;
            m[i] = C(g->coeff[2 * res], g->coeff[2 * res + 1]);
        }
        const uint64_t nq = 1ull << (n - 2), A = 1ull << a, B = 1ull << b;
#pragma omp parallel for schedule(static)
        for (uint64_t p = 0; p < nq; ++p) {
            uint64_t i = ins0(ins0(p, a), b);
            cx q[4] = {ld(s, i), ld(s, i + A), ld(s, i + B), ld(s, i + A + B)};
            uint64_t off[4] = {i, i + A, i + B, i + A + B};
            for (int r = 0; r < 4; ++r) {
                cx v = add(add(add(mul(m[4 * r], q[0]), mul(m[4 * r + 1], q[1])), mul(m[4 * r + 2], q[2])),
                           mul(m[4 * r + 3], q[3]));
                st(s, off[r], v);
            }
        }
        return 0;
    }
    case QK_GATE_SWAP: /* SWAPGate (:351-355) */
    case QK_GATE_VSWAP:
    case QK_GATE_MPI_VSWAP: {
        /* VSWAP_k_k swaps q[i] with q[k+i]; VSWAP_1_1 is SWAP (:2937-2940),
         * VSWAP_2_2 is SWAP(q0,q2) SWAP(q1,q3) (:3457-3556) */
        const int k = g->nq / 2;
        const uint64_t N = 1ull << n;
#pragma omp parallel for schedule(static)
        for (uint64_t e = 0; e < N; ++e) {
            uint64_t f = e;
            for (int i = 0; i < k; ++i) {
                uint64_t x = (e >> g->q[i]) & 1, y = (e >> g->q[k + i]) & 1;
                f = (f & ~(1ull << g->q[i]) & ~(1ull << g->q[k + i])) | (y << g->q[i]) | (x << g->q[k + i]);
            }
            if (e < f) {
                cx t = ld(s, e);
                st(s, e, ld(s, f));
                st(s, f, t);
            }
        }
        return 0;
    }
    case QK_GATE_CP: { /* exp_iPhi (:2947-2949), CPGATE (:362-363) */
        cx ph = C(cos(phi), sin(phi));
        const uint64_t nq = 1ull << (n - 2), AB = (1ull << a) | (1ull << b);
#pragma omp parallel for schedule(static)
        for (uint64_t p = 0; p < nq; ++p) {
            uint64_t i = ins0(ins0(p, a), b) | AB;
            st(s, i, mul(ld(s, i), ph));
        }
        return 0;
    }
    case QK_GATE_RZZ: { /* (:2988-2991), RZZGATE (:365-369) */
        cx ep = C(cos(phi / 2), sin(phi / 2)), en = C(cos(-phi / 2), sin(-phi / 2));
        const uint64_t nq = 1ull << (n - 2), A = 1ull << a, B = 1ull << b;
#pragma omp parallel for schedule(static)
        for (uint64_t p = 0; p < nq; ++p) {
            uint64_t i = ins0(ins0(p, a), b);
            st(s, i, mul(ld(s, i), en));
            st(s, i + A, mul(ld(s, i + A), ep));
            st(s, i + B, mul(ld(s, i + B), ep));
            st(s, i + A + B, mul(ld(s, i + A + B), en));
        }
        return 0;
    }
    default:
        return -1;
    }
}

int qko_apply_list(double *state, int n, const qk_gate *gates, size_t ng) {
    for (size_t i = 0; i < ng; ++i)
        if (qko_apply(state, n, &gates[i])) return -1;
    return 0;
}

double qko_expval_zz_x(const double *s, int n, const double *J, const double *h) {
    const uint64_t N = 1ull << n;
    double acc = 0;
    for (int i = 0; i + 1 < n; ++i) {
        double e = 0;
#pragma omp parallel for reduction(+ : e) schedule(static)
        for (uint64_t k = 0; k < N; ++k) {
            double p = s[2 * k] * s[2 * k] + s[2 * k + 1] * s[2 * k + 1];
            e += (((k >> i) ^ (k >> (i + 1))) & 1) ? -p : p;
        }
        acc += J[i] * e;
    }
    for (int i = 0; i < n; ++i) {
        double e = 0;
        const uint64_t h1 = 1ull << i;
#pragma omp parallel for reduction(+ : e) schedule(static)
        for (uint64_t p = 0; p < N / 2; ++p) {
            uint64_t k = ins0(p, i);
            /* <psi|X_i|psi> = 2 Re sum conj(a0) a1 */
            e += 2 * (s[2 * k] * s[2 * (k + h1)] + s[2 * k + 1] * s[2 * (k + h1) + 1]);
        }
        acc += h[i] * e;
    }
    return acc;
}

/* ---------------------------------------------------------------------------
 * Adjoint gradient (the engine's own addition; the reference has none).
 * psi = U_L..U_1 psi0, lambda = H psi, then for k = L..1:
 *   g[p(k)] += Im <lambda|G_k|psi>,  psi <- U_k^-1 psi,  lambda <- U_k^dag lambda
 * with U^-1 = U^dag (a gate with negated angle, or the conjugate transpose).
 * ------------------------------------------------------------------------- */
static int inverse_gate(const qk_gate *g, qk_gate *inv) {
    *inv = *g;
    switch (g->kind) {
    case QK_GATE_H: case QK_GATE_X: case QK_GATE_Y: case QK_GATE_Z: case QK_GATE_SWAP:
    case QK_GATE_VSWAP: case QK_GATE_MPI_VSWAP:
        return 0;
    case QK_GATE_P: case QK_GATE_RX: case QK_GATE_RY: case QK_GATE_RZ: case QK_GATE_CP: case QK_GATE_RZZ:
        inv->param = -g->param;
        return 0;
    case QK_GATE_U1: case QK_GATE_U2: {
        const int d = g->kind == QK_GATE_U1 ? 2 : 4;
        for (int r = 0; r < d; ++r)
            for (int c = 0; c < d; ++c) {
                inv->coeff[2 * (r * d + c)] = g->coeff[2 * (c * d + r)];
                inv->coeff[2 * (r * d + c) + 1] = -g->coeff[2 * (c * d + r) + 1];
            }
        return 0;
    }
    default:
        return -1;
    }
}

static void apply_terms(double *out, const double *psi, int n, const qko_term *t, size_t nt) {
    const uint64_t N = 1ull << n;
    memset(out, 0, sizeof(double) * 2 * N);
    for (size_t k = 0; k < nt; ++k) {
        const int ip = __builtin_popcountll(t[k].x & t[k].z) & 3;
#pragma omp parallel for schedule(static)
        for (uint64_t j = 0; j < N; ++j) {
            const uint64_t src = j ^ t[k].x;
            const double c = (__builtin_popcountll(src & t[k].z) & 1) ? -t[k].coeff : t[k].coeff;
            const double fr = ip == 0 ? c : ip == 2 ? -c : 0, fi = ip == 1 ? c : ip == 3 ? -c : 0;
            out[2 * j] += fr * psi[2 * src] - fi * psi[2 * src + 1];
            out[2 * j + 1] += fr * psi[2 * src + 1] + fi * psi[2 * src];
        }
    }
}

int qko_adjoint_grad(double *psi, int n, const qk_gate *gates, size_t ng, const int *pidx, size_t nparams,
                     const qko_term *terms, size_t nterms, double *expval, double *grad) {
    const uint64_t N = 1ull << n;
    if (qko_apply_list(psi, n, gates, ng)) return -1;
    double *lam = (double *)malloc(sizeof(double) * 2 * N);
    if (!lam) return -1;
    apply_terms(lam, psi, n, terms, nterms);
    double e = 0;
#pragma omp parallel for reduction(+ : e) schedule(static)
    for (uint64_t j = 0; j < N; ++j) e += psi[2 * j] * lam[2 * j] + psi[2 * j + 1] * lam[2 * j + 1];
    *expval = e;
    for (size_t p = 0; p < nparams; ++p) grad[p] = 0;
    for (size_t k = ng; k-- > 0;) {
        const qk_gate *g = &gates[k];
        if (pidx && pidx[k] >= 0) {
            const int gen = g->kind == QK_GATE_RX ? 1 : g->kind == QK_GATE_RY ? 2 : g->kind == QK_GATE_RZ ? 3 : 0;
            if (!gen) { free(lam); return -1; }
            const int t = g->q[0];
            const uint64_t h = 1ull << t;
            double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
            for (uint64_t p = 0; p < N / 2; ++p) {
                const uint64_t i0 = ins0(p, t), i1 = i0 + h;
                const cx a0 = ld(psi, i0), a1 = ld(psi, i1), l0 = ld(lam, i0), l1 = ld(lam, i1);
                /* Im conj(l) a = l.re a.im - l.im a.re;  Re conj(l) a = l.re a.re + l.im a.im */
                if (gen == 1) s += (l0.re * a1.im - l0.im * a1.re) + (l1.re * a0.im - l1.im * a0.re);
                else if (gen == 2) s += (l1.re * a0.re + l1.im * a0.im) - (l0.re * a1.re + l0.im * a1.im);
                else s += (l0.re * a0.im - l0.im * a0.re) - (l1.re * a1.im - l1.im * a1.re);
            }
            grad[pidx[k]] += s;
        }
        qk_gate inv;
        if (inverse_gate(g, &inv)) { free(lam); return -1; }
        qko_apply(psi, n, &inv);
        qko_apply(lam, n, &inv);
    }
    free(lam);
    return 0;
}
