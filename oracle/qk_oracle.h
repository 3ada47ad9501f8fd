/*
 * ORACLE -- test infrastructure only.  Nothing in the product links this.
 *
 * A CPU restatement, in plain C, of the reference's in-memory (MEM) gate
 * kernels, plus the FP64 references for the engine's added forms
 * (expectation values and gradients), which the reference does not have.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * and only as the checker.
 *
 * Parity pin: the restatement is checked against golden states produced by
 * the UNMODIFIED reference (oracle/_ref/quokka_ref, built by `make ref` from
 * the reference's own sources) and committed under tests/golden/.
 *
 * State layout: 2^n complex128 amplitudes as interleaved doubles, qubit q =
 * bit q of the index (src/MEM_Runner.cpp:79-99).
 */
#ifndef QK_ORACLE_H
#define QK_ORACLE_H
#include <stddef.h>
#include "quokka_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Apply one gate / a gate list in place.  Returns 0, or -1 for a gate this
 * restatement does not know. */
int qko_apply(double *state, int n, const qk_gate *g);
int qko_apply_list(double *state, int n, const qk_gate *gates, size_t ng);

/* <psi| H |psi> for H = sum_i J[i] Z_i Z_{i+1} (i < n-1) + sum_i h[i] X_i. */
double qko_expval_zz_x(const double *state, int n, const double *J, const double *h);

/* One Pauli string coeff * i^popcount(x & z) X^x Z^z (the engine's qk_pauli_term). */
typedef struct { double coeff; unsigned long long x, z; } qko_term;

/* FP64 adjoint gradient of <H> after gates[0..ng) applied to state (which is
 * overwritten): gate i with pidx[i] >= 0 is trainable (RX, RY, RZ) and adds
 * Im <lambda|G|psi> to grad[pidx[i]]; *expval receives <H>.  Returns 0, or -1
 * for a gate this restatement cannot invert or differentiate. */
int qko_adjoint_grad(double *state, int n, const qk_gate *gates, size_t ng, const int *pidx, size_t nparams,
                     const qko_term *terms, size_t nterms, double *expval, double *grad);

#ifdef __cplusplus
}
#endif
#endif
