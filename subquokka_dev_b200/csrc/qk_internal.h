// Internal types shared by the host code (C++) and the kernels (CUDA).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "quokka_gpu.h"

namespace qk {

// Kernel-level operation.  Every parsed gate lowers to one of these; the
// coefficients are complex FP64 values computed on the host with the
// reference's own formulas (src/circuit.cpp:2655-2991).
enum OpKind : int32_t {
    OP_DENSE1 = 0,  // 2x2 matrix m[0..3] on q[0]                 (H X Y U1 RX RY)
    OP_PHASE1 = 1,  // amplitudes with bit q[0] set *= m[0]        (Z P)
    OP_DIAG1 = 2,   // bit q[0] = 0: *= m[0], = 1: *= m[1]         (RZ)
    OP_DENSE2 = 3,  // 4x4 matrix on (q[0], q[1]), index bit0=q[0] (U2)
    OP_PHASE2 = 4,  // amplitudes with bits q[0], q[1] set *= m[0] (CP)
    OP_DIAG2 = 5,   // *= m[b0 + 2 b1]                             (RZZ)
    OP_SWAP2 = 6,   // exchange |01> and |10> of (q[0], q[1])      (SWAP, VSWAP_1_1)
    OP_PERM = 7,    // swap bit q[i] with bit q[k+i], i < k = nq/2 (VSWAP_k_k)
};

struct Op {
    int32_t kind;
    int32_t nq;
    int32_t q[QK_MAX_TARGETS];
    double m[32];  // complex coefficients, (re, im) interleaved
};

// Thread-local error message; returns code so callers can `return fail(...)`.
int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();

// Lower a parsed gate to a kernel op (host, FP64).
int lower_gate(const qk_gate &g, Op &op);

// True when the op is diagonal in the computational basis.
inline bool op_is_diagonal(const Op &op) {
    return op.kind == OP_PHASE1 || op.kind == OP_DIAG1 || op.kind == OP_PHASE2 ||
           op.kind == OP_DIAG2;
}

}  // namespace qk

// Parsed circuit container behind the opaque qk_circuit handle.
struct qk_circuit {
    std::vector<qk_gate> gates;
    std::vector<int32_t> group_sizes;
};
