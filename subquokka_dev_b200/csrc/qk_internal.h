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
    OP_SWAP2 = 6,   // exchange |01> and |10> of (q[0], q[1])      (SWAP, VSWAP_1_1: aux = 1)
    OP_PERM = 7,    // swap bit q[i] with bit q[k+i], i < k = nq/2 (VSWAP_k_k)
    OP_GRAD = 8,    // adjoint sweep: grad[aux] += Im <lambda|G|psi>, G on q[0] = X/Y/Z by m[0] = 1/2/3
    OP_CX = 9,      // flip bit q[1 - aux] where bit q[aux] is set (a U2 that is exactly a CNOT)
    OP_CDENSE1 = 10,  // 2x2 on q[0]: m[0..7] where bit q[1] is 0, m[8..15] where it is 1 (planner-made)
};

struct Op {
    int32_t kind;
    int32_t nq;
    int32_t q[QK_MAX_TARGETS];
    int32_t aux;   // OP_GRAD: parameter index; OP_CX: control index; OP_SWAP2 / OP_PERM: 1 from a VSWAP
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

// Qubits of an op that a fused pass must hold in registers: q[reg_first(op)
// .. + reg_count(op)).  None for diagonal ops, the target for OP_CX and
// OP_CDENSE1 (the control / condition may be any qubit, as for a diagonal
// op), all of them otherwise.
inline int op_reg_count(const Op &op) {
    return op_is_diagonal(op) ? 0 : (op.kind == OP_CX || op.kind == OP_CDENSE1) ? 1 : op.nq;
}
inline int op_reg_first(const Op &op) { return op.kind == OP_CX ? 1 - op.aux : 0; }

}  // namespace qk

// Parsed circuit container behind the opaque qk_circuit handle.
struct qk_circuit {
    std::vector<qk_gate> gates;
    std::vector<int32_t> group_sizes;
};

namespace qk {

// ---------------------------------------------------------------------------
// Fused passes.  A pass stages tiles of 2^T amplitudes (tile bits bpos[0..T))
// and runs a small program on them; each thread keeps R = 2^r amplitudes in
// registers, indexed by r "register" tile bits, the rest of the tile bits
// index the thread.  Programs are built on the host (qk_plan.cpp).
// ---------------------------------------------------------------------------
constexpr int kPassMaxBits = 14;
constexpr int kPassMaxReg = 5;

enum TOpKind : uint8_t {
    TOP_REMAP = 0,  // re-distribute the tile: register slot s <- tile bit bits[s]
    TOP_G1 = 1,     // dense 2x2 on register slot a; coef -> 4 complex
    TOP_G2 = 2,     // dense 4x4 on register slots a < b (index bit0 = a); coef -> 16 complex
    TOP_DIAG = 3,   // amplitude *= coef[bit(a) + 2 bit(b)]; a, b are qubit codes
    TOP_PHASE = 4,  // amplitude *= coef[0] where bit(a) = bit(b) = 1 (Z, P, CP; b may be none)
    TOP_GRAD = 5,   // two-state passes: gacc[coef] += Im <lambda|G|psi>, G = X/Y/Z (b = 1/2/3) on slot a
    TOP_CX = 6,     // swap register slot a's pairs where qubit code b is 1 (controlled X)
    TOP_CG1 = 7,    // dense 2x2 on slot a: coef[0..3] or coef[4..7] by qubit code b (not a register slot)
    TOP_R1 = 8,     // real 2x2 on slot a: coef[0] = (m00, m01), coef[1] = (m10, m11)
    TOP_R2 = 9,     // real 4x4 on slots a < b (index bit0 = a): coef[2 r + h] = (m[r][2h], m[r][2h + 1])
};
// The kernel instance for passes marked xops carries factors that are the
// same for all of a thread's amplitudes (TOP_DIAG / TOP_PHASE on qubits
// outside the register slots) as one pending scalar, applied before the
// tile is re-distributed or stored -- except where the register amplitudes
// take 256 bytes or more (complex128 with 16 a thread, two states of 8
// complex128 or 16 complex64): those kernels run at their register limit,
// and the scalar's registers cost spills.
constexpr bool pending_scalar_ok(int amp_bytes, int reg_amps, int nstates) {
    return amp_bytes * reg_amps * nstates < 256;
}

// Qubit codes of TOP_DIAG / TOP_PHASE: < 0x80 tile-local bit; 0x80 | q global
// qubit q that is not a tile bit (constant over a tile); 0xFF no qubit (bit =
// 0 for TOP_DIAG, 1 for TOP_PHASE).
constexpr uint8_t kOuterFlag = 0x80;
constexpr uint8_t kNoQubit = 0xFF;

struct TOp {
    uint8_t kind;
    uint8_t a, b;
    uint8_t nbits;
    uint8_t bits[kPassMaxReg + 3];
    uint32_t coef;
};
static_assert(sizeof(TOp) == 16, "TOp must stay 16 bytes");
constexpr uint8_t kNoSlot = 0xFF;   // TOp.bits[k] of a condition qubit held in no register slot

struct PassDesc {
    int32_t T;                    // tile bits
    int32_t L;                    // tile bits 0..L-1 are state bits 0..L-1 (contiguous runs)
    int32_t bpos[kPassMaxBits];   // state bit of each tile bit, ascending
    int32_t prog0, nprog;         // program slice in the plan's op array
    int32_t coef0, ncoef;         // coefficient slice (complex values) used by the program
    int32_t grad0, ngrad;         // gradient slots of the pass: plan.grad_params[grad0 .. grad0 + ngrad)
    int32_t perm;                 // 1: a qubit-permutation pass (VSWAP), prog unused
    int32_t nperm;
    int32_t perm_a[6], perm_b[6]; // tile-local bit pairs swapped on store (perm passes)
    int32_t xops;                 // 1: the program has real or diagonal ops (TOP_R1, TOP_R2, TOP_DIAG,
                                  // TOP_PHASE), run by the kernel instance that specialises them
};

// Host plan: passes + programs + complex coefficient pool (FP64).
struct HostPlan {
    int n = 0;
    int dtype = 0;
    int T = 0, r = 0;
    std::vector<PassDesc> passes;
    std::vector<TOp> ops;
    std::vector<double> coef;  // (re, im) pairs
    std::vector<int32_t> grad_params;  // parameter index of each pass's gradient slots
    int nstates = 1;           // 2: adjoint passes over (psi, lambda)
    size_t nremaps = 0, ngates = 0;
};

struct PlanOptions {
    int dtype;
    int tile_bits;   // T
    int reg_bits;    // r
    int plain_ops = 0;    // 1: no TOP_R1 / TOP_R2 (real ops as TOP_G1 / TOP_G2) and no pass marked
                          // xops (plans of the batched kernel, which has one instance)
};

// Build a fused plan for a flat gate list (greedy tile-bit choice).
int build_plan(const qk_gate *gates, size_t ng, int n, const PlanOptions &o, HostPlan &plan);
// One permutation pass (an OP_PERM of 1 to 6 bit pairs), with no program.
int build_perm_plan(const Op &op, int n, const PlanOptions &o, HostPlan &plan);
// Op-list rewrites before planning (qk_rewrite.cpp).
bool one_qubit(const Op &op);
void as_matrix(const Op &op, double (&m)[8]);
void mat2_mul(const double (&x)[8], const double (&y)[8], double (&z)[8]);
void asap_order(std::vector<Op> &ops, int n);
void merge_one_qubit_runs(std::vector<Op> &ops, int n);
void absorb_into_two_qubit_ops(std::vector<Op> &ops, int n, bool keep_real = false);
bool op_is_real(const Op &op);
void hoist_gradients(std::vector<Op> &ops, int n);
void pair_gradients(std::vector<Op> &ops);
void relabel_perms(std::vector<Op> &ops, int n, int L, int max_bits, int max_pairs, bool swaps);
// Plan of a subcircuit file (the subcircuit path): the gates of all groups
// as one gate list, VSWAPs as renamings of the qubits after them.
int build_group_plan(const qk_gate *gates, const int32_t *sizes, size_t ngroups, int n, const PlanOptions &o,
                     HostPlan &plan);
PlanOptions default_plan_options(int dtype, int n);

// Dense fused blocks: consecutive gates on at most kDenseQubits qubits
// multiplied (FP64, host) into one 2^k x 2^k unitary, applied as a
// tensor-core contraction.  A block with perm != 0 is a VSWAP instead.
constexpr int kDenseQubits = 6;
constexpr int kDenseDim = 1 << kDenseQubits;
struct DenseBlock {
    int q[kDenseQubits];               // block qubits, ascending; local bit b = q[b]
    std::vector<double> u;             // 64 x 64 complex, row-major, (re, im)
    int perm = 0;                      // VSWAP: the Op below instead of u
    Op perm_op;
    int ngates = 0;
};
// width (5 or 6): most qubits a block's gates may touch; blocks are padded to
// kDenseQubits with idle qubits.  dtype sets the tile limits of the
// permutation blocks.
int build_dense_blocks(const qk_gate *gates, size_t ng, int n, int width, int dtype, std::vector<DenseBlock> &blocks);

// A dense block's pass over the state: a supertile is the block's qubits plus
// the lowest other state bits (tile-local bits ascending in state position).
struct DenseDesc {
    PassDesc p;         // tile bits T, contiguous run L
    uint32_t blockmask; // tile-local bits that are the block's qubits
};
DenseDesc dense_block_desc(const DenseBlock &b, int n, int max_tile_bits);

// complex128 blocks (qk_dense_i8.cu): 64 x 64 supertiles; the operand of a
// block is its digit planes (128 rows x 224 words) and 128 row scales.
constexpr int kI8TileBits = 12;
constexpr int kI8Digits = 7;
constexpr size_t kI8OperandWords = 128 * 32 * kI8Digits;
constexpr size_t kI8OperandBytes = kI8OperandWords * 4 + 128 * sizeof(double);
void dense_i8_operand(const DenseBlock &b, std::vector<uint32_t> &out);   // kI8OperandBytes / 4 words
// complex64 blocks (qk_dense_tc.cu): W split into bf16 hi and lo operands
void dense_block_operand(const DenseBlock &b, std::vector<uint16_t> &out);   // 2 x 128 x 128
// Bytes of one block's device operand for dtype.
size_t dense_operand_bytes(int dtype);
// Backward sweep of an adjoint gradient: the inverses of gates[ng-1..0] on
// (psi, lambda), with the gradient of trainable gates (pidx[i] >= 0) taken
// just before their inverse.
int build_adjoint_plan(const qk_gate *gates, size_t ng, const int32_t *pidx, int n, const PlanOptions &o,
                       HostPlan &plan);
PlanOptions default_adjoint_options(int dtype, int n);
void invert_op(Op &op);

}  // namespace qk
