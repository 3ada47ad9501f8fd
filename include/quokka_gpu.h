/*
 * quokka_gpu.h -- C ABI of the B200 state-vector engine (libquokka_gpu.so).
 *
 * The engine is a GPU runner for the SubQuokka simulator's in-memory path:
 * the state vector of 2^N amplitudes stays resident in HBM and every gate of
 * a circuit.txt file is applied by a hand-written sm_100a kernel.  The ABI
 * uses plain C types only (no torch, no C++), so the reference's C++ host, a
 * ctypes stub or any other FFI can bind it.  Every entry point returns an int
 * status (0 = QK_OK, negative = error); the message of the last error on the
 * calling thread is qk_last_error().  The library never exits the process.
 *
 * Conventions shared with the reference (src/MEM_Runner.cpp:79-81,
 * src/MEM_Runner.cpp:90-99): amplitude k of an N-qubit state is stored at
 * index k, qubit q is bit q of k (little-endian), each amplitude is an
 * interleaved (re, im) pair, the initial state is |0...0>.  Multi-qubit gates
 * take their targets in ascending order, as the reference's loop nests
 * require; the parser refuses anything else instead of computing a wrong
 * state.
 *
 * Threading: one host thread per qk_sv at a time; work is ordered on the
 * state's CUDA stream.  Distinct handles may be used from distinct threads.
 */
#ifndef QUOKKA_GPU_H
#define QUOKKA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QK_ABI_VERSION 3   /* 2: qk_config.init_file; 3: qk_config.device_qbit */
#define QK_MAX_TARGETS 12

/* Status codes.  The reference reports errors by printing to cerr and calling
 * exit(1) (src/simulator.cpp:190-193, :594-596, :764-774); here the same
 * conditions return one of these codes. */
typedef enum qk_status {
    QK_OK = 0,
    QK_ERR_ARG = -1,          /* bad argument, size or handle */
    QK_ERR_PARSE = -2,        /* malformed circuit/ini line, unknown gate */
    QK_ERR_QUBIT = -3,        /* target >= total qubits ("Qubit Index Error") */
    QK_ERR_ORDER = -4,        /* multi-qubit targets not strictly ascending */
    QK_ERR_IO = -5,           /* file could not be opened or read */
    QK_ERR_CUDA = -6,         /* a CUDA runtime call failed */
    QK_ERR_OOM = -7,          /* device allocation failed */
    QK_ERR_UNSUPPORTED = -8,  /* valid input that this engine does not run */
    QK_ERR_NOT_BUILT = -9     /* the CUDA code for this call is missing */
} qk_status;

/* Amplitude type of a state: complex128 (the reference's type) or complex64. */
typedef enum qk_dtype { QK_C128 = 0, QK_C64 = 1 } qk_dtype;

/* Gate kinds: the gate tokens of the reference's MEM parser
 * (Simulator::setGate_MEM, src/simulator.cpp:542-597). */
typedef enum qk_gate_kind {
    QK_GATE_H = 1,          /* "H q"                                         */
    QK_GATE_X = 2,          /* "X q"                                         */
    QK_GATE_Y = 3,          /* "Y q"                                         */
    QK_GATE_Z = 4,          /* "Z q"                                         */
    QK_GATE_P = 5,          /* "P q phi"                                     */
    QK_GATE_RX = 6,         /* "RX q phi"                                    */
    QK_GATE_RY = 7,         /* "RY q phi"                                    */
    QK_GATE_RZ = 8,         /* "RZ q phi"                                    */
    QK_GATE_U1 = 9,         /* "U1 q" + 4 (re im) pairs, row-major 2x2       */
    QK_GATE_U2 = 10,        /* "U2 a b" + 16 (re im) pairs, basis |a b>, a MSB */
    QK_GATE_SWAP = 11,      /* "SWAP a b"                                    */
    QK_GATE_CP = 12,        /* "CP a b phi"                                  */
    QK_GATE_RZZ = 13,       /* "RZZ a b phi"                                 */
    QK_GATE_VSWAP = 14,     /* "VSWAP_k_k" + 2k qubits: SWAP(q[i], q[k+i])  */
    QK_GATE_MPI_VSWAP = 15  /* "MPI_VSWAP_k_k", k in {1,2}: same permutation */
} qk_gate_kind;

/* One gate as parsed from a circuit.txt line.  Angles and matrices are kept
 * exactly as written; the engine derives the kernel coefficients on the host
 * in FP64 with the reference's own formulas. */
typedef struct qk_gate {
    int32_t kind;                   /* qk_gate_kind */
    int32_t nq;                     /* number of targets used in q[] */
    int32_t q[QK_MAX_TARGETS];      /* targets as written */
    double param;                   /* phi of P, RX, RY, RZ, CP, RZZ */
    double coeff[32];               /* U1: 4, U2: 16 complex (re, im) in file order */
} qk_gate;

/* The [system] keys of the reference's .ini (setSEG/setENV,
 * src/simulator.cpp:88-186) plus the engine's own optional keys, which the
 * reference ignores. */
typedef struct qk_config {
    int32_t total_qbit;       /* total_qbit, default 0                       */
    int32_t mpi_qbit;         /* mpi_qbit, default 0 (must be 0 here)        */
    int32_t file_qbit;        /* file_qbit, default 0 (advisory on the GPU)  */
    int32_t chunk_qbit;       /* chunk_qbit, default 0 (must be >= 1)        */
    int32_t is_subcircuit;    /* is_subcircuit, default 1                    */
    int32_t MPI_testing;      /* MPI_testing, default 0                      */
    int32_t MPI_buffe_size;   /* MPI_buffe_size (sic), default 16            */
    int32_t precision;        /* precision=c128|c64 -> qk_dtype, default c128 */
    int32_t fuse_width;       /* fuse_width, default 0: per-gate kernels for a
                                 flat circuit, fused passes for a subcircuit
                                 file; > 0 fused passes for a flat circuit
                                 too; 5 or 6 with precision=c64 tensor-core
                                 blocks for either                           */
    int32_t dump_binary;      /* dump_format=bin -> 1, default 0 (text)      */
    char runner_type[32];     /* runner_type, default "IO"; "GPU" selects us */
    char dump_file[256];      /* dump_file, default ""                       */
    char init_file[256];      /* init_file, default "": a state file
                                 (qk_sv_load) to start from instead of
                                 |0...0>                                     */
    int32_t device_qbit;      /* device_qbit, default 0: with runner_type IO
                                 or DirectIO the state lives in host memory
                                 (qk_hsv) and the GPU takes chunks of
                                 2^device_qbit amplitudes; 0 = the largest
                                 that fits three chunks in free HBM         */
} qk_config;

typedef struct qk_circuit qk_circuit;   /* parsed gate list (+ group sizes) */
typedef struct qk_sv qk_sv;             /* device-resident state vector     */

/* ---- errors and version ------------------------------------------------ */

/* Message of the last failed call on this thread ("" if none). */
const char *qk_last_error(void);
/* QK_ABI_VERSION of the loaded library. */
int qk_abi_version(void);

/* ---- configuration and circuit files (host only) ----------------------- */

/* Read an .ini file.  Replaces setSEG + setENV (src/simulator.cpp:88-186):
 * same keys, same defaults, and the reference's asserts (chunk_qbit >= 1,
 * total_qbit >= file_qbit + chunk_qbit) become QK_ERR_ARG. */
int qk_config_load(const char *ini_path, qk_config *out);

/* Parse one gate line.  Replaces Simulator::setGate_MEM and its builders
 * (src/simulator.cpp:259-356, :542-597) and check_targ_in_N (:764-774). */
int qk_gate_parse_line(const char *line, int total_qbit, qk_gate *out);

/* Parse a whole circuit file.  is_subcircuit = 0: one gate per line
 * (setupCircuit_MEM, src/simulator.cpp:601-615); is_subcircuit = 1: a count
 * line followed by that many gate lines, repeated
 * (setupSubCircuits_MEM, src/simulator.cpp:619-636). */
int qk_circuit_load(const char *path, int is_subcircuit, int total_qbit, qk_circuit **out);
/* Same, from an in-memory text. */
int qk_circuit_parse(const char *text, int is_subcircuit, int total_qbit, qk_circuit **out);
size_t qk_circuit_num_gates(const qk_circuit *c);
const qk_gate *qk_circuit_gates(const qk_circuit *c);
/* Number of groups and their sizes (one group per gate for flat files). */
size_t qk_circuit_num_groups(const qk_circuit *c);
const int32_t *qk_circuit_group_sizes(const qk_circuit *c);
void qk_circuit_destroy(qk_circuit *c);

/* Dense matrix of one gate over its targets in little-endian target order
 * (row r, column c; bit i of r is target q[i]), FP64, built with the
 * reference's coefficient formulas (src/circuit.cpp:2655-2991).
 * out must hold 2 * 4^nq doubles; *dim receives 2^nq.  VSWAP gates are
 * permutation matrices of dimension 2^(2k). */
int qk_gate_matrix(const qk_gate *g, double *out, int *dim);

/* Group a flat gate list into a subcircuit file for the reference's
 * subcircuit runner: the job of subcircuitFinder (subcircuitFinder/finder.cpp:
 * 771-877), for every gate of the MEM grammar and any chunk size.  Every
 * compute group acts on bit positions below chunk_qbit only; single-gate
 * groups `VSWAP_1_1 a c` / `VSWAP_2_2 a b c d` (a < b < chunk_qbit <= c < d)
 * move other qubits into the chunk; at the end the state is back in the
 * input's layout, so the grouped file computes the same state as the flat
 * one.  VSWAP gates of the input are absorbed as renamings.  *out is a new
 * circuit (free with qk_circuit_destroy). */
int qk_circuit_chunk_groups(const qk_gate *gates, size_t n, int nqubits, int chunk_qbit, qk_circuit **out);
/* Write a circuit in the circuit.txt grammar: one gate per line
 * (is_subcircuit = 0) or group-count lines each followed by its gates
 * (is_subcircuit = 1); numbers with 17 significant digits. */
int qk_circuit_write(const qk_circuit *c, int is_subcircuit, const char *path);

/* ---- state vectors ----------------------------------------------------- */

/* Allocate a 2^nqubits state on the current CUDA device and set it to
 * |0...0>.  Replaces MEM_Runner::MEM_Runner (src/MEM_Runner.cpp:57-88). */
int qk_sv_create(int nqubits, int dtype, qk_sv **out);
void qk_sv_destroy(qk_sv *sv);
/* Set |0...0>. */
int qk_sv_reset(qk_sv *sv);
/* Copy a host complex128 state (2^n interleaved pairs) in / out.  For a
 * complex64 state the values are converted on the device. */
int qk_sv_upload(qk_sv *sv, const double *host_c128);
int qk_sv_download(qk_sv *sv, double *host_c128);
/* Write / read a state file: raw little-endian complex128, 2^n interleaved
 * (re, im) pairs (16 * 2^n bytes), the layout of dump_format=bin.  A
 * complex64 state is widened on write and rounded on read; a file of any
 * other size is refused.  The reference writes only its text dump
 * (src/simulator.cpp:696-704) and reads no state. */
int qk_sv_save(qk_sv *sv, const char *path);
int qk_sv_load(qk_sv *sv, const char *path);
/* Shape, type, device pointer and byte size of a state. */
int qk_sv_info(const qk_sv *sv, int *nqubits, int *dtype, void **device_ptr, size_t *bytes);
/* Order the state's work on a caller's cudaStream_t (NULL = default). */
int qk_sv_set_stream(qk_sv *sv, void *cuda_stream);
/* Wait for all work queued on the state's stream. */
int qk_sv_synchronize(qk_sv *sv);
/* Free the device workspace that adjoint sweeps and expectation values keep
 * with the state (lambda, checkpoints, accumulators, pass programs).  The
 * reference has no counterpart (its runner allocates nothing besides the
 * state, src/MEM_Runner.cpp:57-88). */
int qk_sv_release_workspace(qk_sv *sv);

/* ---- the hot path ------------------------------------------------------ */

/* Per-gate path: apply gates[0..n) in order, one state sweep per gate.
 * Replaces MEM_Runner::run(std::vector<Gate*>&) (src/MEM_Runner.cpp:101-134).
 * Asynchronous on the state's stream. */
int qk_apply_gates(qk_sv *sv, const qk_gate *gates, size_t n);

/* Subcircuit path: gates are split into consecutive groups of
 * group_sizes[0..ngroups) gates.  The result is the state the reference's
 * subcircuit runner computes, with fewer state sweeps:
 * - VSWAP groups move no amplitudes: they rename the qubits of the gates
 *   after them, and one or two permutation rounds at the end bring the state
 *   into the file's layout;
 * - the gates of all other groups are fused into shared-memory-resident
 *   passes as qk_plan_create fuses a flat list, across group bounds.
 * Replaces MEM_Runner::run(std::vector<std::vector<Gate*>>&)
 * (src/MEM_Runner.cpp:136-185).  Asynchronous on the state's stream. */
int qk_apply_groups(qk_sv *sv, const qk_gate *gates, const int32_t *group_sizes, size_t ngroups);

/* Per-gate path on caller-owned device memory (for example a torch tensor):
 * state points to 2^nqubits amplitudes of dtype on the current device,
 * cuda_stream is a cudaStream_t (NULL = default). */
int qk_apply_gates_dev(void *state, int nqubits, int dtype, const qk_gate *gates, size_t n,
                       void *cuda_stream);

/* The per-gate path (qk_apply_gates' launches) captured once as a CUDA
 * graph bound to sv's state and replayed on sv's stream: the same kernels and
 * results, one launch for the whole gate list.  For small states, where a
 * gate's kernel runs for about as long as the host takes to launch it.  The
 * graph must not outlive sv.  No reference counterpart (MEM_Runner::run
 * loops over the gates, src/MEM_Runner.cpp:101-134). */
typedef struct qk_graph qk_graph;
int qk_graph_create(qk_sv *sv, const qk_gate *gates, size_t ngates, qk_graph **out);
int qk_graph_launch(qk_graph *g);
void qk_graph_destroy(qk_graph *g);

/* Per-gate path with a CUDA event pair around every gate's kernel on the
 * state's stream; gate_ms[i] receives gate i's device time in milliseconds.
 * Synchronises the stream before returning.  Used for per-kernel rooflines. */
int qk_apply_gates_timed(qk_sv *sv, const qk_gate *gates, size_t n, float *gate_ms);

/* ---- fused passes ------------------------------------------------------ */

/* Options of a fused plan; zero fields take the defaults. */
typedef struct qk_plan_opts {
    int32_t dtype;        /* qk_dtype of the states the plan runs on        */
    int32_t tile_bits;    /* qubits per shared-memory tile (default 11; at
                             most 14)                                       */
    int32_t reg_bits;     /* qubits held in registers per thread (default 4;
                             at most 5)                                     */
    int32_t fuse_width;   /* 0: register passes.  5 or 6: gates fused into
                             dense unitaries on at most that many qubits
                             (FP64 on the host, padded to 6 qubits), each
                             applied as a 64 x 64 complex contraction on the
                             tensor cores, for states of >= 12 qubits:
                             complex64 in split precision (3 x BF16, FP32
                             accumulate); complex128 exactly in integer
                             arithmetic (seven 8-bit digits an operand row,
                             int8 products, int32 accumulate, FP64
                             recombination), within about 2^-48 of FP64 */
    int32_t reserved[4];
} qk_plan_opts;

typedef struct qk_plan qk_plan;

/* Fuse a flat gate list into passes: each pass is one HBM read and write of
 * the state that applies every gate it carries in shared memory and
 * registers.  This replaces the reference's two-step recipe -- group gates
 * into 12-qubit chunks with subcircuitFinder (subcircuitFinder/finder.cpp:
 * 629-698) and run the groups chunk by chunk (src/MEM_Runner.cpp:172-183) --
 * for any circuit, with no VSWAP: a tile's qubits need not be contiguous.
 * VSWAP gates of the list rename qubits instead of moving amplitudes, and so
 * do SWAP gates when that gives fewer passes; a final permutation restores
 * the layout. */
int qk_plan_create(const qk_gate *gates, size_t n, int nqubits, const qk_plan_opts *opts, qk_plan **out);
/* The plan of a subcircuit file that qk_apply_groups runs: the gates of all
 * groups fused as one list, VSWAPs as renamings of the qubits after them.
 * With opts->fuse_width 5 or 6: tensor-core dense blocks over the same list,
 * as qk_plan_create makes them. */
int qk_plan_create_groups(const qk_gate *gates, const int32_t *group_sizes, size_t ngroups, int nqubits,
                          const qk_plan_opts *opts, qk_plan **out);
/* Number of passes, program operations and register re-mappings. */
int qk_plan_stats(const qk_plan *p, size_t *passes, size_t *program_ops, size_t *remaps);
/* Block k of a fuse_width = 5 or 6 plan (host data): its six qubits ascending
 * (local index bit b = qubits[b]) and its 64 x 64 unitary, row-major complex
 * (re, im) in u[2 * 64 * 64]; *is_perm = 1 for a VSWAP kept as a permutation
 * (qubits then holds its targets, unused entries -1). */
int qk_plan_dense_block(const qk_plan *p, size_t k, int32_t *qubits, double *u, int *is_perm);
/* Run a plan on a state (same qubit count and dtype).  The first call copies
 * the plan's programs to the device (owned by the plan). */
int qk_plan_apply(qk_sv *sv, qk_plan *p);
void qk_plan_destroy(qk_plan *p);

/* ---- observables and gradients ----------------------------------------- */
/* No counterpart in the reference, which computes no observables or
 * gradients: these serve variational workloads built on the same gates. */

/* One real-weighted Pauli string: coeff * i^popcount(x & z) X^x Z^z, i.e.
 * qubit q carries X if only bit q of x_mask is set, Z if only bit q of
 * z_mask is set, Y if both are. */
typedef struct qk_pauli_term {
    double coeff;
    uint64_t x_mask;
    uint64_t z_mask;
} qk_pauli_term;

/* <psi| H |psi> for H = sum of the terms (one state sweep per distinct
 * x_mask; the state is not modified). */
int qk_expval_pauli(qk_sv *sv, const qk_pauli_term *terms, size_t nterms, double *out);

/* Adjoint gradient of <H> after gates[0..ngates) applied to the state in sv.
 * Gate i with param_index[i] >= 0 is trainable (RX, RY or RZ; its angle is
 * the current value); gradients of gates sharing an index add up into
 * grad[index] (nparams entries).  The forward state is uncomputed gate by gate
 * (U^dag) instead of stored; `checkpoints` forward states (-1: min(8,
 * ceil(sqrt(ngates))), 0: none) are kept at evenly spaced gates, and when the
 * backward sweep reaches one, the uncomputed state is replaced by it; *drift
 * receives the root sum of squared differences found there.  *expval
 * receives <H>.  On return sv holds the initial state again (uncomputed, or
 * restored from the first checkpoint).  Device memory: one extra state plus
 * the checkpoints, kept by sv as its workspace for the next call (grown when
 * a call needs more) until qk_sv_release_workspace or qk_sv_destroy. */
int qk_adjoint_grad(qk_sv *sv, const qk_gate *gates, size_t ngates, const int32_t *param_index, size_t nparams,
                    const qk_pauli_term *terms, size_t nterms, int checkpoints, double *expval, double *grad,
                    double *drift);

/* qk_adjoint_grad with fused passes: the gates are cut into segments at the
 * checkpoints (-1: about sqrt(ngates)/4, at most 8); every segment runs
 * forward as fused passes and backward as two-state passes that apply the
 * inverse gates to psi and lambda and take each gradient inside the pass.
 * Same arguments and results. */
int qk_adjoint_grad_fused(qk_sv *sv, const qk_gate *gates, size_t ngates, const int32_t *param_index, size_t nparams,
                          const qk_pauli_term *terms, size_t nterms, int checkpoints, double *expval, double *grad,
                          double *drift);

/* No counterpart in the reference.  Device time of the last qk_adjoint_grad /
 * qk_adjoint_grad_fused on sv (CUDA events on the state's stream, from its
 * first device operation to its last; host planning excluded), the bytes its
 * kernels and copies must read and write (fused sweeps: 2S per forward pass,
 * 4S per two-state pass, plus the H application, reductions and checkpoint
 * copies; 0 for the per-gate sweep, whose traffic is not counted), and its
 * forward and backward pass (or, per-gate, launch) counts. */
int qk_sv_last_sweep(const qk_sv *sv, double *device_ms, double *alg_bytes, int *forward_passes,
                     int *backward_passes);

/* ---- batches of variational circuits ------------------------------------ */
/* No counterpart in the reference.  Many circuits of different sizes, each
 * with its own trainable RX/RY/RZ gates and Pauli-sum H: <H> and the adjoint
 * gradient of every circuit from one CUDA graph.  Step k of the batch is one
 * persistent kernel launch that runs the k-th fused pass of every circuit. */

typedef struct qk_batch_opts {
    int32_t dtype;          /* qk_dtype of the states (default complex64)     */
    int32_t autotune;       /* 1: time candidate tile shapes on the batch and
                               keep the fastest                                */
    int32_t tile_bits, reg_bits;          /* forward passes (0 = default)     */
    int32_t adj_tile_bits, adj_reg_bits;  /* adjoint passes (0 = default)     */
    int32_t reserved[2];
} qk_batch_opts;

typedef struct qk_batch qk_batch;

/* Circuit c has nqubits[c] qubits and gate_counts[c] gates (concatenated in
 * gates); param_index (one entry per gate, concatenated; NULL = none
 * trainable) indexes that circuit's own param_counts[c] parameters; its H is
 * term_counts[c] terms (concatenated).  Builds the plans, allocates every
 * state and captures the graph. */
int qk_batch_create(int ncirc, const int32_t *nqubits, const qk_gate *gates, const size_t *gate_counts,
                    const int32_t *param_index, const size_t *param_counts, const qk_pauli_term *terms,
                    const size_t *term_counts, const qk_batch_opts *opts, qk_batch **out);
/* Run the graph: every circuit from |0...0>.  expvals[c], grads (all
 * parameters, circuit by circuit), drift[c] = || uncomputed state - |0..0> ||. */
int qk_batch_run(qk_batch *b, double *expvals, double *grads, double *drift);
/* New values of all parameters (circuit by circuit); the next run uses them. */
int qk_batch_set_params(qk_batch *b, const double *params);
/* Graph steps, kernel launches per run and the chosen tile shapes. */
int qk_batch_stats(const qk_batch *b, int *steps, int *launches, int *tile_bits, int *reg_bits, int *adj_tile_bits,
                   int *adj_reg_bits);
/* Device time of the last qk_batch_run (CUDA events around the graph launch
 * on the batch's stream) and the bytes one run must read and write: per
 * circuit of S bytes, 2S per forward pass, 4S per two-state pass, S for the
 * reset, 2S for lambda = H psi, S for the drift check. */
int qk_batch_timing(const qk_batch *b, double *device_ms, double *alg_bytes);
void qk_batch_destroy(qk_batch *b);

/* ---- fused passes without device allocation --------------------------- */

/* Bytes of device memory, fixed at load time, that hold the pass programs and
 * coefficients of one qk_apply_fused_noalloc call. */
#define QK_NOALLOC_SCRATCH_BYTES (1u << 20)

/* No counterpart in the reference (its runner allocates nothing on a GPU).
 * The fused-pass path for callers that cannot allocate device memory -- a
 * process whose HBM is all handed to a memory pool or to its own state
 * vectors, or a loop that must not stall other streams on a cudaMalloc /
 * cudaFree.  Same result as qk_plan_create + qk_plan_apply with default
 * options on caller-owned memory (state: 2^nqubits amplitudes of dtype on the
 * current device; cuda_stream: a cudaStream_t, NULL = default), but the pass
 * programs go to a fixed __device__ array of QK_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit; a circuit whose programs do
 * not fit returns QK_ERR_ARG.  The first call on a device looks up that
 * array's address (make it before any stream capture on the device) and keeps
 * it, so the library must not be used across a cudaDeviceReset.  Every call
 * shares the array and overwrites it: calls that overlap on the GPU
 * (unordered streams) race; calls on one stream are safe.  The programs are
 * copied from host memory the call frees, so it waits for those copies before
 * returning, and a call on a stream under capture returns QK_ERR_UNSUPPORTED. */
int qk_apply_fused_noalloc(void *state, int nqubits, int dtype, const qk_gate *gates, size_t n, void *cuda_stream);

/* ---- states larger than HBM: host memory, GPU compute ------------------- */

typedef struct qk_hsv qk_hsv;   /* host-resident state vector */

/* Replaces IO_Runner (src/IO_Runner.cpp:309-488, state in files, chunks of
 * 2^chunk_qbit run on the host cores) for states that do not fit in HBM: the
 * 2^nqubits amplitudes of dtype live in pinned host memory (index k = the
 * in-memory layout, never permuted), and the GPU holds three buffers of
 * 2^chunk_qubits amplitudes.  Starts in |0...0>. */
int qk_hsv_create(int nqubits, int chunk_qubits, int dtype, qk_hsv **out);
/* |0...0> again. */
int qk_hsv_reset(qk_hsv *h);
/* The host amplitudes: 2^nqubits interleaved (re, im) doubles (complex128)
 * or floats (complex64); read or write them between calls. */
void *qk_hsv_data(qk_hsv *h);
/* Apply gates[0..n).  The gates are cut into segments whose qubits fit in
 * chunk_qubits "local" qubits; each segment is one sweep that copies every
 * chunk (the amplitudes sharing one value of the other qubits) to the GPU,
 * runs the segment's fused passes on it and copies it back, copies and
 * compute overlapped on three streams.  A qubit enters the local set by a
 * change of the copy addresses, not by moving amplitudes (the reference's
 * VSWAP).  Synchronous: returns when the host state holds the result. */
int qk_hsv_apply_gates(qk_hsv *h, const qk_gate *gates, size_t n);
/* Segments of the last qk_hsv_apply_gates, its device time (CUDA events from
 * the first copy-in to the last copy-out) and the bytes it moved over the
 * host link (2 x state bytes per segment). */
int qk_hsv_stats(const qk_hsv *h, int *segments, double *device_ms, double *link_bytes);
void qk_hsv_destroy(qk_hsv *h);
/* The segmentation qk_hsv_apply_gates uses (host only): *nsegments; when it
 * is <= cap, per segment its local qubit mask and gate count, and in order[]
 * (n entries) the gate indices in execution order, segment after segment. */
int qk_ooc_segments(const qk_gate *gates, size_t n, int nqubits, int chunk_qubits, uint64_t *local_masks,
                    int32_t *segment_sizes, int32_t *order, size_t cap, size_t *nsegments);

/* Run a parsed circuit the way Simulator::run does (src/simulator.cpp:671-706):
 * groups if cfg->is_subcircuit, else gates (fused passes if cfg->fuse_width >
 * 0); *seconds receives the device time of the runner span alone. */
int qk_run(const qk_config *cfg, const qk_circuit *c, qk_sv *sv, double *seconds);

#ifdef __cplusplus
}
#endif
#endif /* QUOKKA_GPU_H */
