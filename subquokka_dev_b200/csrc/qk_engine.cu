// State handles, kernel dispatch and the hot-path entry points of the C ABI.
//
// qk_apply_gates is the GPU counterpart of MEM_Runner::run(vector<Gate*>&)
// (src/MEM_Runner.cpp:101-134): gates in order, one state sweep each.
// qk_apply_groups is the counterpart of MEM_Runner::run(vector<vector<Gate*>>&)
// (src/MEM_Runner.cpp:136-185): every gate group becomes one shared-memory
// tile pass over the state.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "qk_device.h"
#include "qk_internal.h"
#include "qk_kernels.cuh"

using namespace qk;

namespace qk {
struct DevPlan;
void release_scratch_plan(DevPlan &dp);
int apply_group_plan(qk_sv *sv, const qk_gate *gates, const int32_t *sizes, size_t ngroups);
int apply_perm_gate(void *state, int n, int dtype, const Op &op, cudaStream_t st);
int plan_prepare(qk_sv *sv, qk_plan *p);
}  // namespace qk

// qk_pass.cu's DevPlan, defined there; the state keeps one as scratch for the
// subcircuit path (device copy of the last group plan's programs).
#include "qk_devplan.h"

struct qk_sv {
    int n = 0;
    int dtype = QK_C128;
    void *d = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    qk::DevPlan scratch;
    qk::Workspace ws;   // adjoint sweeps: lambda, checkpoints, programs
    int device = 0;
};

namespace qk {

DevPlan &state_scratch_plan(qk_sv *sv) { return sv->scratch; }
cudaStream_t state_stream(const qk_sv *sv) { return sv->stream; }
void *state_ptr(const qk_sv *sv) { return sv->d; }
Workspace &state_workspace(qk_sv *sv) { return sv->ws; }
int state_qubits(const qk_sv *sv) { return sv->n; }
int state_dtype(const qk_sv *sv) { return sv->dtype; }

__global__ void k_c128_to_c64(const double2 *in, float2 *out, uint64_t namp) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < namp; e += (uint64_t)gridDim.x * blockDim.x)
        out[e] = make_float2((float)in[e].x, (float)in[e].y);
}

__global__ void k_c64_to_c128(const float2 *in, double2 *out, uint64_t namp) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < namp; e += (uint64_t)gridDim.x * blockDim.x)
        out[e] = make_double2((double)in[e].x, (double)in[e].y);
}

static int cuda_fail(cudaError_t e, const char *what) {
    // An allocation failure is not sticky, but it stays as the thread's last
    // error; clear it so the next launch check does not report it again.
    if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? QK_ERR_OOM : QK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define QK_CUDA(call)                                   \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

static int num_sms() { return device_sms(); }

static unsigned sweep_blocks(uint64_t items) {
    return (unsigned)std::max<uint64_t>(1, (items + kBlock * kUnroll - 1) / (kBlock * kUnroll));
}

// ---- per-gate dispatch ------------------------------------------------------

template <typename C>
static int launch_op(C *s, int n, const Op &op, cudaStream_t st) {
    const uint64_t namp = 1ull << n;
    switch (op.kind) {
    case OP_DENSE1: {
        Mat2<C> m;
        for (int k = 0; k < 4; ++k) m.m[k] = mk<C>(op.m[2 * k], op.m[2 * k + 1]);
        const int t = op.q[0];
        if (t < 5) k_dense1_lane<C><<<sweep_blocks(namp), kBlock, 0, st>>>(s, namp, t, m);
        else k_dense1_pair<C><<<sweep_blocks(namp / 2), kBlock, 0, st>>>(s, namp / 2, t, m);
        break;
    }
    case OP_PHASE1:
        k_phase1<C><<<sweep_blocks(namp / 2), kBlock, 0, st>>>(s, namp / 2, op.q[0], mk<C>(op.m[0], op.m[1]));
        break;
    case OP_DIAG1:
        k_diag1<C><<<sweep_blocks(namp), kBlock, 0, st>>>(s, namp, op.q[0], mk<C>(op.m[0], op.m[1]),
                                                          mk<C>(op.m[2], op.m[3]));
        break;
    case OP_DENSE2: {
        Mat4<C> m;
        for (int k = 0; k < 16; ++k) m.m[k] = mk<C>(op.m[2 * k], op.m[2 * k + 1]);
        k_dense2<C><<<sweep_blocks(namp / 4), kBlock, 0, st>>>(s, namp / 4, op.q[0], op.q[1], m);
        break;
    }
    case OP_PHASE2:
        k_phase2<C><<<sweep_blocks(namp / 4), kBlock, 0, st>>>(s, namp / 4, op.q[0], op.q[1],
                                                               mk<C>(op.m[0], op.m[1]));
        break;
    case OP_DIAG2: {
        Diag4<C> d;
        for (int k = 0; k < 4; ++k) d.d[k] = mk<C>(op.m[2 * k], op.m[2 * k + 1]);
        k_diag2<C><<<sweep_blocks(namp), kBlock, 0, st>>>(s, namp, op.q[0], op.q[1], d);
        break;
    }
    case OP_SWAP2: {
        const int a = std::min(op.q[0], op.q[1]), b = std::max(op.q[0], op.q[1]);
        k_swap2<C><<<sweep_blocks(namp / 4), kBlock, 0, st>>>(s, namp / 4, a, b);
        break;
    }
    case OP_CX:
        k_cx<C><<<sweep_blocks(namp / 4), kBlock, 0, st>>>(s, namp / 4, op.q[op.aux], op.q[1 - op.aux]);
        break;
    case OP_PERM:
        // a VSWAP is a pure permutation: a tile pass over the swapped qubits
        // writes each tile back permuted, reads and writes stay coalesced
        return apply_perm_gate(s, n, sizeof(C) == sizeof(double2) ? QK_C128 : QK_C64, op, st);
    default:
        return fail(QK_ERR_ARG, "unknown op kind %d", op.kind);
    }
    QK_CUDA(cudaGetLastError());
    return QK_OK;
}

// One lowered op on a raw state (used by the adjoint sweep).
int launch_gate_op(void *state, int n, int dtype, const Op &op, cudaStream_t st) {
    return dtype == QK_C128 ? launch_op<double2>((double2 *)state, n, op, st) : launch_op<float2>((float2 *)state, n, op, st);
}

template <typename C>
static int apply_gates_t(C *s, int n, const qk_gate *gates, size_t ng, cudaStream_t st) {
    for (size_t i = 0; i < ng; ++i) {
        Op op;
        int rc = lower_gate(gates[i], op);
        if (rc) return rc;
        for (int k = 0; k < op.nq; ++k)
            if (op.q[k] < 0 || op.q[k] >= n)
                return fail(QK_ERR_QUBIT, "gate %zu: qubit %d outside a %d-qubit state", i, op.q[k], n);
        rc = launch_op<C>(s, n, op, st);
        if (rc) return rc;
    }
    return QK_OK;
}

}  // namespace qk

// ---- C ABI --------------------------------------------------------------------

extern "C" {

int qk_sv_create(int nqubits, int dtype, qk_sv **out) {
    if (!out) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 36) return fail(QK_ERR_ARG, "nqubits must be in [1, 36], got %d", nqubits);
    if (dtype != QK_C128 && dtype != QK_C64) return fail(QK_ERR_ARG, "unknown dtype %d", dtype);
    auto *sv = new qk_sv();
    sv->n = nqubits;
    sv->dtype = dtype;
    sv->bytes = (dtype == QK_C128 ? sizeof(double2) : sizeof(float2)) << nqubits;
    cudaGetDevice(&sv->device);
    cudaError_t e = cudaMalloc(&sv->d, sv->bytes);
    if (e != cudaSuccess) {
        delete sv;
        return cuda_fail(e, "cudaMalloc(state)");
    }
    *out = sv;
    int rc = qk_sv_reset(sv);
    if (rc) {
        qk_sv_destroy(sv);
        *out = nullptr;
        return rc;
    }
    clear_error();
    return QK_OK;
}

void qk_sv_destroy(qk_sv *sv) {
    if (!sv) return;
    if (sv->d) cudaFree(sv->d);
    release_scratch_plan(sv->scratch);
    sv->ws.release();
    delete sv;
}

int qk_sv_release_workspace(qk_sv *sv) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    sv->ws.release();
    clear_error();
    return QK_OK;
}

int qk_sv_last_sweep(const qk_sv *sv, double *device_ms, double *alg_bytes, int *forward_passes,
                     int *backward_passes) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    if (!sv->ws.ev0) return fail(QK_ERR_ARG, "no adjoint sweep has run on this state");
    if (device_ms) *device_ms = sv->ws.last_ms;
    if (alg_bytes) *alg_bytes = sv->ws.last_bytes;
    if (forward_passes) *forward_passes = sv->ws.last_fwd;
    if (backward_passes) *backward_passes = sv->ws.last_bwd;
    clear_error();
    return QK_OK;
}

int qk_sv_reset(qk_sv *sv) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    const uint64_t namp = 1ull << sv->n;
    const unsigned grid = (unsigned)std::min<uint64_t>((namp + 255) / 256, (uint64_t)num_sms() * 16);
    if (sv->dtype == QK_C128) k_zero_state<double2><<<grid, 256, 0, sv->stream>>>((double2 *)sv->d, namp);
    else k_zero_state<float2><<<grid, 256, 0, sv->stream>>>((float2 *)sv->d, namp);
    QK_CUDA(cudaGetLastError());
    return QK_OK;
}

// Host complex128 <-> device state, converted in bounded chunks for c64.
int qk_sv_upload(qk_sv *sv, const double *host) {
    if (!sv || !host) return fail(QK_ERR_ARG, "null argument");
    if (sv->dtype == QK_C128) {
        QK_CUDA(cudaMemcpyAsync(sv->d, host, sv->bytes, cudaMemcpyHostToDevice, sv->stream));
        QK_CUDA(cudaStreamSynchronize(sv->stream));
        return QK_OK;
    }
    const uint64_t namp = 1ull << sv->n;
    const uint64_t chunk = std::min<uint64_t>(namp, 1ull << 24);
    double2 *tmp = nullptr;
    QK_CUDA(cudaMalloc(&tmp, chunk * sizeof(double2)));
    int rc = QK_OK;
    for (uint64_t off = 0; off < namp && !rc; off += chunk) {
        cudaError_t e = cudaMemcpyAsync(tmp, host + 2 * off, chunk * sizeof(double2), cudaMemcpyHostToDevice, sv->stream);
        if (e != cudaSuccess) { rc = cuda_fail(e, "upload"); break; }
        k_c128_to_c64<<<(unsigned)((chunk + 255) / 256), 256, 0, sv->stream>>>(tmp, (float2 *)sv->d + off, chunk);
    }
    cudaError_t e = cudaStreamSynchronize(sv->stream);
    cudaFree(tmp);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "upload");
    return rc;
}

int qk_sv_download(qk_sv *sv, double *host) {
    if (!sv || !host) return fail(QK_ERR_ARG, "null argument");
    if (sv->dtype == QK_C128) {
        QK_CUDA(cudaMemcpyAsync(host, sv->d, sv->bytes, cudaMemcpyDeviceToHost, sv->stream));
        QK_CUDA(cudaStreamSynchronize(sv->stream));
        return QK_OK;
    }
    const uint64_t namp = 1ull << sv->n;
    const uint64_t chunk = std::min<uint64_t>(namp, 1ull << 24);
    double2 *tmp = nullptr;
    QK_CUDA(cudaMalloc(&tmp, chunk * sizeof(double2)));
    int rc = QK_OK;
    for (uint64_t off = 0; off < namp && !rc; off += chunk) {
        k_c64_to_c128<<<(unsigned)((chunk + 255) / 256), 256, 0, sv->stream>>>((const float2 *)sv->d + off, tmp, chunk);
        cudaError_t e = cudaMemcpyAsync(host + 2 * off, tmp, chunk * sizeof(double2), cudaMemcpyDeviceToHost, sv->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sv->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "download");
    }
    cudaFree(tmp);
    return rc;
}

int qk_sv_save(qk_sv *sv, const char *path) {
    if (!sv || !path) return fail(QK_ERR_ARG, "null argument");
    const uint64_t namp = 1ull << sv->n;
    const uint64_t chunk = std::min<uint64_t>(namp, 1ull << 22);   // 64 MiB of complex128
    std::vector<double2> host(chunk);
    double2 *tmp = nullptr;
    if (sv->dtype == QK_C64) QK_CUDA(cudaMalloc(&tmp, chunk * sizeof(double2)));
    FILE *f = std::fopen(path, "wb");
    int rc = f ? QK_OK : fail(QK_ERR_IO, "cannot open %s for writing", path);
    for (uint64_t off = 0; off < namp && !rc; off += chunk) {
        const double2 *src = (const double2 *)sv->d + off;
        if (tmp) {
            k_c64_to_c128<<<(unsigned)((chunk + 255) / 256), 256, 0, sv->stream>>>((const float2 *)sv->d + off, tmp, chunk);
            src = tmp;
        }
        cudaError_t e = cudaMemcpyAsync(host.data(), src, chunk * sizeof(double2), cudaMemcpyDeviceToHost, sv->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sv->stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "save");
        else if (std::fwrite(host.data(), sizeof(double2), chunk, f) != chunk) rc = fail(QK_ERR_IO, "cannot write %s", path);
    }
    if (f && std::fclose(f) != 0 && !rc) rc = fail(QK_ERR_IO, "cannot write %s", path);
    if (tmp) cudaFree(tmp);
    if (!rc) clear_error();
    return rc;
}

int qk_sv_load(qk_sv *sv, const char *path) {
    if (!sv || !path) return fail(QK_ERR_ARG, "null argument");
    const uint64_t namp = 1ull << sv->n;
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(QK_ERR_IO, "cannot open state file %s", path);
    int rc = QK_OK;
    if (std::fseek(f, 0, SEEK_END) != 0 || (uint64_t)std::ftell(f) != namp * sizeof(double2))
        rc = fail(QK_ERR_ARG, "state file %s does not hold %llu complex128 amplitudes", path,
                  (unsigned long long)namp);
    std::rewind(f);
    const uint64_t chunk = std::min<uint64_t>(namp, 1ull << 22);
    std::vector<double2> host(chunk);
    double2 *tmp = nullptr;
    if (!rc && sv->dtype == QK_C64) {
        cudaError_t e = cudaMalloc(&tmp, chunk * sizeof(double2));
        if (e != cudaSuccess) rc = cuda_fail(e, "load");
    }
    for (uint64_t off = 0; off < namp && !rc; off += chunk) {
        if (std::fread(host.data(), sizeof(double2), chunk, f) != chunk) {
            rc = fail(QK_ERR_IO, "cannot read %s", path);
            break;
        }
        double2 *dst = tmp ? tmp : (double2 *)sv->d + off;
        cudaError_t e = cudaMemcpyAsync(dst, host.data(), chunk * sizeof(double2), cudaMemcpyHostToDevice, sv->stream);
        if (e == cudaSuccess && tmp)
            k_c128_to_c64<<<(unsigned)((chunk + 255) / 256), 256, 0, sv->stream>>>(tmp, (float2 *)sv->d + off, chunk);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sv->stream);   // host buffer reused next chunk
        if (e != cudaSuccess) rc = cuda_fail(e, "load");
    }
    std::fclose(f);
    if (tmp) cudaFree(tmp);
    if (!rc) clear_error();
    return rc;
}

int qk_sv_info(const qk_sv *sv, int *nqubits, int *dtype, void **device_ptr, size_t *bytes) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    if (nqubits) *nqubits = sv->n;
    if (dtype) *dtype = sv->dtype;
    if (device_ptr) *device_ptr = sv->d;
    if (bytes) *bytes = sv->bytes;
    return QK_OK;
}

int qk_sv_set_stream(qk_sv *sv, void *stream) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    sv->stream = (cudaStream_t)stream;
    return QK_OK;
}

int qk_sv_synchronize(qk_sv *sv) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    QK_CUDA(cudaStreamSynchronize(sv->stream));
    return QK_OK;
}

int qk_apply_gates_dev(void *state, int nqubits, int dtype, const qk_gate *gates, size_t n, void *stream) {
    if (!state || (!gates && n)) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 36) return fail(QK_ERR_ARG, "nqubits must be in [1, 36], got %d", nqubits);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == QK_C128) return apply_gates_t<double2>((double2 *)state, nqubits, gates, n, st);
    if (dtype == QK_C64) return apply_gates_t<float2>((float2 *)state, nqubits, gates, n, st);
    return fail(QK_ERR_ARG, "unknown dtype %d", dtype);
}

int qk_apply_gates(qk_sv *sv, const qk_gate *gates, size_t n) {
    if (!sv) return fail(QK_ERR_ARG, "null state");
    return qk_apply_gates_dev(sv->d, sv->n, sv->dtype, gates, n, sv->stream);
}

// ---- the per-gate path as a CUDA graph -------------------------------------

struct qk_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    qk_sv *sv = nullptr;
};

int qk_graph_create(qk_sv *sv, const qk_gate *gates, size_t n, qk_graph **out) {
    if (!sv || !out || (!gates && n)) return fail(QK_ERR_ARG, "null argument");
    std::vector<Op> ops(n);
    for (size_t i = 0; i < n; ++i) {
        int rc = lower_gate(gates[i], ops[i]);
        if (rc) return rc;
        for (int k = 0; k < ops[i].nq; ++k)
            if (ops[i].q[k] < 0 || ops[i].q[k] >= sv->n)
                return fail(QK_ERR_QUBIT, "gate %zu: qubit %d outside a %d-qubit state", i, ops[i].q[k], sv->n);
    }
    // capture the same launches qk_apply_gates makes, on a private stream
    // (thread-local mode: other threads' CUDA calls are unaffected)
    cudaStream_t cs = nullptr;
    QK_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return cuda_fail(e, "cudaStreamBeginCapture");
    }
    int rc = QK_OK;
    for (size_t i = 0; i < n && !rc; ++i) rc = launch_gate_op(sv->d, sv->n, sv->dtype, ops[i], cs);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc ? rc : cuda_fail(e, "cudaStreamEndCapture");
    }
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(e, "cudaGraphInstantiate");
    }
    auto *h = new qk_graph();
    h->graph = g;
    h->exec = ex;
    h->sv = sv;
    *out = h;
    clear_error();
    return QK_OK;
}

int qk_graph_launch(qk_graph *g) {
    if (!g) return fail(QK_ERR_ARG, "null graph");
    QK_CUDA(cudaGraphLaunch(g->exec, g->sv->stream));
    clear_error();
    return QK_OK;
}

void qk_graph_destroy(qk_graph *g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

int qk_apply_gates_timed(qk_sv *sv, const qk_gate *gates, size_t n, float *gate_ms) {
    if (!sv || !gate_ms || (!gates && n)) return fail(QK_ERR_ARG, "null argument");
    std::vector<cudaEvent_t> ev(n + 1);
    for (auto &e : ev) QK_CUDA(cudaEventCreate(&e));
    int rc = QK_OK;
    cudaError_t ce = cudaEventRecord(ev[0], sv->stream);
    for (size_t i = 0; i < n && !rc && ce == cudaSuccess; ++i) {
        rc = qk_apply_gates_dev(sv->d, sv->n, sv->dtype, gates + i, 1, sv->stream);
        if (!rc) ce = cudaEventRecord(ev[i + 1], sv->stream);
    }
    if (!rc && ce == cudaSuccess) ce = cudaEventSynchronize(ev[n]);
    for (size_t i = 0; i < n && !rc && ce == cudaSuccess; ++i) ce = cudaEventElapsedTime(&gate_ms[i], ev[i], ev[i + 1]);
    for (auto &e : ev) cudaEventDestroy(e);
    if (!rc && ce != cudaSuccess) rc = cuda_fail(ce, "per-gate timing");
    return rc;
}

int qk_apply_groups(qk_sv *sv, const qk_gate *gates, const int32_t *group_sizes, size_t ngroups) {
    if (!sv || (!group_sizes && ngroups)) return fail(QK_ERR_ARG, "null argument");
    return apply_group_plan(sv, gates, group_sizes, ngroups);
}

int qk_run(const qk_config *cfg, const qk_circuit *c, qk_sv *sv, double *seconds) {
    if (!cfg || !c || !sv) return fail(QK_ERR_ARG, "null argument");
    // fuse_width > 0 on a flat circuit: fused plan; a subcircuit file: its
    // group plan.  Both are built before the timed span, like the reference's
    // parsing.
    qk_plan *plan = nullptr;
    if (cfg->is_subcircuit) {
        qk_plan_opts o;
        std::memset(&o, 0, sizeof o);
        o.dtype = sv->dtype;
        o.fuse_width = (cfg->fuse_width == 5 || cfg->fuse_width == 6) && sv->dtype == QK_C64 ? cfg->fuse_width : 0;
        int rc = qk_plan_create_groups(c->gates.data(), c->group_sizes.data(), c->group_sizes.size(), sv->n, &o, &plan);
        if (rc) return rc;
    } else if (cfg->fuse_width > 0) {
        qk_plan_opts o;
        std::memset(&o, 0, sizeof o);
        o.dtype = sv->dtype;
        o.fuse_width = (cfg->fuse_width == 5 || cfg->fuse_width == 6) && sv->dtype == QK_C64 ? cfg->fuse_width : 0;
        int rc = qk_plan_create(c->gates.data(), c->gates.size(), sv->n, &o, &plan);
        if (rc) return rc;
    }
    if (plan) {
        int rc = qk::plan_prepare(sv, plan);
        if (rc) {
            qk_plan_destroy(plan);
            return rc;
        }
    }
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaError_t e0 = cudaEventCreate(&t0);
    if (e0 == cudaSuccess) e0 = cudaEventCreate(&t1);
    if (e0 == cudaSuccess) e0 = cudaEventRecord(t0, sv->stream);
    int rc = e0 != cudaSuccess ? cuda_fail(e0, "timing events")
             : plan            ? qk_plan_apply(sv, plan)
                               : qk_apply_gates(sv, c->gates.data(), c->gates.size());
    if (!rc) {
        cudaError_t e = cudaEventRecord(t1, sv->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (e != cudaSuccess) rc = cuda_fail(e, "timing");
        else if (seconds) *seconds = ms / 1e3;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (plan) qk_plan_destroy(plan);
    return rc;
}

}  // extern "C"
