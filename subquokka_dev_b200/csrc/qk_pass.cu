// Fused-pass kernel and the plan entry points of the C ABI.
//
// One CTA owns one tile of 2^T amplitudes at a time (grid-stride over tiles):
//   1. coalesced load HBM -> shared memory (runs of 2^L contiguous amplitudes),
//   2. the pass program: TOP_REMAP moves the tile shared -> registers with a
//      new choice of register qubits, TOP_G1/TOP_G2 apply dense gates to
//      register-resident amplitude pairs/quads, TOP_DIAG multiplies phases
//      (any qubit, tile-local or not),
//   3. registers -> shared memory -> coalesced store to HBM.
// A pass is one HBM read and one write of the state however many gates it
// carries.  Permutation passes (VSWAP) write element j of the tile to the
// position of perm(j).
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "qk_device.h"
#include "qk_internal.h"
#include "qk_kernels.cuh"
#include "qk_devplan.h"
#include "qk_pass_device.cuh"

namespace qk {

// nbuf = 2: the next tile is prefetched (cp.async) into the other buffer
// while the current one is processed; nbuf = 1: load, process, store.
// NS = 2 runs an adjoint pass over psi (s) and lambda (s2) together; the
// gradient accumulators of the pass live in shared memory and are added to
// ggrad[gparams[grad0 + i]] once per CTA.
template <typename C, int R, int NS, bool NARROW, bool XOPS>
__global__ void __launch_bounds__(NARROW ? 128 : pass_max_threads<C, R, NS>(), NARROW ? 3 : 1) k_pass(C *__restrict__ s, C *__restrict__ s2, uint64_t ntiles,
                                                       const __grid_constant__ PassDesc d, const TOp *__restrict__ gprog,
                                                       const C *__restrict__ gcoef, const int32_t *__restrict__ gparams,
                                                       double *__restrict__ ggrad, int nbuf) {
    constexpr int LOG2R = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : R == 16 ? 4 : 5;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t N = 1u << d.T;
    C *buf0 = reinterpret_cast<C *>(smem_raw);                 // psi, buffer 0
    C *buf1 = buf0 + (nbuf > 1 ? N : 0);                       // psi, buffer 1
    C *wuf0 = buf0 + (size_t)N * nbuf;                         // lambda buffers (NS = 2)
    C *wuf1 = wuf0 + (nbuf > 1 ? N : 0);
    const uint32_t NT = blockDim.x;
    // program, coefficients and gradient accumulators after the tiles
    TOp *prog = reinterpret_cast<TOp *>(buf0 + (size_t)N * nbuf * NS);
    C *coef = reinterpret_cast<C *>(prog + d.nprog);
    double *gsm = reinterpret_cast<double *>(coef + d.ncoef);
    for (int i = threadIdx.x; i < d.nprog; i += NT) prog[i] = gprog[d.prog0 + i];
    for (int i = threadIdx.x; i < d.ncoef; i += NT) coef[i] = gcoef[d.coef0 + i];
    if constexpr (NS == 2)
        for (int i = threadIdx.x; i < d.ngrad; i += NT) gsm[i] = 0.0;
    if (d.perm) {
        // permutation pass: plain load / permuted store, one buffer
        run_perm_pass(s, buf0, ntiles, d, N, NT);
        return;
    }
    TileAddr<C, LOG2R> ta;
    ta.init(d, NT);
    uint64_t o = blockIdx.x;
    if (o < ntiles) {
        const uint64_t b0 = pass_base(o, d);
        if constexpr (NS == 2) {
#pragma unroll
            for (int u = 0; u < R; ++u) cp_async_amp(wuf0 + ta.sidx(u), s2 + (b0 | ta.g(u)));
        }
        prefetch_tile<C, R, LOG2R>(buf0, s, b0, ta);
    }
    for (int it = 0; o < ntiles; o += gridDim.x, ++it) {
        C *tl = (it & 1) ? buf1 : buf0;
        C *nx = (it & 1) ? buf0 : buf1;
        C *tw = (it & 1) ? wuf1 : wuf0;
        C *nw = (it & 1) ? wuf0 : wuf1;
        const uint64_t base = pass_base(o, d);
        cp_async_wait_all();
        __syncthreads();
        const uint64_t on = o + gridDim.x;
        if (nbuf > 1 && on < ntiles) {
            const uint64_t bn = pass_base(on, d);
            if constexpr (NS == 2) {
#pragma unroll
                for (int u = 0; u < R; ++u) cp_async_amp(nw + ta.sidx(u), s2 + (bn | ta.g(u)));
            }
            prefetch_tile<C, R, LOG2R>(nx, s, bn, ta);
        }
        run_program<C, R, NS, XOPS>(tl, tw, base, d, prog, coef, gsm, N);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < R; ++u) {
            s[base | ta.g(u)] = tl[ta.sidx(u)];
            if constexpr (NS == 2) s2[base | ta.g(u)] = tw[ta.sidx(u)];
        }
        if (nbuf == 1) {
            __syncthreads();
            if (on < ntiles) {
                const uint64_t bn = pass_base(on, d);
                if constexpr (NS == 2) {
#pragma unroll
                    for (int u = 0; u < R; ++u) cp_async_amp(tw + ta.sidx(u), s2 + (bn | ta.g(u)));
                }
                prefetch_tile<C, R, LOG2R>(tl, s, bn, ta);
            }
        }
    }
    cp_async_wait_all();
    if constexpr (NS == 2) {
        __syncthreads();
        for (int i = threadIdx.x; i < d.ngrad; i += NT) atomicAdd(ggrad + gparams[d.grad0 + i], gsm[i]);
    }
}

// In-place permutation sweep for a VSWAP whose qubits do not fit in a tile.
template <typename C>
__global__ void k_perm_flat(C *__restrict__ s, uint64_t namp, PassDesc d) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < namp; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t f = e;
        for (int i = 0; i < d.nperm; ++i) {
            const uint64_t a = (e >> d.perm_a[i]) & 1, b = (e >> d.perm_b[i]) & 1;
            f = (f & ~(1ull << d.perm_a[i]) & ~(1ull << d.perm_b[i])) | (b << d.perm_a[i]) | (a << d.perm_b[i]);
        }
        if (e < f) {
            const C a = s[e];
            s[e] = s[f];
            s[f] = a;
        }
    }
}

static int cuda_err(cudaError_t e, const char *what) {
    // An allocation failure is not sticky, but it stays as the thread's last
    // error; clear it so the next launch check does not report it again.
    if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? QK_ERR_OOM : QK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Device pointers of one pass launch.
template <typename C> struct PassArgs {
    C *s;                    // psi
    C *s2;                   // lambda (two-state passes), else null
    const TOp *ops;
    const C *coef;
    const int32_t *gparams;  // gradient slot -> parameter (two-state passes)
    double *ggrad;           // gradient accumulators (two-state passes)
};

template <typename C, int R, int NS, bool NARROW, bool XOPS>
static int launch_pass_k(const PassArgs<C> &a, int n, const PassDesc &d, uint32_t threads, cudaStream_t st) {
    static std::atomic<uint64_t> smem_done{0};
    const size_t tile = (sizeof(C) << d.T) * NS;
    const int nbuf = d.perm ? 1 : (2 * tile <= (200u << 10) ? 2 : 1);
    const size_t smem = tile * nbuf + d.nprog * sizeof(TOp) + d.ncoef * sizeof(C) + (NS == 2 ? d.ngrad * sizeof(double) : 0);
    if (smem > (220u << 10)) return fail(QK_ERR_ARG, "pass needs %zu bytes of shared memory", smem);
    cudaError_t e;
    e = smem_limit_once(smem_done, (const void *)k_pass<C, R, NS, NARROW, XOPS>, 220 << 10);
    if (e != cudaSuccess) return cuda_err(e, "cudaFuncSetAttribute(k_pass)");
    const int sms = device_sms();
    int mb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mb, k_pass<C, R, NS, NARROW, XOPS>, (int)threads, smem);
    if (e != cudaSuccess || mb < 1) mb = 1;
    const uint64_t ntiles = 1ull << (n - d.T);
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sms * mb);
    k_pass<C, R, NS, NARROW, XOPS><<<grid, threads, smem, st>>>(a.s, a.s2, ntiles, d, a.ops, a.coef, a.gparams, a.ggrad, nbuf);
    e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_err(e, "k_pass launch");
}

template <typename C, int R, int NS>
static int launch_pass_r(const PassArgs<C> &a, int n, const PassDesc &d, cudaStream_t st) {
    const uint32_t threads = d.perm ? std::max<uint32_t>(1, std::min<uint32_t>(kPassThreads, 1u << d.T))
                                    : (uint32_t)((1u << d.T) / R);
    if (threads > kPassThreads || threads == 0) return fail(QK_ERR_ARG, "pass of %d tile bits needs %u threads", d.T, threads);
    // programs with real or diagonal ops run on the instance that
    // specialises them; the others on one without that code, whose register
    // allocation it would otherwise change (the 30-qubit random circuit and
    // HEA forward passes, which have neither, 1-2.5 % slower with it)
    if constexpr (pass_narrow_ok<C, R, NS>())
        if (!d.perm && threads <= 128)
            return d.xops ? launch_pass_k<C, R, NS, true, true>(a, n, d, threads, st)
                          : launch_pass_k<C, R, NS, true, false>(a, n, d, threads, st);
    return d.xops ? launch_pass_k<C, R, NS, false, true>(a, n, d, threads, st)
                  : launch_pass_k<C, R, NS, false, false>(a, n, d, threads, st);
}

template <typename C>
static int launch_pass(C *s, int n, int r, const PassDesc &d, const TOp *ops, const C *coef, cudaStream_t st,
                       C *s2 = nullptr, const int32_t *gparams = nullptr, double *ggrad = nullptr) {
    if (d.perm) {
        // a permutation pass acts on each state on its own
        for (C *x : {s, s2}) {
            if (!x) continue;
            int rc;
            if (d.perm == 2) {
                const uint64_t namp = 1ull << n;
                const unsigned grid = (unsigned)std::min<uint64_t>((namp + 255) / 256, 148ull * 16);
                k_perm_flat<C><<<grid, 256, 0, st>>>(x, namp, d);
                cudaError_t e = cudaGetLastError();
                rc = e == cudaSuccess ? QK_OK : cuda_err(e, "k_perm_flat launch");
            } else {
                PassArgs<C> a{x, nullptr, ops, coef, nullptr, nullptr};
                rc = launch_pass_r<C, 2, 1>(a, n, d, st);
            }
            if (rc) return rc;
        }
        return QK_OK;
    }
    // a compute pass reads its program and coefficients from device memory
    if ((d.nprog && !ops) || (d.ncoef && !coef))
        return fail(QK_ERR_ARG, "compute pass without its program in device memory");
    PassArgs<C> a{s, s2, ops, coef, gparams, ggrad};
    // register-resident amplitudes per thread: up to 8 complex128 or 16
    // complex64 per state (more would spill)
    if (s2) {
        switch (r) {
        case 1: return launch_pass_r<C, 2, 2>(a, n, d, st);
        case 2: return launch_pass_r<C, 4, 2>(a, n, d, st);
        case 3:
            return launch_pass_r<C, 8, 2>(a, n, d, st);
        case 4:
            if constexpr (sizeof(C) == sizeof(float2)) return launch_pass_r<C, 16, 2>(a, n, d, st);
            break;
        }
        return fail(QK_ERR_ARG, "reg_bits %d unsupported for two-state passes", r);
    }
    switch (r) {
    case 1: return launch_pass_r<C, 2, 1>(a, n, d, st);
    case 2: return launch_pass_r<C, 4, 1>(a, n, d, st);
    case 3: return launch_pass_r<C, 8, 1>(a, n, d, st);
    case 4: return launch_pass_r<C, 16, 1>(a, n, d, st);
    }
    return fail(QK_ERR_ARG, "reg_bits %d unsupported", r);
}

static int upload_plan(const HostPlan &hp, int dtype, DevPlan &dp, cudaStream_t st) {
    const size_t ob = std::max<size_t>(1, hp.ops.size()) * sizeof(TOp);
    const size_t nc = hp.coef.size() / 2;
    const size_t cb = std::max<size_t>(1, nc) * (dtype == QK_C128 ? sizeof(double2) : sizeof(float2));
    cudaError_t e;
    if (ob > dp.ops_cap) {
        if (dp.ops) cudaFree(dp.ops);
        dp.ops = nullptr;
        e = cudaMalloc(&dp.ops, ob);
        if (e != cudaSuccess) { dp.ops_cap = 0; return cuda_err(e, "cudaMalloc(plan ops)"); }
        dp.ops_cap = ob;
    }
    if (cb > dp.coef_cap) {
        if (dp.coef) cudaFree(dp.coef);
        dp.coef = nullptr;
        e = cudaMalloc(&dp.coef, cb);
        if (e != cudaSuccess) { dp.coef_cap = 0; return cuda_err(e, "cudaMalloc(plan coefficients)"); }
        dp.coef_cap = cb;
    }
    const size_t gb = std::max<size_t>(1, hp.grad_params.size()) * sizeof(int32_t);
    if (gb > dp.gparams_cap) {
        if (dp.gparams) cudaFree(dp.gparams);
        dp.gparams = nullptr;
        e = cudaMalloc(&dp.gparams, gb);
        if (e != cudaSuccess) { dp.gparams_cap = 0; return cuda_err(e, "cudaMalloc(plan gradient slots)"); }
        dp.gparams_cap = gb;
    }
    if (!hp.ops.empty()) {
        e = cudaMemcpyAsync(dp.ops, hp.ops.data(), hp.ops.size() * sizeof(TOp), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_err(e, "upload plan ops");
    }
    if (!hp.grad_params.empty()) {
        e = cudaMemcpyAsync(dp.gparams, hp.grad_params.data(), hp.grad_params.size() * sizeof(int32_t),
                            cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return cuda_err(e, "upload plan gradient slots");
    }
    std::vector<float> f;   // complex64 coefficients; must outlive the copy
    if (nc) {
        if (dtype == QK_C128) {
            e = cudaMemcpyAsync(dp.coef, hp.coef.data(), nc * sizeof(double2), cudaMemcpyHostToDevice, st);
        } else {
            f.assign(hp.coef.begin(), hp.coef.end());
            e = cudaMemcpyAsync(dp.coef, f.data(), nc * sizeof(float2), cudaMemcpyHostToDevice, st);
        }
        if (e != cudaSuccess) return cuda_err(e, "upload plan coefficients");
    }
    // One rule for every upload from host memory in this library: a copy whose
    // source the caller may free (f here; hp itself when the plan is a
    // temporary, as for subcircuit files) has finished before the call returns.
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "upload plan");
    return QK_OK;
}

static int run_plan(void *state, int dtype, const HostPlan &hp, const DevPlan &dp, cudaStream_t st) {
    for (const PassDesc &d : hp.passes) {
        int rc = dtype == QK_C128
                     ? launch_pass<double2>((double2 *)state, hp.n, hp.r, d, dp.ops, (const double2 *)dp.coef, st)
                     : launch_pass<float2>((float2 *)state, hp.n, hp.r, d, dp.ops, (const float2 *)dp.coef, st);
        if (rc) return rc;
    }
    return QK_OK;
}

// Run a two-state (adjoint) plan over psi and lambda, adding gradients into ggrad.
int run_adjoint_plan(void *psi, void *lam, int dtype, const HostPlan &hp, const DevPlan &dp, double *ggrad,
                     cudaStream_t st) {
    for (const PassDesc &d : hp.passes) {
        int rc = dtype == QK_C128
                     ? launch_pass<double2>((double2 *)psi, hp.n, hp.r, d, dp.ops, (const double2 *)dp.coef, st,
                                            (double2 *)lam, dp.gparams, ggrad)
                     : launch_pass<float2>((float2 *)psi, hp.n, hp.r, d, dp.ops, (const float2 *)dp.coef, st,
                                           (float2 *)lam, dp.gparams, ggrad);
        if (rc) return rc;
    }
    return QK_OK;
}

int upload_host_plan(const HostPlan &hp, DevPlan &dp, cudaStream_t st) { return upload_plan(hp, hp.dtype, dp, st); }
int run_forward_plan(void *state, const HostPlan &hp, const DevPlan &dp, cudaStream_t st) {
    return run_plan(state, hp.dtype, hp, dp, st);
}

// Run a host plan whose programs and coefficients are already in device
// memory at ops / coef (coefficients in the state's type).
int run_plan_at(void *state, int dtype, const HostPlan &hp, const TOp *ops, const void *coef, cudaStream_t st) {
    for (const PassDesc &d : hp.passes) {
        int rc = dtype == QK_C128
                     ? launch_pass<double2>((double2 *)state, hp.n, hp.r, d, ops, (const double2 *)coef, st)
                     : launch_pass<float2>((float2 *)state, hp.n, hp.r, d, ops, (const float2 *)coef, st);
        if (rc) return rc;
    }
    return QK_OK;
}

}  // namespace qk

using namespace qk;

namespace qk {
// the blocks of a dense plan in order (qk_dense_tc.cu)
int run_dense_blocks(void *state, int n, int dtype, const std::vector<DenseBlock> &blocks, const void *dA, int *derr,
                     cudaStream_t st);
}  // namespace qk

struct qk_plan {
    HostPlan hp;
    DevPlan dp;
    bool uploaded = false;
    // fuse_width = 5 or 6: dense blocks on the tensor cores instead of passes
    bool dense = false;
    std::vector<DenseBlock> blocks;
    void *dA = nullptr;
    int *derr = nullptr;
};

// Per-state scratch for the subcircuit path (one uploaded group plan).
namespace qk {
DevPlan &state_scratch_plan(qk_sv *sv);
cudaStream_t state_stream(const qk_sv *sv);
void *state_ptr(const qk_sv *sv);
int state_qubits(const qk_sv *sv);
int state_dtype(const qk_sv *sv);

int apply_group_plan(qk_sv *sv, const qk_gate *gates, const int32_t *sizes, size_t ngroups) {
    HostPlan hp;
    PlanOptions o = default_plan_options(state_dtype(sv), state_qubits(sv));
    int rc = build_group_plan(gates, sizes, ngroups, state_qubits(sv), o, hp);
    if (rc) return rc;
    DevPlan &dp = state_scratch_plan(sv);
    rc = upload_plan(hp, state_dtype(sv), dp, state_stream(sv));
    if (rc) return rc;
    return run_plan(state_ptr(sv), state_dtype(sv), hp, dp, state_stream(sv));
}

int apply_perm_gate(void *state, int n, int dtype, const Op &op, cudaStream_t st) {
    HostPlan hp;
    int rc = build_perm_plan(op, n, default_plan_options(dtype, n), hp);
    if (rc) return rc;
    DevPlan none;   // permutation passes run no program
    return run_plan(state, dtype, hp, none, st);
}

void release_scratch_plan(DevPlan &dp) { dp.release(); }
}  // namespace qk

extern "C" {

int qk_plan_create(const qk_gate *gates, size_t n, int nqubits, const qk_plan_opts *opts, qk_plan **out) {
    if (!out || (!gates && n)) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 36) return fail(QK_ERR_ARG, "nqubits must be in [1, 36], got %d", nqubits);
    const int dtype = opts ? opts->dtype : QK_C128;
    if (opts && opts->fuse_width) {
        if (opts->fuse_width != 5 && opts->fuse_width != kDenseQubits)
            return fail(QK_ERR_ARG, "fuse_width must be 0, 5 or %d", kDenseQubits);
        if (dtype != QK_C64 && dtype != QK_C128) return fail(QK_ERR_ARG, "unknown dtype %d", dtype);
        if (nqubits < 12) return fail(QK_ERR_UNSUPPORTED, "tensor-core dense blocks need at least 12 qubits");
        auto *p = new qk_plan();
        p->dense = true;
        p->hp.n = nqubits;
        p->hp.dtype = dtype;
        int rc = build_dense_blocks(gates, n, nqubits, opts->fuse_width, dtype, p->blocks);
        if (rc) {
            delete p;
            return rc;
        }
        p->hp.ngates = n;
        *out = p;
        return QK_OK;
    }
    PlanOptions o = default_plan_options(dtype, nqubits);
    if (opts && opts->tile_bits) o.tile_bits = opts->tile_bits;
    if (opts && opts->reg_bits) o.reg_bits = opts->reg_bits;
    auto *p = new qk_plan();
    int rc = build_plan(gates, n, nqubits, o, p->hp);
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return QK_OK;
}

int qk_plan_create_groups(const qk_gate *gates, const int32_t *group_sizes, size_t ngroups, int nqubits,
                          const qk_plan_opts *opts, qk_plan **out) {
    if (!out || (!group_sizes && ngroups)) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 36) return fail(QK_ERR_ARG, "nqubits must be in [1, 36], got %d", nqubits);
    if (opts && opts->fuse_width) {
        // tensor-core blocks: the groups' gates as one list (their VSWAPs
        // become renamings inside build_dense_blocks)
        size_t ng = 0;
        for (size_t g = 0; g < ngroups; ++g) {
            if (group_sizes[g] < 0) return fail(QK_ERR_ARG, "group %zu has negative size", g);
            ng += (size_t)group_sizes[g];
        }
        return qk_plan_create(gates, ng, nqubits, opts, out);
    }
    const int dtype = opts ? opts->dtype : QK_C128;
    PlanOptions o = default_plan_options(dtype, nqubits);
    if (opts && opts->tile_bits) o.tile_bits = opts->tile_bits;
    if (opts && opts->reg_bits) o.reg_bits = opts->reg_bits;
    auto *p = new qk_plan();
    int rc = build_group_plan(gates, group_sizes, ngroups, nqubits, o, p->hp);
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return QK_OK;
}

int qk_plan_stats(const qk_plan *p, size_t *passes, size_t *program_ops, size_t *remaps) {
    if (!p) return fail(QK_ERR_ARG, "null plan");
    if (p->dense) {
        if (passes) *passes = p->blocks.size();
        if (program_ops) *program_ops = p->hp.ngates;
        if (remaps) *remaps = 0;
        return QK_OK;
    }
    if (passes) *passes = p->hp.passes.size();
    if (program_ops) *program_ops = p->hp.ops.size();
    if (remaps) *remaps = p->hp.nremaps;
    return QK_OK;
}

}  // extern "C"

namespace qk {
// Device copies of a plan's programs (or tensor-core operands), made once;
// qk_plan_apply calls it, qk_run calls it before its timed span.
int plan_prepare(qk_sv *sv, qk_plan *p) {
    if (p->uploaded) return QK_OK;
    if (p->dense) {
        // one operand per block (zeros for permutation blocks), dense_operand_bytes apart
        const size_t step = dense_operand_bytes(p->hp.dtype);
        std::vector<unsigned char> all(p->blocks.size() * step, 0);
        std::vector<uint16_t> one16;
        std::vector<uint32_t> one32;
        for (size_t k = 0; k < p->blocks.size(); ++k) {
            const DenseBlock &b = p->blocks[k];
            if (b.perm) continue;
            if (p->hp.dtype == QK_C128) {
                dense_i8_operand(b, one32);
                std::memcpy(all.data() + k * step, one32.data(), step);
            } else {
                dense_block_operand(b, one16);
                std::memcpy(all.data() + k * step, one16.data(), step);
            }
        }
        cudaError_t e = cudaMalloc(&p->dA, std::max<size_t>(1, all.size()));
        if (e == cudaSuccess) e = cudaMalloc(&p->derr, sizeof(int));
        if (e == cudaSuccess && !all.empty()) e = cudaMemcpy(p->dA, all.data(), all.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_err(e, "upload dense blocks");
    } else {
        int rc = upload_plan(p->hp, p->hp.dtype, p->dp, state_stream(sv));
        if (rc) return rc;
        cudaError_t e = cudaStreamSynchronize(state_stream(sv));
        if (e != cudaSuccess) return cuda_err(e, "plan upload");
    }
    p->uploaded = true;
    return QK_OK;
}
}  // namespace qk

extern "C" {

int qk_plan_apply(qk_sv *sv, qk_plan *p) {
    if (!sv || !p) return fail(QK_ERR_ARG, "null argument");
    if (state_qubits(sv) != p->hp.n || state_dtype(sv) != p->hp.dtype)
        return fail(QK_ERR_ARG, "plan built for %d qubits dtype %d, state has %d qubits dtype %d", p->hp.n,
                    p->hp.dtype, state_qubits(sv), state_dtype(sv));
    int rc = plan_prepare(sv, p);
    if (rc) return rc;
    if (p->dense) {
        cudaStream_t st = state_stream(sv);
        cudaError_t e = cudaMemsetAsync(p->derr, 0, sizeof(int), st);
        if (e != cudaSuccess) return cuda_err(e, "reset error flag");
        rc = run_dense_blocks(state_ptr(sv), p->hp.n, p->hp.dtype, p->blocks, p->dA, p->derr, st);
        if (rc) return rc;
        int herr = 0;
        e = cudaMemcpyAsync(&herr, p->derr, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_err(e, "dense blocks");
        if (herr == 2) return fail(QK_ERR_CUDA, "tensor-core pass: shared memory not 1024-byte aligned");
        if (herr == 3)
            return fail(QK_ERR_CUDA, "a tensor-core pass gave up waiting for its last MMAs before releasing TMEM");
        if (herr) return fail(QK_ERR_CUDA, "a tensor-core pass gave up waiting for its contraction");
        return QK_OK;
    }
    return run_plan(state_ptr(sv), p->hp.dtype, p->hp, p->dp, state_stream(sv));
}

int qk_plan_dense_block(const qk_plan *p, size_t k, int32_t *qubits, double *u, int *is_perm) {
    if (!p || !qubits || !u || !is_perm) return fail(QK_ERR_ARG, "null argument");
    if (!p->dense) return fail(QK_ERR_ARG, "not a dense plan");
    if (k >= p->blocks.size()) return fail(QK_ERR_ARG, "block %zu of %zu", k, p->blocks.size());
    const DenseBlock &b = p->blocks[k];
    *is_perm = b.perm;
    if (b.perm) {
        for (int i = 0; i < kDenseQubits; ++i) qubits[i] = -1;
        for (int i = 0; i < b.perm_op.nq && i < kDenseQubits; ++i) qubits[i] = b.perm_op.q[i];
        return QK_OK;
    }
    for (int i = 0; i < kDenseQubits; ++i) qubits[i] = b.q[i];
    std::memcpy(u, b.u.data(), b.u.size() * sizeof(double));
    return QK_OK;
}

void qk_plan_destroy(qk_plan *p) {
    if (!p) return;
    if (p->dA) cudaFree(p->dA);
    if (p->derr) cudaFree(p->derr);
    p->dp.release();
    delete p;
}

}  // extern "C"
