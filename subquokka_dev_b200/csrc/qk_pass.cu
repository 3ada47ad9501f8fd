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

#include "qk_internal.h"
#include "qk_kernels.cuh"
#include "qk_devplan.h"

namespace qk {

constexpr int kPassThreads = 512;

__device__ __forceinline__ uint64_t pass_base(uint64_t o, const PassDesc &d) {
    uint64_t x = o << d.L;
#pragma unroll 1
    for (int k = d.L; k < d.T; ++k) x = ins0(x, d.bpos[k]);
    return x;
}

__device__ __forceinline__ uint64_t pass_off(uint32_t j, const PassDesc &d) {
    uint64_t g = j & ((1u << d.L) - 1);
#pragma unroll 1
    for (int k = d.L; k < d.T; ++k) g |= (uint64_t)((j >> k) & 1) << d.bpos[k];
    return g;
}

// Scatter the low bits of v into the set bits of mask, lowest first.
__device__ __forceinline__ uint32_t deposit_bits(uint32_t v, uint32_t mask) {
    uint32_t r = 0;
    while (mask) {
        const uint32_t low = mask & (0u - mask);
        if (v & 1) r |= low;
        v >>= 1;
        mask ^= low;
    }
    return r;
}

template <int LOG2R>
__device__ __forceinline__ uint32_t reg_offset(int kk, const uint32_t (&bm)[kPassMaxReg]) {
    uint32_t x = 0;
#pragma unroll
    for (int s = 0; s < LOG2R; ++s)
        if ((kk >> s) & 1) x |= bm[s];
    return x;
}

template <int S, typename C, int R>
__device__ __forceinline__ void reg_g1(C (&v)[R], const C m0, const C m1, const C m2, const C m3) {
    if constexpr ((1 << S) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & (1 << S)) continue;
            const C a = v[k], b = v[k | (1 << S)];
            v[k] = cmul2(m0, a, m1, b);
            v[k | (1 << S)] = cmul2(m2, a, m3, b);
        }
    }
}

template <int A, int B, typename C, int R>
__device__ __forceinline__ void reg_g2(C (&v)[R], const C *__restrict__ m) {
    if constexpr (A < B && (1 << B) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & ((1 << A) | (1 << B))) continue;
            const int k1 = k | (1 << A), k2 = k | (1 << B), k3 = k | (1 << A) | (1 << B);
            const C x0 = v[k], x1 = v[k1], x2 = v[k2], x3 = v[k3];
            C y[4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
                y[r] = cadd(cmul2(m[4 * r], x0, m[4 * r + 1], x1), cmul2(m[4 * r + 2], x2, m[4 * r + 3], x3));
            v[k] = y[0];
            v[k1] = y[1];
            v[k2] = y[2];
            v[k3] = y[3];
        }
    }
}


// Shared-memory layout of a tile: element j lives at swz(j), which XORs the
// low index bits with folds of the higher ones.  A warp's lanes differ in
// three (complex128) or four (complex64) consecutive thread bits wherever the
// register qubits sit, and the fold sends those bits to distinct banks, so
// the re-mappings stay (nearly) conflict-free.
template <typename C> __device__ __forceinline__ uint32_t swz(uint32_t j) {
    if constexpr (sizeof(C) == 16) {
        return j ^ (((j >> 3) ^ (j >> 6) ^ (j >> 9) ^ (j >> 12)) & 7u);
    } else {
        return j ^ (((j >> 4) ^ (j >> 8) ^ (j >> 12)) & 15u);
    }
}

// Asynchronous global -> shared copy of one amplitude (cp.async, sm_80+).
template <typename C> __device__ __forceinline__ void cp_async_amp(C *dst_smem, const C *src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_smem);
    if constexpr (sizeof(C) == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Per-thread address tables of a pass.  Thread tid handles tile elements
// j = tid + u * NT (u < R), i.e. u sits in the top r tile bits.  Both the HBM
// offset (a bit deposit) and the shared-memory index (swz) are linear over
// disjoint bit groups, so each is the thread's own part combined with the
// parts of the set bits of u (compile-time after unrolling).
template <typename C, int LOG2R> struct TileAddr {
    uint64_t g_t;                 // HBM offset of tid's bits
    uint64_t g_u[LOG2R];          // HBM offset of bit b of u
    uint32_t s_t;                 // swz of tid
    uint32_t s_u[LOG2R];          // swz of bit b of u
    __device__ __forceinline__ void init(const PassDesc &d, uint32_t NT) {
        g_t = pass_off(threadIdx.x, d);
        s_t = swz<C>(threadIdx.x);
#pragma unroll
        for (int b = 0; b < LOG2R; ++b) {
            g_u[b] = pass_off(NT << b, d);
            s_u[b] = swz<C>(NT << b);
        }
    }
    __device__ __forceinline__ uint64_t g(int u) const {
        uint64_t x = g_t;
#pragma unroll
        for (int b = 0; b < LOG2R; ++b)
            if ((u >> b) & 1) x |= g_u[b];
        return x;
    }
    __device__ __forceinline__ uint32_t sidx(int u) const {
        uint32_t x = s_t;
#pragma unroll
        for (int b = 0; b < LOG2R; ++b)
            if ((u >> b) & 1) x ^= s_u[b];
        return x;
    }
};

template <typename C, int R, int LOG2R>
__device__ __forceinline__ void prefetch_tile(C *buf, const C *__restrict__ s, uint64_t base,
                                              const TileAddr<C, LOG2R> &ta) {
#pragma unroll
    for (int u = 0; u < R; ++u) cp_async_amp(buf + ta.sidx(u), s + (base | ta.g(u)));
    cp_async_commit();
}

// Permutation pass: tile element j goes to the position of perm(j).
template <typename C>
__device__ void run_perm_tile(C *__restrict__ s, C *tl, uint64_t base, const PassDesc &d, uint32_t N, uint32_t NT) {
    for (uint32_t j = threadIdx.x; j < N; j += NT) {
        uint32_t f = j;
        for (int i = 0; i < d.nperm; ++i) {
            const uint32_t a = (j >> d.perm_a[i]) & 1, b = (j >> d.perm_b[i]) & 1;
            f = (f & ~(1u << d.perm_a[i]) & ~(1u << d.perm_b[i])) | (b << d.perm_a[i]) | (a << d.perm_b[i]);
        }
        s[base | pass_off(f, d)] = tl[swz<C>(j)];
    }
}

// Bit pattern over the register index kk (R bits) of "register slot s is 1".
__device__ __forceinline__ uint32_t slot_pattern(int s) {
    return s == 0 ? 0xAAAAAAAAu : s == 1 ? 0xCCCCCCCCu : s == 2 ? 0xF0F0F0F0u : s == 3 ? 0xFF00FF00u : 0xFFFF0000u;
}

// For a diagonal-op qubit code: the set of register indices kk at which that
// qubit's bit is 1, given the current mapping (reg slots -> tile bits, thread
// bits tb, tile base).
template <int LOG2R>
__device__ __forceinline__ uint32_t bit_set(uint8_t code, uint32_t none, uint64_t base, uint32_t tb,
                                            const uint32_t (&bm)[kPassMaxReg]) {
    if (code == kNoQubit) return none ? 0xFFFFFFFFu : 0u;
    if (code & kOuterFlag) return ((base >> (code & 0x7F)) & 1) ? 0xFFFFFFFFu : 0u;
    const uint32_t m = 1u << code;
#pragma unroll
    for (int s = 0; s < LOG2R; ++s)
        if (bm[s] == m) return slot_pattern(s);
    return (tb & m) ? 0xFFFFFFFFu : 0u;
}

// swz index of register element kk under the current mapping
template <int LOG2R>
__device__ __forceinline__ uint32_t reg_sidx(int kk, uint32_t stb, const uint32_t (&sb)[LOG2R]) {
    uint32_t x = stb;
#pragma unroll
    for (int q = 0; q < LOG2R; ++q)
        if ((kk >> q) & 1) x ^= sb[q];
    return x;
}

template <typename C> __device__ __forceinline__ double imdot(C l, C a) { return (double)l.x * a.y - (double)l.y * a.x; }
template <typename C> __device__ __forceinline__ double redot(C l, C a) { return (double)l.x * a.x + (double)l.y * a.y; }

// Im <lambda|G|psi> over this thread's register pairs of slot S (G = X, Y, Z by gen 1, 2, 3).
template <int S, typename C, int R>
__device__ __forceinline__ double reg_grad(const C (&v)[R], const C (&w)[R], int gen) {
    double s = 0;
    if constexpr ((1 << S) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & (1 << S)) continue;
            const C a0 = v[k], a1 = v[k | (1 << S)], l0 = w[k], l1 = w[k | (1 << S)];
            if (gen == 1) s += imdot(l0, a1) + imdot(l1, a0);
            else if (gen == 2) s += redot(l1, a0) - redot(l0, a1);
            else s += imdot(l0, a0) - imdot(l1, a1);
        }
    }
    return s;
}

// Run a pass program on one tile (NS = 1) or on the matching tiles of two
// states (NS = 2: psi in tl/v, lambda in tw/w; every gate acts on both and
// TOP_GRAD accumulates Im<lambda|G|psi> into gsm).
template <typename C, int R, int NS>
__device__ __forceinline__ void run_program(C *tl, C *tw, uint64_t base, const PassDesc &d, const TOp *prog,
                                            const C *coef, double *gsm, uint32_t N) {
    constexpr int LOG2R = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : R == 16 ? 4 : 5;
    const uint32_t tid = threadIdx.x;
    C v[R];
    C w[NS == 2 ? R : 1];
    uint32_t bm[kPassMaxReg] = {0, 0, 0, 0, 0};
    uint32_t sb[LOG2R];  // swz of each register slot's tile bit
    uint32_t tb = 0, stb = 0;
    bool mapped = false;
    for (int p = 0; p < d.nprog; ++p) {
        const TOp op = prog[p];
        switch (op.kind) {
        case TOP_REMAP: {
            if (mapped) {
#pragma unroll
                for (int kk = 0; kk < R; ++kk) {
                    const uint32_t x = reg_sidx<LOG2R>(kk, stb, sb);
                    tl[x] = v[kk];
                    if constexpr (NS == 2) tw[x] = w[kk];
                }
            }
            __syncthreads();
            uint32_t regmask = 0;
#pragma unroll
            for (int q = 0; q < LOG2R; ++q) {
                bm[q] = 1u << op.bits[q];
                sb[q] = swz<C>(bm[q]);
                regmask |= bm[q];
            }
            tb = deposit_bits(tid, (N - 1) & ~regmask);
            stb = swz<C>(tb);
#pragma unroll
            for (int kk = 0; kk < R; ++kk) {
                const uint32_t x = reg_sidx<LOG2R>(kk, stb, sb);
                v[kk] = tl[x];
                if constexpr (NS == 2) w[kk] = tw[x];
            }
            __syncthreads();
            mapped = true;
            break;
        }
        case TOP_G1: {
            const C m0 = coef[op.coef], m1 = coef[op.coef + 1], m2 = coef[op.coef + 2], m3 = coef[op.coef + 3];
            switch (op.a) {
#define QK_G1(S)                                                   \
    case S:                                                        \
        reg_g1<S>(v, m0, m1, m2, m3);                              \
        if constexpr (NS == 2) reg_g1<S>(w, m0, m1, m2, m3);       \
        break;
            QK_G1(0) QK_G1(1) QK_G1(2) QK_G1(3) QK_G1(4)
#undef QK_G1
            }
            break;
        }
        case TOP_G2: {
            const C *m = coef + op.coef;
            switch (op.a * 8 + op.b) {
#define QK_G2(A, B)                                     \
    case A * 8 + B:                                     \
        reg_g2<A, B>(v, m);                             \
        if constexpr (NS == 2) reg_g2<A, B>(w, m);      \
        break;
            QK_G2(0, 1) QK_G2(0, 2) QK_G2(0, 3) QK_G2(0, 4) QK_G2(1, 2)
            QK_G2(1, 3) QK_G2(1, 4) QK_G2(2, 3) QK_G2(2, 4) QK_G2(3, 4)
#undef QK_G2
            }
            break;
        }
        case TOP_DIAG: {
            const C d0 = coef[op.coef], d1 = coef[op.coef + 1], d2 = coef[op.coef + 2], d3 = coef[op.coef + 3];
            const uint32_t A = bit_set<LOG2R>(op.a, 0, base, tb, bm), B = bit_set<LOG2R>(op.b, 0, base, tb, bm);
#pragma unroll
            for (int kk = 0; kk < R; ++kk) {
                const uint32_t idx = ((A >> kk) & 1) | (((B >> kk) & 1) << 1);
                const C ph = idx == 0 ? d0 : idx == 1 ? d1 : idx == 2 ? d2 : d3;
                v[kk] = cmul(v[kk], ph);
                if constexpr (NS == 2) w[kk] = cmul(w[kk], ph);
            }
            break;
        }
        case TOP_PHASE: {
            const C ph = coef[op.coef];
            const uint32_t M = bit_set<LOG2R>(op.a, 1, base, tb, bm) & bit_set<LOG2R>(op.b, 1, base, tb, bm);
            if (!(M & ((R >= 32) ? 0xFFFFFFFFu : ((1u << R) - 1)))) break;
#pragma unroll
            for (int kk = 0; kk < R; ++kk)
                if ((M >> kk) & 1) {
                    v[kk] = cmul(v[kk], ph);
                    if constexpr (NS == 2) w[kk] = cmul(w[kk], ph);
                }
            break;
        }
        case TOP_GRAD: {
            if constexpr (NS == 2) {
                double g = 0;
                switch (op.a) {
                case 0: g = reg_grad<0>(v, w, op.b); break;
                case 1: g = reg_grad<1>(v, w, op.b); break;
                case 2: g = reg_grad<2>(v, w, op.b); break;
                case 3: g = reg_grad<3>(v, w, op.b); break;
                case 4: g = reg_grad<4>(v, w, op.b); break;
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
                if ((tid & 31) == 0) atomicAdd(gsm + op.coef, g);
            }
            break;
        }
        }
    }
    if (mapped) {
#pragma unroll
        for (int kk = 0; kk < R; ++kk) {
            const uint32_t x = reg_sidx<LOG2R>(kk, stb, sb);
            tl[x] = v[kk];
            if constexpr (NS == 2) tw[x] = w[kk];
        }
    }
}

// nbuf = 2: the next tile is prefetched (cp.async) into the other buffer
// while the current one is processed; nbuf = 1: load, process, store.
// NS = 2 runs an adjoint pass over psi (s) and lambda (s2) together; the
// gradient accumulators of the pass live in shared memory and are added to
// ggrad[gparams[grad0 + i]] once per CTA.
template <typename C, int R, int NS>
__global__ void __launch_bounds__(kPassThreads) k_pass(C *__restrict__ s, C *__restrict__ s2, uint64_t ntiles,
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
        for (uint64_t o = blockIdx.x; o < ntiles; o += gridDim.x) {
            const uint64_t base = pass_base(o, d);
            for (uint32_t j = threadIdx.x; j < N; j += NT) buf0[swz<C>(j)] = s[base | pass_off(j, d)];
            __syncthreads();
            run_perm_tile(s, buf0, base, d, N, NT);
            __syncthreads();
        }
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
        run_program<C, R, NS>(tl, tw, base, d, prog, coef, gsm, N);
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

template <typename C, int R, int NS>
static int launch_pass_r(const PassArgs<C> &a, int n, const PassDesc &d, cudaStream_t st) {
    static int sms = 0;
    const size_t tile = (sizeof(C) << d.T) * NS;
    const int nbuf = d.perm ? 1 : (2 * tile <= (200u << 10) ? 2 : 1);
    const size_t smem = tile * nbuf + d.nprog * sizeof(TOp) + d.ncoef * sizeof(C) + (NS == 2 ? d.ngrad * sizeof(double) : 0);
    if (smem > (220u << 10)) return fail(QK_ERR_ARG, "pass needs %zu bytes of shared memory", smem);
    cudaError_t e;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        e = cudaFuncSetAttribute(k_pass<C, R, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 << 10);
        if (e != cudaSuccess) return cuda_err(e, "cudaFuncSetAttribute(k_pass)");
    }
    const uint32_t threads = d.perm ? std::max<uint32_t>(1, std::min<uint32_t>(kPassThreads, 1u << d.T))
                                    : (uint32_t)((1u << d.T) / R);
    if (threads > kPassThreads || threads == 0) return fail(QK_ERR_ARG, "pass of %d tile bits needs %u threads", d.T, threads);
    int mb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mb, k_pass<C, R, NS>, (int)threads, smem);
    if (e != cudaSuccess || mb < 1) mb = 1;
    const uint64_t ntiles = 1ull << (n - d.T);
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sms * mb);
    k_pass<C, R, NS><<<grid, threads, smem, st>>>(a.s, a.s2, ntiles, d, a.ops, a.coef, a.gparams, a.ggrad, nbuf);
    e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_err(e, "k_pass launch");
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
    PassArgs<C> a{s, s2, ops, coef, gparams, ggrad};
    // register-resident amplitudes per thread: up to 8 complex128 or 16
    // complex64 per state (more would spill)
    if (s2) {
        switch (r) {
        case 1: return launch_pass_r<C, 2, 2>(a, n, d, st);
        case 2: return launch_pass_r<C, 4, 2>(a, n, d, st);
        case 3:
            if constexpr (sizeof(C) == sizeof(float2)) return launch_pass_r<C, 8, 2>(a, n, d, st);
            break;
        }
        return fail(QK_ERR_ARG, "reg_bits %d unsupported for two-state passes", r);
    }
    switch (r) {
    case 1: return launch_pass_r<C, 2, 1>(a, n, d, st);
    case 2: return launch_pass_r<C, 4, 1>(a, n, d, st);
    case 3: return launch_pass_r<C, 8, 1>(a, n, d, st);
    case 4:
        if constexpr (sizeof(C) == sizeof(float2)) return launch_pass_r<C, 16, 1>(a, n, d, st);
        break;
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
    if (nc) {
        if (dtype == QK_C128) {
            e = cudaMemcpyAsync(dp.coef, hp.coef.data(), nc * sizeof(double2), cudaMemcpyHostToDevice, st);
        } else {
            std::vector<float> f(hp.coef.begin(), hp.coef.end());
            e = cudaMemcpyAsync(dp.coef, f.data(), nc * sizeof(float2), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // f is a temporary
        }
        if (e != cudaSuccess) return cuda_err(e, "upload plan coefficients");
    }
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

struct qk_plan {
    HostPlan hp;
    DevPlan dp;
    bool uploaded = false;
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
    qk_gate g;
    std::memset(&g, 0, sizeof g);
    g.kind = QK_GATE_VSWAP;
    g.nq = op.nq;
    for (int i = 0; i < op.nq; ++i) g.q[i] = op.q[i];
    PlanOptions o = default_plan_options(dtype, n);
    int rc = build_plan(&g, 1, n, o, hp);
    if (rc) return rc;
    DevPlan none;
    return run_plan(state, dtype, hp, none, st);
}

void release_scratch_plan(DevPlan &dp) { dp.release(); }
}  // namespace qk

extern "C" {

int qk_plan_create(const qk_gate *gates, size_t n, int nqubits, const qk_plan_opts *opts, qk_plan **out) {
    if (!out || (!gates && n)) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 36) return fail(QK_ERR_ARG, "nqubits must be in [1, 36], got %d", nqubits);
    const int dtype = opts ? opts->dtype : QK_C128;
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
    if (passes) *passes = p->hp.passes.size();
    if (program_ops) *program_ops = p->hp.ops.size();
    if (remaps) *remaps = p->hp.nremaps;
    return QK_OK;
}

int qk_plan_apply(qk_sv *sv, qk_plan *p) {
    if (!sv || !p) return fail(QK_ERR_ARG, "null argument");
    if (state_qubits(sv) != p->hp.n || state_dtype(sv) != p->hp.dtype)
        return fail(QK_ERR_ARG, "plan built for %d qubits dtype %d, state has %d qubits dtype %d", p->hp.n,
                    p->hp.dtype, state_qubits(sv), state_dtype(sv));
    if (!p->uploaded) {
        int rc = upload_plan(p->hp, p->hp.dtype, p->dp, state_stream(sv));
        if (rc) return rc;
        cudaError_t e = cudaStreamSynchronize(state_stream(sv));
        if (e != cudaSuccess) return cuda_err(e, "plan upload");
        p->uploaded = true;
    }
    return run_plan(state_ptr(sv), p->hp.dtype, p->hp, p->dp, state_stream(sv));
}

void qk_plan_destroy(qk_plan *p) {
    if (!p) return;
    p->dp.release();
    delete p;
}

}  // extern "C"
