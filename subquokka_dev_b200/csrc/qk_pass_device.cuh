// Device building blocks of the fused-pass kernels (single-circuit passes in
// qk_pass.cu, batched passes in qk_batch.cu): tile addressing, the shared-
// memory layout, cp.async staging and the per-tile program interpreter.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "qk_internal.h"
#include "qk_kernels.cuh"

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

// Threads per CTA bound of a pass kernel: 512, or 256 when a thread's
// register amplitudes take 256 bytes (complex128 with 16 amplitudes, or 8 of
// each of two states; about 220-240 registers a thread).
template <typename C, int R, int NS>
constexpr int pass_max_threads() {
    return sizeof(C) * R * NS >= 256 ? 256 : kPassThreads;
}

// The complex128 single-state pass with 16 amplitudes a thread on its
// default 2048-amplitude tiles has 128 threads; a second instance of it is
// bounded to 128 threads and three CTAs an SM: 168 registers instead of 241,
// 12 warps an SM instead of 8 (0.645 -> 0.600 s on the 30-qubit random
// circuit).
template <typename C, int R, int NS>
constexpr bool pass_narrow_ok() {
    return sizeof(C) == 16 && R == 16 && NS == 1;
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

// Real 2x2 on register slot S: c0 = (m00, m01), c1 = (m10, m11); two
// multiply-adds a component instead of the complex 2x2's four.
template <int S, typename C, int R>
__device__ __forceinline__ void reg_r1(C (&v)[R], const C c0, const C c1) {
    if constexpr ((1 << S) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & (1 << S)) continue;
            const C a = v[k], b = v[k | (1 << S)];
            v[k].x = fma(c0.x, a.x, c0.y * b.x);
            v[k].y = fma(c0.x, a.y, c0.y * b.y);
            v[k | (1 << S)].x = fma(c1.x, a.x, c1.y * b.x);
            v[k | (1 << S)].y = fma(c1.x, a.y, c1.y * b.y);
        }
    }
}

// Real 4x4 on register slots A < B (index bit 0 = A): m[2 r + h] =
// (row r's entries 2h, 2h + 1).
template <int A, int B, typename C, int R>
__device__ __forceinline__ void reg_r2(C (&v)[R], const C *__restrict__ m) {
    if constexpr (A < B && (1 << B) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & ((1 << A) | (1 << B))) continue;
            const int k1 = k | (1 << A), k2 = k | (1 << B), k3 = k | (1 << A) | (1 << B);
            const C x0 = v[k], x1 = v[k1], x2 = v[k2], x3 = v[k3];
            C y[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const C p = m[2 * r], q = m[2 * r + 1];
                y[r].x = fma(p.x, x0.x, fma(p.y, x1.x, fma(q.x, x2.x, q.y * x3.x)));
                y[r].y = fma(p.x, x0.y, fma(p.y, x1.y, fma(q.x, x2.y, q.y * x3.y)));
            }
            v[k] = y[0];
            v[k1] = y[1];
            v[k2] = y[2];
            v[k3] = y[3];
        }
    }
}

// Phase on the register elements whose bit S (and bit T) is set.
template <int S, typename C, int R>
__device__ __forceinline__ void reg_phase1(C (&v)[R], const C ph) {
    if constexpr ((1 << S) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k)
            if (k & (1 << S)) v[k] = cmul(v[k], ph);
    }
}
template <int S, int T, typename C, int R>
__device__ __forceinline__ void reg_phase2(C (&v)[R], const C ph) {
    if constexpr ((1 << S) < R && (1 << T) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k)
            if ((k & (1 << S)) && (k & (1 << T))) v[k] = cmul(v[k], ph);
    }
}

// Every register amplitude of the thread (both states) times f.
template <typename C, int R, int NW>
__device__ __forceinline__ void scale_regs(C (&v)[R], C (&w)[NW], const C f) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        v[k] = cmul(v[k], f);
        if constexpr (NW == R) w[k] = cmul(w[k], f);
    }
}

// Controlled X on register slot S: swap the pair (k, k | 2^S) where bit k of
// M (the control's value at register index k) is set.
template <int S, typename C, int R>
__device__ __forceinline__ void reg_cx(C (&v)[R], uint32_t M) {
    if constexpr ((1 << S) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & (1 << S)) continue;
            const bool f = (M >> k) & 1;
            const C a = v[k], b = v[k | (1 << S)];
            v[k] = f ? b : a;
            v[k | (1 << S)] = f ? a : b;
        }
    }
}

template <int A, int B, typename C, int R>
__device__ __forceinline__ void reg_g2(C (&v)[R], const C *__restrict__ m) {
    if constexpr (A < B && (1 << B) < R && sizeof(C) == 16 && R >= 8) {
        // complex128: row by row, each row's four coefficients loaded once and
        // applied to every quad of the thread's registers (567 against 575 ms
        // on the 30-qubit circuit; complex64 is faster quad by quad, 356
        // against 381 ms)
        C y[R];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const C a = m[4 * r], b = m[4 * r + 1], c = m[4 * r + 2], e = m[4 * r + 3];
#pragma unroll
            for (int k = 0; k < R; ++k) {
                if (k & ((1 << A) | (1 << B))) continue;
                const int k1 = k | (1 << A), k2 = k | (1 << B), k3 = k | (1 << A) | (1 << B);
                const int out = (r & 1 ? (1 << A) : 0) | (r & 2 ? (1 << B) : 0) | k;
                const C x0 = v[k], x1 = v[k1], x2 = v[k2], x3 = v[k3];
                y[out].x = fma(a.x, x0.x, fma(-a.y, x0.y, fma(b.x, x1.x, fma(-b.y, x1.y,
                           fma(c.x, x2.x, fma(-c.y, x2.y, fma(e.x, x3.x, -e.y * x3.y)))))));
                y[out].y = fma(a.x, x0.y, fma(a.y, x0.x, fma(b.x, x1.y, fma(b.y, x1.x,
                           fma(c.x, x2.y, fma(c.y, x2.x, fma(e.x, x3.y, e.y * x3.x)))))));
            }
        }
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = y[k];
    } else if constexpr (A < B && (1 << B) < R) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (k & ((1 << A) | (1 << B))) continue;
            const int k1 = k | (1 << A), k2 = k | (1 << B), k3 = k | (1 << A) | (1 << B);
            const C x0 = v[k], x1 = v[k1], x2 = v[k2], x3 = v[k3];
            C y[4];
            // one chain of eight fused multiply-adds per component: fewer
            // live values than two chains and an add (fewer spills in the
            // complex128 pass; 0.599 -> 0.574 s c128, 0.412 -> 0.390 s c64 on
            // the 30-qubit circuit)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const C a = m[4 * r], b = m[4 * r + 1], c = m[4 * r + 2], e = m[4 * r + 3];
                y[r].x = fma(a.x, x0.x, fma(-a.y, x0.y, fma(b.x, x1.x, fma(-b.y, x1.y,
                         fma(c.x, x2.x, fma(-c.y, x2.y, fma(e.x, x3.x, -e.y * x3.y)))))));
                y[r].y = fma(a.x, x0.y, fma(a.y, x0.x, fma(b.x, x1.y, fma(b.y, x1.x,
                         fma(c.x, x2.y, fma(c.y, x2.x, fma(e.x, x3.y, e.y * x3.x)))))));
            }
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

// Tile-local image of j under a permutation pass's bit-pair swaps.
__device__ __forceinline__ uint32_t perm_bits(uint32_t j, const PassDesc &d) {
    uint32_t f = j;
    for (int i = 0; i < d.nperm; ++i) {
        const uint32_t a = (j >> d.perm_a[i]) & 1, b = (j >> d.perm_b[i]) & 1;
        f = (f & ~(1u << d.perm_a[i]) & ~(1u << d.perm_b[i])) | (b << d.perm_a[i]) | (a << d.perm_b[i]);
    }
    return f;
}

// Permutation pass: tile element j goes to the position of perm(j) (perm
// is a product of disjoint bit-pair swaps, its own inverse).  A thread
// loads the elements f = tid + i NT (i < N / NT <= 32) and stores, at the
// same positions, the elements perm(f), read from the shared-memory tile:
// both global accesses stay in the tile's contiguous runs, the permutation
// is a shared-memory gather.  The state offset (a bit deposit) and the
// shared-memory indices of f and perm(f) (an XOR fold) are each linear in f
// over disjoint bits, so each is the thread's part combined with the parts
// of the set bits of i, computed once per thread.
template <typename C>
__device__ void run_perm_pass(C *__restrict__ s, C *buf, uint64_t ntiles, const PassDesc &d, uint32_t N,
                              uint32_t NT) {
    constexpr int kMaxB = 5;
    const uint32_t tid = threadIdx.x;
    const uint64_t g_t = pass_off(tid, d);
    const uint32_t sw_t = swz<C>(tid), sp_t = swz<C>(perm_bits(tid, d));
    uint64_t g_u[kMaxB];
    uint32_t sw_u[kMaxB], sp_u[kMaxB];
    int nb = 0;
#pragma unroll
    for (int b = 0; b < kMaxB; ++b) {
        const uint32_t m = NT << b;
        g_u[b] = m < N ? pass_off(m, d) : 0;
        sw_u[b] = m < N ? swz<C>(m) : 0;
        sp_u[b] = m < N ? swz<C>(perm_bits(m, d)) : 0;
        nb += m < N;
    }
    const uint32_t R = 1u << nb;
    for (uint64_t o = blockIdx.x; o < ntiles; o += gridDim.x) {
        const uint64_t base = pass_base(o, d);
        for (uint32_t i = 0; i < R; ++i) {
            uint64_t a = g_t;
            uint32_t x = sw_t;
#pragma unroll
            for (int b = 0; b < kMaxB; ++b)
                if ((i >> b) & 1) { a |= g_u[b]; x ^= sw_u[b]; }
            cp_async_amp(buf + x, s + (base | a));
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        for (uint32_t i = 0; i < R; ++i) {
            uint64_t a = g_t;
            uint32_t x = sp_t;
#pragma unroll
            for (int b = 0; b < kMaxB; ++b)
                if ((i >> b) & 1) { a |= g_u[b]; x ^= sp_u[b]; }
            s[base | a] = buf[x];
        }
        __syncthreads();
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

// The same two lookups with the register slot supplied by the planner
// (kNoSlot: the qubit is a thread bit, an outer bit, or none).
__device__ __forceinline__ uint32_t bit_set_at(uint8_t code, uint8_t slot, uint32_t none, uint64_t base, uint32_t tb) {
    if (slot != kNoSlot) return slot_pattern(slot);
    if (code == kNoQubit) return none ? 0xFFFFFFFFu : 0u;
    if (code & kOuterFlag) return ((base >> (code & 0x7F)) & 1) ? 0xFFFFFFFFu : 0u;
    return (tb >> code) & 1 ? 0xFFFFFFFFu : 0u;
}
__device__ __forceinline__ int code_slot_at(uint8_t code, uint8_t slot, uint64_t base, uint32_t tb, uint32_t *bit) {
    *bit = 0;
    if (slot != kNoSlot) return slot;
    if (code == kNoQubit) return -1;
    *bit = (code & kOuterFlag) ? (uint32_t)(base >> (code & 0x7F)) & 1u : (tb >> code) & 1u;
    return -1;
}

// Register slot holding a diagonal-op qubit code, or -1 with *bit set to the
// qubit's value, which is then the same for every register element.
template <int LOG2R>
__device__ __forceinline__ int code_slot(uint8_t code, uint64_t base, uint32_t tb, const uint32_t (&bm)[kPassMaxReg],
                                         uint32_t *bit) {
    *bit = 0;
    if (code == kNoQubit) return -1;
    if (code & kOuterFlag) {
        *bit = (uint32_t)(base >> (code & 0x7F)) & 1u;
        return -1;
    }
    const uint32_t m = 1u << code;
#pragma unroll
    for (int s = 0; s < LOG2R; ++s)
        if (bm[s] == m) return s;
    *bit = (tb & m) ? 1u : 0u;
    return -1;
}

// Diagonal phases by register element: element k gets p1 where bit S of k is
// set, else p0 (S = -1: p0 everywhere).
template <int S, typename C, int R>
__device__ __forceinline__ void reg_diag1(C (&v)[R], const C p0, const C p1) {
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = cmul(v[k], (S >= 0 && (k >> (S < 0 ? 0 : S)) & 1) ? p1 : p0);
}
// element k gets d[bit A of k + 2 bit B of k]
template <int A, int B, typename C, int R>
__device__ __forceinline__ void reg_diag2(C (&v)[R], const C d0, const C d1, const C d2, const C d3) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int i = ((k >> A) & 1) | (((k >> B) & 1) << 1);
        v[k] = cmul(v[k], i == 0 ? d0 : i == 1 ? d1 : i == 2 ? d2 : d3);
    }
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

// Im <lambda|G|psi> over this thread's register pairs of slot S, summed in
// the state's precision (a thread holds at most 16 pairs).  G = X, Y, Z by
// gen 1, 2, 3; gen 4: G = a X + b Y + c Z with (a, b) = g[0], (c, .) = g[1]
// (a Pauli generator carried past one-qubit gates U as U^dag P U); gen 5: two
// such generators (g[0..1], g[2..3]), the second sum in *s2.
template <int S, typename C, int R>
__device__ __forceinline__ auto reg_grad(const C (&v)[R], const C (&w)[R], int gen, const C *g,
                                         decltype(v[0].x) *s2) {
    using T = decltype(v[0].x);
    T s = 0;
    if constexpr ((1 << S) < R) {
        auto im = [](C l, C a) { return l.x * a.y - l.y * a.x; };
        auto re = [](C l, C a) { return l.x * a.x + l.y * a.y; };
        if (gen >= 4) {
            T sx = 0, sy = 0, sz = 0;
#pragma unroll
            for (int k = 0; k < R; ++k)
                if (!(k & (1 << S))) {
                    const C v0 = v[k], v1 = v[k | (1 << S)], w0 = w[k], w1 = w[k | (1 << S)];
                    sx += im(w0, v1) + im(w1, v0);
                    sy += re(w1, v0) - re(w0, v1);
                    sz += im(w0, v0) - im(w1, v1);
                }
            s = g[0].x * sx + g[0].y * sy + g[1].x * sz;
            if (gen == 5) *s2 = g[2].x * sx + g[2].y * sy + g[3].x * sz;
        } else if (gen == 1) {
#pragma unroll
            for (int k = 0; k < R; ++k)
                if (!(k & (1 << S))) s += im(w[k], v[k | (1 << S)]) + im(w[k | (1 << S)], v[k]);
        } else if (gen == 2) {
#pragma unroll
            for (int k = 0; k < R; ++k)
                if (!(k & (1 << S))) s += re(w[k | (1 << S)], v[k]) - re(w[k], v[k | (1 << S)]);
        } else {
#pragma unroll
            for (int k = 0; k < R; ++k)
                if (!(k & (1 << S))) s += im(w[k], v[k]) - im(w[k | (1 << S)], v[k | (1 << S)]);
        }
    }
    return s;
}

// Run a pass program on one tile (NS = 1) or on the matching tiles of two
// states (NS = 2: psi in tl/v, lambda in tw/w; every gate acts on both and
// TOP_GRAD accumulates Im<lambda|G|psi> into gsm).
template <typename C, int R, int NS, bool XOPS>
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
    // factor common to all of the thread's amplitudes (diagonal ops on
    // qubits outside the register slots), applied before they leave the
    // registers
    constexpr bool PEND = XOPS && pending_scalar_ok((int)sizeof(C), R, NS);
    C pend;
    pend.x = 1;
    pend.y = 0;
    bool pending = false;
    for (int p = 0; p < d.nprog; ++p) {
        const TOp op = prog[p];
        switch (op.kind) {
        case TOP_REMAP: {
            if constexpr (PEND) {
                if (pending) {
                    scale_regs(v, w, pend);
                    pend.x = 1;
                    pend.y = 0;
                    pending = false;
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
        case TOP_R1:
        case TOP_R2:
            if constexpr (XOPS) {
                if (op.kind == TOP_R1) {
                    const C c0 = coef[op.coef], c1 = coef[op.coef + 1];
                    switch (op.a) {
#define QK_R1(S)                                     \
    case S:                                          \
        reg_r1<S>(v, c0, c1);                        \
        if constexpr (NS == 2) reg_r1<S>(w, c0, c1); \
        break;
                    QK_R1(0) QK_R1(1) QK_R1(2) QK_R1(3) QK_R1(4)
#undef QK_R1
                    }
                } else {
                    const C *m = coef + op.coef;
                    switch (op.a * 8 + op.b) {
#define QK_R2(A, B)                                     \
    case A * 8 + B:                                     \
        reg_r2<A, B>(v, m);                             \
        if constexpr (NS == 2) reg_r2<A, B>(w, m);      \
        break;
                    QK_R2(0, 1) QK_R2(0, 2) QK_R2(0, 3) QK_R2(0, 4) QK_R2(1, 2)
                    QK_R2(1, 3) QK_R2(1, 4) QK_R2(2, 3) QK_R2(2, 4) QK_R2(3, 4)
#undef QK_R2
                    }
                }
            }
            break;
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
            // phases by the two qubits' values: a register-slot qubit varies
            // over the elements (pattern fixed at compile time), any other is
            // the same for all of them
            const C d0 = coef[op.coef], d1 = coef[op.coef + 1], d2 = coef[op.coef + 2], d3 = coef[op.coef + 3];
            uint32_t ba, bb;
            const int sa = code_slot_at(op.a, op.bits[0], base, tb, &ba), sb = code_slot_at(op.b, op.bits[1], base, tb, &bb);
            if (sa >= 0 && sb >= 0) {
                switch (sa * 8 + sb) {
#define QK_D2(A, B)                                                  \
    case A * 8 + B:                                                  \
        reg_diag2<A, B>(v, d0, d1, d2, d3);                          \
        if constexpr (NS == 2) reg_diag2<A, B>(w, d0, d1, d2, d3);   \
        break;                                                       \
    case B * 8 + A:                                                  \
        reg_diag2<B, A>(v, d0, d1, d2, d3);                          \
        if constexpr (NS == 2) reg_diag2<B, A>(w, d0, d1, d2, d3);   \
        break;
                QK_D2(0, 1) QK_D2(0, 2) QK_D2(0, 3) QK_D2(0, 4) QK_D2(1, 2)
                QK_D2(1, 3) QK_D2(1, 4) QK_D2(2, 3) QK_D2(2, 4) QK_D2(3, 4)
#undef QK_D2
                }
                break;
            }
            // at most one register-slot qubit: two phases p0 / p1 by its value
            const int sl = sa >= 0 ? sa : sb;
            C p0, p1;
            if (sa >= 0) { p0 = bb ? d2 : d0; p1 = bb ? d3 : d1; }
            else if (sb >= 0) { p0 = ba ? d1 : d0; p1 = ba ? d3 : d2; }
            else {
                // the same factor for all of the thread's amplitudes
                p0 = p1 = ba ? (bb ? d3 : d1) : (bb ? d2 : d0);
                if constexpr (PEND) {
                    pend = cmul(pend, p0);
                    pending = true;
                    break;
                }
            }
            switch (sl) {
#define QK_D1(S)                                       \
    case S:                                            \
        reg_diag1<S>(v, p0, p1);                       \
        if constexpr (NS == 2) reg_diag1<S>(w, p0, p1); \
        break;
            QK_D1(-1) QK_D1(0) QK_D1(1) QK_D1(2) QK_D1(3) QK_D1(4)
#undef QK_D1
            }
            break;
        }
        case TOP_CX: {
            const uint32_t M = bit_set_at(op.b, op.bits[1], 1, base, tb);
            switch (op.a) {
#define QK_CX(S)                                   \
    case S:                                        \
        reg_cx<S>(v, M);                           \
        if constexpr (NS == 2) reg_cx<S>(w, M);    \
        break;
            QK_CX(0) QK_CX(1) QK_CX(2) QK_CX(3) QK_CX(4)
#undef QK_CX
            }
            break;
        }
        case TOP_CG1: {
            // the condition qubit holds no register slot here, so its value is
            // the same for all of the thread's amplitudes: one 2x2 of the two
            const C *m = coef + op.coef + ((bit_set_at(op.b, op.bits[1], 0, base, tb) & 1u) ? 4 : 0);
            const C m0 = m[0], m1 = m[1], m2 = m[2], m3 = m[3];
            switch (op.a) {
#define QK_CG1(S)                                                  \
    case S:                                                        \
        reg_g1<S>(v, m0, m1, m2, m3);                              \
        if constexpr (NS == 2) reg_g1<S>(w, m0, m1, m2, m3);       \
        break;
            QK_CG1(0) QK_CG1(1) QK_CG1(2) QK_CG1(3) QK_CG1(4)
#undef QK_CG1
            }
            break;
        }
        case TOP_PHASE: {
            if constexpr (!XOPS) {
                const C ph = coef[op.coef];
                const uint32_t M = bit_set_at(op.a, op.bits[0], 1, base, tb) & bit_set_at(op.b, op.bits[1], 1, base, tb);
                if (!(M & ((R >= 32) ? 0xFFFFFFFFu : ((1u << R) - 1)))) break;
#pragma unroll
                for (int kk = 0; kk < R; ++kk)
                    if ((M >> kk) & 1) {
                        v[kk] = cmul(v[kk], ph);
                        if constexpr (NS == 2) w[kk] = cmul(w[kk], ph);
                    }
                break;
            } else {
                const C ph = coef[op.coef];
                uint32_t ba, bb;
                const int sa = code_slot_at(op.a, op.bits[0], base, tb, &ba);
                const int sb = code_slot_at(op.b, op.bits[1], base, tb, &bb);
                if (op.a == kNoQubit) ba = 1;
                if (op.b == kNoQubit) bb = 1;
                if (sa < 0 && sb < 0) {
                    if (ba & bb) {
                        if constexpr (PEND) {
                            pend = cmul(pend, ph);
                            pending = true;
                        } else {
                            scale_regs(v, w, ph);
                        }
                    }
                    break;
                }
                if (sa >= 0 && sb >= 0) {
                    switch (sa * 8 + sb) {
#define QK_P2(A, B)                                            \
    case A * 8 + B:                                            \
    case B * 8 + A:                                            \
        reg_phase2<A, B>(v, ph);                               \
        if constexpr (NS == 2) reg_phase2<A, B>(w, ph);        \
        break;
                    QK_P2(0, 1) QK_P2(0, 2) QK_P2(0, 3) QK_P2(0, 4) QK_P2(1, 2)
                    QK_P2(1, 3) QK_P2(1, 4) QK_P2(2, 3) QK_P2(2, 4) QK_P2(3, 4)
#undef QK_P2
                    }
                    break;
                }
                if (!(sa >= 0 ? bb : ba)) break;
                switch (sa >= 0 ? sa : sb) {
#define QK_P1(S)                                       \
    case S:                                            \
        reg_phase1<S>(v, ph);                          \
        if constexpr (NS == 2) reg_phase1<S>(w, ph);   \
        break;
                QK_P1(0) QK_P1(1) QK_P1(2) QK_P1(3) QK_P1(4)
#undef QK_P1
                }
                break;
            }
        }
        case TOP_GRAD: {
            if constexpr (NS == 2) {
                if constexpr (PEND) {
                    if (pending) {
                        scale_regs(v, w, pend);
                        pend.x = 1;
                        pend.y = 0;
                        pending = false;
                    }
                }
                // summed over the warp in the state's precision, added to
                // the CTA's double accumulator once per warp
                decltype(v[0].x) g = 0, g2 = 0;
                const C *gc = coef + op.coef;
                switch (op.a) {
                case 0: g = reg_grad<0>(v, w, op.b, gc, &g2); break;
                case 1: g = reg_grad<1>(v, w, op.b, gc, &g2); break;
                case 2: g = reg_grad<2>(v, w, op.b, gc, &g2); break;
                case 3: g = reg_grad<3>(v, w, op.b, gc, &g2); break;
                case 4: g = reg_grad<4>(v, w, op.b, gc, &g2); break;
                }
                // a tile of fewer than 32 threads (2^(T - r) < 32) is a
                // partial warp: the shuffles stay within its lanes
                const uint32_t nl = blockDim.x < 32 ? blockDim.x : 32;
                const uint32_t lanes = nl == 32 ? 0xffffffffu : (1u << nl) - 1;
#pragma unroll
                for (uint32_t o = 16; o; o >>= 1)
                    if (o < nl) g += __shfl_xor_sync(lanes, g, (int)o);
                if ((tid & 31) == 0) atomicAdd(gsm + (op.bits[0] | (op.bits[1] << 8)), (double)g);
                if (op.b == 5) {
#pragma unroll
                    for (uint32_t o = 16; o; o >>= 1)
                        if (o < nl) g2 += __shfl_xor_sync(lanes, g2, (int)o);
                    if ((tid & 31) == 0) atomicAdd(gsm + (op.bits[2] | (op.bits[3] << 8)), (double)g2);
                }
            }
            break;
        }
        }
    }
    if (mapped) {
        if constexpr (PEND) {
            if (pending) scale_regs(v, w, pend);
        }
#pragma unroll
        for (int kk = 0; kk < R; ++kk) {
            const uint32_t x = reg_sidx<LOG2R>(kk, stb, sb);
            tl[x] = v[kk];
            if constexpr (NS == 2) tw[x] = w[kk];
        }
    }
}

}  // namespace qk
