// Dense fused blocks on the 5th-generation tensor cores (complex64 states).
//
// A block is a 64 x 64 complex unitary U on six qubits (the product of
// consecutive gates, built on the host in FP64).  A pass applies one block to
// the whole state.  Each CTA owns one SM, loads the block's operand once,
// and streams supertiles of 64 x 128 amplitudes (the block's six qubits plus
// the lowest seven other state bits; 64 x 64 at 12 qubits):
//
//   supertile as X[i][n]: i = block-qubit index (64), n = other tile bits (128)
//   real embedding, columns interleaved (2i + re/im):
//     S[n][2i+b]  = (re, im)_b X[i][n]                           (128 x 128)
//     W[2i'+a][2i+b] = [[Ur, -Ui], [Ui, Ur]][a][b](i', i)         (128 x 128)
//     D[n][m] = sum_k S[n][k] W[m][k]   ->  X'[i'][n] = D[n][2i'] + i D[n][2i'+1]
//   split precision (3 x BF16, FP32 accumulate in TMEM):
//     S = Sh + Sl, W = Wh + Wl,  D = Sh Wh + Sl Wh + Sh Wl   (K = 3 x 128)
//
// 24 tcgen05.mma (M128 N128 K16, kind::f16, BF16 operands) per supertile,
// issued by one thread, completion through tcgen05.commit -> mbarrier.  The
// state is the M operand so that TMEM lane = state row n: after tcgen05.ld a
// thread holds whole (re, im) pairs of one row, and a warp's stores run along
// n, the contiguous direction of the state whenever the block does not own
// qubit 0.  Operands sit in shared memory in the canonical K-major
// 128-byte-swizzle layout (rows of 64 K elements, 16-byte chunks XORed with
// the row index mod 8, SBO = 1024 B between 8-row groups, atoms 1024-byte
// aligned); an MMA step's descriptor points at its 32 bytes inside the atom.
//
// Pipeline per CTA (state operand double-buffered in shared memory, two
// accumulators in TMEM): convert supertile s into buffer s % 2, issue its
// contraction, load supertile s + 2 grid into the registers it came from
// (two register sets keep two supertiles of loads in flight), then wait for
// contraction s - 1 and drain its accumulator straight to HBM.  Each thread
// loads and stores the same 16 amplitudes of every supertile (row n, block
// indices 16 (tid / 128) ..).
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "qk_device.h"
#include "qk_internal.h"
#include "qk_pass_device.cuh"
#include "qk_operand.h"
#include "qk_tc_device.cuh"

namespace qk {

constexpr int kTcDataWarps = 16;                     // load, convert, drain
constexpr int kTcThreads = 32 * (kTcDataWarps + 1);   // + one MMA-issuer warp
constexpr int kTcMaxTileBits = 13;                    // 64 x 128 amplitudes
constexpr int kTcMinTileBits = 12;                    // 64 x 64
constexpr uint32_t kTcOpBytes = 128 * 128 * 2;        // one 128 x 128 bf16 operand
constexpr uint32_t kTcSmem = 6 * kTcOpBytes;          // W hi/lo + two state buffers hi/lo
constexpr uint32_t kTcTmemCols = 256;                 // two 128-column accumulators

// Shared-memory descriptor of MMA step kk (K = 16 kk .. 16 kk + 15) of an
// operand at saddr (1024-byte aligned): the step's 32 bytes inside its atom.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, int kk) {
    return sw128_desc(saddr + (uint32_t)(kk >> 2) * 16384u + (uint32_t)(kk & 3) * 32u);
}

// kind::f16, A = B = BF16, D = F32, both K-major, M = 128, N = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void store_bf16x8(unsigned char *dst, const float *v) {
    uint4 w;
    uint32_t *u = reinterpret_cast<uint32_t *>(&w);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
        u[k] = *reinterpret_cast<const uint32_t *>(&h);
    }
    *reinterpret_cast<uint4 *>(dst) = w;
}

// Per-thread work of one supertile, two layouts:
//
// STATE_M (the block does not own qubit 0; the supertile's n index runs along
// the contiguous direction of the state): the state is the M operand,
// D[n][m] = sum_k S[n][k] W[m][k], TMEM lane = row n.  Thread t owns row
// n = t % 128 and block indices 16 (t / 128) .. + 15: it loads them (warp
// lanes along n), converts them into 16-byte K chunks, and drains the same
// amplitudes from TMEM lane n, columns 32 (t / 128) .. + 31.
//
// STATE_N (the block owns qubit 0; block indices run along the contiguous
// direction): the state is the N operand, D[m][n] = sum_k W[m][k] S[n][k],
// TMEM lane = m = 2 i' + re/im.  Loads take chunks of four consecutive block
// indices (two 16-byte vectors) with warp lanes over n bits 0-2 and chunk
// bits 0-1; the drain pairs re/im lanes with one shuffle so that each lane
// stores whole amplitudes, the warp's stores running along i'.
//
// NROWS = state rows per supertile: 128, or 64 for a 12-qubit state (rows
// 64..127 of the state operand then stay zero and are not stored).
template <int NROWS, bool STATE_N>
__global__ void __launch_bounds__(kTcThreads, 1) k_dense_tc(float2 *__restrict__ s, uint64_t nsup,
                                                            const __grid_constant__ DenseDesc dd,
                                                            const uint16_t *__restrict__ gW, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    // full[b]: buffer b converted (one arrival per data warp); mma[b]: the
    // contraction of buffer b done (tcgen05.commit); empty[b]: accumulator b
    // drained (one arrival per data warp); fin: every MMA the issuer ever
    // issued has completed (its last tcgen05.commit, made on every exit path)
    __shared__ __align__(8) uint64_t full[2], mma[2], empty[2], fin;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int bad_s;
    const PassDesc &d = dd.p;
    unsigned char *Wh = sm;
    unsigned char *Wl = Wh + kTcOpBytes;
    unsigned char *S0 = Wl + kTcOpBytes;    // buffer b: hi at S0 + 2b op, lo after it
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool issuer = warp == kTcDataWarps;
    if (s_u32(sm) & 1023u) {   // the swizzle pattern needs 1024-byte aligned operands
        if (tid == 0) atomicExch(err, 2);
        return;
    }

    for (uint32_t i = tid; i < 2 * kTcOpBytes / 16; i += kTcThreads)
        reinterpret_cast<uint4 *>(Wh)[i] = reinterpret_cast<const uint4 *>(gW)[i];
    if (NROWS < 128)
        for (uint32_t i = tid; i < 4 * kTcOpBytes / 16; i += kTcThreads)
            reinterpret_cast<uint4 *>(S0)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        bad_s = 0;
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&full[b])), "r"(kTcDataWarps) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&mma[b])), "r"(1) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&empty[b])), "r"(kTcDataWarps) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&fin)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (issuer) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&tmem_slot)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }

    // data warps: this thread's state row n and block indices 16 cg .. 16 cg + 15
    // (STATE_M: loads, conversion and, as TMEM lane n / columns 32 cg .., the
    // drain), offset of amplitude k = lrow + sum of le[b], b in bits(k);
    // STATE_N: load chunk u at lrow + lu[u] (+ lpair for its second pair),
    // drain lane at drow + sum of de[b] over the bits of its column index
    const uint32_t tmask = (1u << d.T) - 1, nmask = tmask & ~dd.blockmask;
    auto jn = [&](uint32_t v) { return pass_off(deposit_bits(v, nmask), d); };
    auto jb = [&](uint32_t v) { return pass_off(deposit_bits(v, dd.blockmask), d); };
    uint32_t n_m = 0, cg_m = 0, conv_n = 0, conv_c = 0;
    bool active = true;
    uint64_t lrow = 0, le[4] = {0, 0, 0, 0}, lu[2] = {0, 0}, lpair = 0, drow = 0, de[4] = {0, 0, 0, 0};
    if (!issuer) {
        if constexpr (!STATE_N) {
            n_m = tid & 127;
            cg_m = tid >> 7;
            active = n_m < NROWS;
            lrow = jn(n_m) + jb(16 * cg_m);
#pragma unroll
            for (int b = 0; b < 4; ++b) le[b] = jb(1u << b);
        } else {
            // chunk (n, c), n = (t & 7) | ((t >> 7) & 3) << 3 | u << 5, c = (t >> 3) & 15
            conv_n = (tid & 7) | (((tid >> 7) & 3) << 3);
            conv_c = (tid >> 3) & 15;
            lrow = jn(conv_n) + jb(4 * conv_c);
            lu[0] = jn(32);
            lu[1] = jn(64);
            lpair = jb(2);
            // drain: lanes m = 32 (warp % 4) + lane, columns 32 (warp / 4) + 16 h + 2 j + (lane & 1)
            drow = jb(16 * (warp & 3) + (lane >> 1)) + jn(32 * (warp >> 2) + (lane & 1));
#pragma unroll
            for (int b = 0; b < 4; ++b) de[b] = jn(2u << b);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    // each CTA takes a contiguous range of supertiles: consecutive supertiles
    // are neighbours along the lowest state bit outside the tile, so a CTA
    // streams each of the block's 64 row runs forward instead of striding
    const uint64_t o_lo = nsup * blockIdx.x / gridDim.x, o_hi = nsup * (blockIdx.x + 1) / gridDim.x;

    if (issuer) {
        // one thread issues every contraction: wait until buffer b is
        // converted and accumulator b drained, then 24 MMAs and a commit
        if (lane == 0) {
            uint32_t it = 0;
            for (uint64_t o = o_lo; o < o_hi && !bad_s; ++o, ++it) {
                const uint32_t b = it & 1;
                if (!tc_wait(&full[b], (it >> 1) & 1u) || (it >= 2 && !tc_wait(&empty[b], ((it - 2) >> 1) & 1u))) {
                    bad_s = 1;
                    break;
                }
                tc_fence_after();
                const unsigned char *Sh = S0 + 2 * b * kTcOpBytes, *Sl = Sh + kTcOpBytes;
#pragma unroll 1
                for (int sp = 0; sp < 3; ++sp) {   // S W products: hi hi, lo hi, hi lo
                    const uint32_t sa = s_u32(sp == 1 ? Sl : Sh), w = s_u32(sp == 2 ? Wl : Wh);
#pragma unroll 1
                    for (int kk = 0; kk < 8; ++kk) {
                        const uint64_t sd = umma_desc(sa, kk), wd = umma_desc(w, kk);
                        const uint64_t ad = STATE_N ? wd : sd, bd = STATE_N ? sd : wd;
                        const uint32_t acc = (sp | kk) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                tmem + b * 128u),
                            "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                            : "memory");
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 s_u32(&mma[b]))
                             : "memory");
            }
            // Teardown invariant: the TMEM is released only after every MMA
            // issued above has completed.  On the normal path the data warps
            // have already waited for the last contraction; on a timeout they
            // stop early, so MMAs of one or two supertiles may still be in
            // flight.  tcgen05.commit tracks all earlier tcgen05 operations of
            // this thread, so one more commit on `fin` arrives only after all
            // of them; the wait is bounded like every other, and a wait that
            // runs out is reported (error 3) before the dealloc.
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             s_u32(&fin))
                         : "memory");
            if (!tc_wait(&fin, 0)) {
                bad_s = 1;
                atomicExch(err, 3);
            }
        }
        __syncwarp();   // the issuer warp reaches the final barrier converged
    } else {
        auto load = [&](float2 (&x)[16], const float2 *p) {
            if constexpr (!STATE_N) {
                if (active) {
                    const float2 *q[16];
                    q[0] = p + lrow;
#pragma unroll
                    for (int k = 1; k < 16; ++k)
                        q[k] = q[k & (k - 1)] + le[(k & 1) ? 0 : (k & 2) ? 1 : (k & 4) ? 2 : 3];
#pragma unroll
                    for (int k = 0; k < 16; ++k) x[k] = *q[k];
                }
            } else {
                constexpr int NU = NROWS / 32;   // chunks per thread
#pragma unroll
                for (int u = 0; u < NU; ++u) {
                    const float2 *q = p + lrow + (u & 1 ? lu[0] : 0) + (u & 2 ? lu[1] : 0);
                    if (lpair == 2 && (reinterpret_cast<uintptr_t>(q) & 31) == 0) {
                        // block bits 0, 1 are state bits 0, 1: the chunk is one
                        // 32-byte sector, read by one 256-bit load
                        float r[8];
                        asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                                     : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]),
                                       "=f"(r[6]), "=f"(r[7])
                                     : "l"(q));
#pragma unroll
                        for (int k = 0; k < 4; ++k) x[4 * u + k] = make_float2(r[2 * k], r[2 * k + 1]);
                    } else {
                        const float4 v0 = *reinterpret_cast<const float4 *>(q);
                        const float4 v1 = *reinterpret_cast<const float4 *>(q + lpair);
                        x[4 * u + 0] = make_float2(v0.x, v0.y);
                        x[4 * u + 1] = make_float2(v0.z, v0.w);
                        x[4 * u + 2] = make_float2(v1.x, v1.y);
                        x[4 * u + 3] = make_float2(v1.z, v1.w);
                    }
                }
            }
        };
        // four amplitudes (consecutive block indices) -> one 16-byte hi and lo chunk
        auto chunk = [&](const float2 *x4, unsigned char *Sh, unsigned char *Sl, uint32_t o) {
            float hi[8], lo[8];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float xs[2] = {x4[q].x, x4[q].y};
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const float h = __bfloat162float(__float2bfloat16_rn(xs[b]));
                    hi[2 * q + b] = h;
                    lo[2 * q + b] = xs[b] - h;
                }
            }
            store_bf16x8(Sh + o, hi);
            store_bf16x8(Sl + o, lo);
        };
        auto convert = [&](const float2 (&x)[16], unsigned char *Sh, unsigned char *Sl) {
            if constexpr (!STATE_N) {
                if (!active) return;
#pragma unroll
                for (int c = 0; c < 4; ++c) chunk(x + 4 * c, Sh, Sl, sw128_off(n_m, 2 * (16 * cg_m + 4 * c)));
            } else {
#pragma unroll
                for (int u = 0; u < NROWS / 32; ++u)
                    chunk(x + 4 * u, Sh, Sl, sw128_off(conv_n | (u << 5), 8 * conv_c));
            }
        };
        auto tmem_ld16 = [&](uint32_t taddr, uint32_t (&r)[16]) {
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        };
        auto drain = [&](uint32_t acc_col, float2 *p) {
            const uint32_t lane_base =
                tmem + ((32u * (uint32_t)(warp & 3)) << 16) + acc_col + 32u * (uint32_t)(warp >> 2);
            float2 *q[16];
            q[0] = p + (STATE_N ? drow : lrow);
#pragma unroll
            for (int k = 1; k < 16; ++k)
                q[k] = q[k & (k - 1)] + (STATE_N ? de : le)[(k & 1) ? 0 : (k & 2) ? 1 : (k & 4) ? 2 : 3];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint32_t r[16];
                tmem_ld16(lane_base + 16u * h, r);
                if constexpr (!STATE_N) {
                    // row n: 8 amplitudes (re, im adjacent columns)
                    if (active) {
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            *q[8 * h + k] = make_float2(__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1]));
                    }
                } else {
                    // one of re/im of block index i' for 16 columns n; after
                    // the swap, lane (re) stores even n, lane (im) odd n
                    const uint32_t comp = lane & 1;
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const float keep = __uint_as_float(comp ? r[2 * j + 1] : r[2 * j]);
                        const float send = __uint_as_float(comp ? r[2 * j] : r[2 * j + 1]);
                        const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
                        if (32 * (warp >> 2) + 16 * h + 2 * j < NROWS)
                            *q[8 * h + j] = comp ? make_float2(recv, keep) : make_float2(keep, recv);
                    }
                }
            }
        };
        auto wait_warp = [&](uint64_t *bb, uint32_t parity) -> uint32_t {
            uint32_t dn = 0;
            if (lane == 0) dn = tc_wait(bb, parity);
            return __shfl_sync(0xffffffffu, dn, 0);
        };
        auto arrive = [&](uint64_t *bb) {
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s_u32(bb)) : "memory");
        };

        // per supertile: convert x (supertile o) into buffer it % 2 and hand
        // it to the issuer, refill x with supertile o + grid, then drain the
        // contraction of supertile it - 1
        uint32_t it = 0;
        bool bad = false;
        float2 x[16];
        uint64_t o = o_lo, base = 0, prev = 0;
        if (o < o_hi) {
            base = pass_base(o, d);
            load(x, s + base);
        }
        for (; o < o_hi; ++o, ++it) {
            if (__shfl_sync(0xffffffffu, bad_s, 0)) {
                bad = true;
                break;
            }
            const uint32_t b = it & 1;
            unsigned char *Sh = S0 + 2 * b * kTcOpBytes, *Sl = Sh + kTcOpBytes;
            // buffer b was released by this warp's wait for contraction it - 2
            convert(x, Sh, Sl);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            arrive(&full[b]);
            const uint64_t cur = base;
            if (o + 1 < o_hi) {
                base = pass_base(o + 1, d);
                load(x, s + base);
            }
            if (it > 0) {
                const uint32_t pb = b ^ 1u;
                if (!wait_warp(&mma[pb], ((it - 1) >> 1) & 1u)) {
                    if (lane == 0) bad_s = 1;
                    bad = true;
                    break;
                }
                tc_fence_after();
                drain(pb * 128u, s + prev);
                tc_fence_before();
                arrive(&empty[pb]);
            }
            prev = cur;
        }
        if (!bad && it > 0) {
            const uint32_t pb = (it - 1) & 1u;
            if (wait_warp(&mma[pb], ((it - 1) >> 1) & 1u)) {
                tc_fence_after();
                drain(pb * 128u, s + prev);
            } else if (lane == 0) {
                bad_s = 1;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (bad_s && tid == 0) atomicCAS(err, 0, 1);   // keeps a more specific code (3) set above
    if (issuer) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols) : "memory");
}

// ---- host side ----------------------------------------------------------------

template <int NROWS, bool STATE_N>
static int launch_dense_tc_n(float2 *state, int n, const DenseDesc &dd, const uint16_t *dW, int *derr,
                             cudaStream_t st) {
    static std::atomic<uint64_t> smem_done{0};
    const cudaError_t ea = smem_limit_once(smem_done, (const void *)k_dense_tc<NROWS, STATE_N>, (int)kTcSmem);
    if (ea != cudaSuccess) return fail(QK_ERR_CUDA, "cudaFuncSetAttribute(k_dense_tc): %s", cudaGetErrorString(ea));
    const int sms = device_sms();
    const uint64_t nsup = 1ull << (n - dd.p.T);
    const unsigned grid = (unsigned)std::min<uint64_t>(nsup, (uint64_t)sms);
    k_dense_tc<NROWS, STATE_N><<<grid, kTcThreads, kTcSmem, st>>>(state, nsup, dd, dW, derr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : fail(QK_ERR_CUDA, "k_dense_tc launch: %s", cudaGetErrorString(e));
}

int launch_dense_tc(float2 *state, int n, const DenseDesc &dd, const uint16_t *dW, int *derr, cudaStream_t st) {
    if (n < kTcMinTileBits || dd.p.T < kTcMinTileBits || dd.p.T > kTcMaxTileBits || dd.p.T > n || dd.p.L < 1)
        return fail(QK_ERR_ARG, "tensor-core blocks need >= %d qubits", kTcMinTileBits);
    // a block on qubit 0 has its block index along the contiguous direction
    const bool state_n = (dd.blockmask & 1u) != 0;
    if (dd.p.T == 12)
        return state_n ? launch_dense_tc_n<64, true>(state, n, dd, dW, derr, st)
                       : launch_dense_tc_n<64, false>(state, n, dd, dW, derr, st);
    return state_n ? launch_dense_tc_n<128, true>(state, n, dd, dW, derr, st)
                   : launch_dense_tc_n<128, false>(state, n, dd, dW, derr, st);
}

// from qk_pass.cu: one VSWAP as a permutation pass
int apply_perm_gate(void *state, int n, int dtype, const Op &op, cudaStream_t st);

int launch_dense_i8(double2 *state, int n, const DenseDesc &dd, const uint32_t *dW, int *derr, cudaStream_t st);

size_t dense_operand_bytes(int dtype) { return dtype == QK_C128 ? kI8OperandBytes : 2 * (size_t)kTcOpBytes; }

int run_dense_blocks(void *state, int n, int dtype, const std::vector<DenseBlock> &blocks, const void *dA, int *derr,
                     cudaStream_t st) {
    const unsigned char *ops = static_cast<const unsigned char *>(dA);
    const size_t step = dense_operand_bytes(dtype);
    for (size_t k = 0; k < blocks.size(); ++k) {
        const DenseBlock &b = blocks[k];
        int rc;
        if (b.perm)
            rc = apply_perm_gate(state, n, dtype, b.perm_op, st);
        else if (dtype == QK_C128)
            rc = launch_dense_i8((double2 *)state, n, dense_block_desc(b, n, kI8TileBits),
                                 reinterpret_cast<const uint32_t *>(ops + k * step), derr, st);
        else
            rc = launch_dense_tc((float2 *)state, n, dense_block_desc(b, n, kTcMaxTileBits),
                                 reinterpret_cast<const uint16_t *>(ops + k * step), derr, st);
        if (rc) return rc;
    }
    return QK_OK;
}

}  // namespace qk
