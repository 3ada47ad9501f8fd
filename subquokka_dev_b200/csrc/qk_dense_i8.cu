// Dense fused blocks on the 5th-generation tensor cores, complex128 states.
//
// The block is the same 64 x 64 complex unitary U on six qubits as in the
// complex64 kernel (qk_dense_tc.cu), applied to supertiles of 64 x 64
// amplitudes (the block's six qubits x the lowest six other state bits) as
// the real contraction
//
//   D[m][n] = sum_k W[m][k] S[n][k]          m, k < 128, n < 64
//   W[2i'+a][2i+c] = [[Ur, -Ui], [Ui, Ur]][a][c] (i', i)
//   S[n][2i+c]     = (re, im)_c X[i][n],     X'[i'][n] = D[2i'][n] + i D[2i'+1][n]
//
// in exact integer arithmetic on the int8 tensor cores (tcgen05.mma
// kind::i8, int32 accumulators), an Ozaki-type split:
//
//   - every row of W and every row n of S is scaled by a power of two to a
//     55-bit integer v = round(x 2^(1076 - e)) (e = the row's largest biased
//     exponent, |v| < 2^54) and cut into seven 8-bit digits: W rows on the
//     host as balanced digits in [-128, 127]; state rows on the device as
//     the seven low bytes of v in two's complement (six unsigned digits and
//     a signed top digit in [-64, 63]);
//   - sum_k v_w v_s = sum_(i, j) 2^(8 (i + j)) sum_k w_i s_j.  The 28 digit
//     products with i + j >= 6 are computed; the dropped ones lie below
//     2^-48 of the largest result of the row.  Products of one weight
//     d = i + j add up in one int32 accumulator (|sum| <= 7 x 128 x 128 x 255
//     < 2^25);
//   - the seven accumulators of a supertile are combined in FP64 and scaled
//     back by 2^(e_w - 1028) 2^(e_s - 1028).  State rows whose largest entry
//     is below 2^-959 come out as zero.
//
// Operands and memory:
//   - W's digit planes are the A operand in shared memory (M = 128 rows m,
//     K-major, 128-byte swizzle: 16 KiB a plane), copied once per CTA.
//   - The state's digit planes are the B operand in shared memory (N = 64
//     rows n, 8 KiB a plane), two supertiles' worth.
//   - Accumulators D[m][n]: eight slots of 64 TMEM columns, a ring over the
//     seven weights of consecutive supertiles, so that the MMAs of a whole
//     supertile can be issued while the one before is drained.
//
// Roles (16 data warps + 1 issuer warp): per supertile the data warps split
// the amplitudes they loaded into digit planes (thread = row n, block
// indices 8 g .. 8 g + 7), hand them to the issuer, load the next supertile,
// then drain the seven accumulators of the previous one (thread = TMEM lane
// m, 16 columns n), combine them in FP64 and store it.  One elected thread
// issues the 28 x 4 MMAs (M128 N64 K32) of a supertile and commits each
// weight's accumulator to an mbarrier.  Every wait is bounded: a wait that
// runs out sets an error code (1) and the warp stops; the issuer releases the
// TMEM only after its last MMAs have completed (3 if that wait runs out).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "qk_device.h"
#include "qk_internal.h"
#include "qk_pass_device.cuh"
#include "qk_operand.h"
#include "qk_tc_device.cuh"

namespace qk {

constexpr int kI8DataWarps = 16;
constexpr int kI8DataThreads = 32 * kI8DataWarps;
constexpr int kI8Threads = kI8DataThreads + 32;             // + one MMA-issuer warp
constexpr uint32_t kI8WPlaneBytes = 128u * 128u;            // one digit plane of W
constexpr uint32_t kI8PlaneBytes = 64u * 128u;              // one digit plane of the state operand
constexpr uint32_t kI8WBytes = kI8Digits * kI8WPlaneBytes;  // 112 KiB
constexpr uint32_t kI8BufBytes = kI8Digits * kI8PlaneBytes; // the seven planes of one supertile
constexpr uint32_t kI8Smem = kI8WBytes + 2u * kI8BufBytes;  // 224 KiB
constexpr int kI8Slots = 8;                                 // accumulators of 64 columns
constexpr int kI8LowWeight = 6;                             // digit products of weight i + j >= this
constexpr int kI8Weights = 2 * (kI8Digits - 1) + 1 - kI8LowWeight;
constexpr uint32_t kI8TmemCols = 64u * kI8Slots;
static_assert(kI8TmemCols <= 512, "accumulators exceed the tensor memory");
static_assert(kI8WBytes == kI8OperandWords * 4, "operand layout");

// kind::i8, D = S32, A = W digits (signed), B = state digits (unsigned for
// planes 0-5, signed for the top plane), both K-major, M = 128, N = 64
constexpr uint32_t kI8IdescU = (2u << 4) | (1u << 7) | (0u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kI8IdescS = kI8IdescU | (1u << 10);

// 4 x 4 byte transpose: out[j] = byte j of in[0], in[1], in[2], in[3]
__device__ __forceinline__ void bytes4x4(const uint32_t (&in)[4], uint32_t (&out)[4]) {
    const uint32_t t0 = __byte_perm(in[0], in[1], 0x5140), t1 = __byte_perm(in[0], in[1], 0x7362);
    const uint32_t t2 = __byte_perm(in[2], in[3], 0x5140), t3 = __byte_perm(in[2], in[3], 0x7362);
    out[0] = __byte_perm(t0, t2, 0x5410);
    out[1] = __byte_perm(t0, t2, 0x7632);
    out[2] = __byte_perm(t1, t3, 0x5410);
    out[3] = __byte_perm(t1, t3, 0x7632);
}

// round(x 2^(1076 - es)) as two's-complement words (lo, hi), es being the
// largest biased exponent of x's row, with `scale` = 2^(1044 - es): y = x
// scale (|y| < 2^22) splits exactly into rint(y) and r = y - rint(y)
// (|r| <= 1/2), and rint(y) 2^32 + rint(r 2^32) = round(x 2^(1076 - es)).
// Each integer is read off the low mantissa bits of 1.5 2^52 + value; bits
// 32.. of the second one's mantissa say whether rint(r 2^32) was negative.
__device__ __forceinline__ void to_fixed(double x, double scale, uint32_t &lo, uint32_t &hi) {
    const double magic = 6755399441055744.0;   // 1.5 2^52
    const double t1 = fma(x, scale, magic);
    const double yh = t1 - magic;
    const double r = fma(x, scale, -yh);
    const double t2 = fma(r, 4294967296.0, magic);
    lo = (uint32_t)__double2loint(t2);
    hi = (uint32_t)__double2loint(t1) + ((uint32_t)__double2hiint(t2) & 0xFFFFFu) - 0x80000u;
}

__global__ void __launch_bounds__(kI8Threads, 1)
    k_dense_i8(double2 *__restrict__ s, uint64_t nsup, const __grid_constant__ DenseDesc dd,
               const uint32_t *__restrict__ gW, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    // full[b]: the digit planes of buffer b written (one arrival per data
    // warp); accf[r]: the MMAs of accumulator slot r done (tcgen05.commit);
    // empty[r]: slot r drained (one arrival per data warp); fin: every MMA
    // the issuer issued has completed
    __shared__ __align__(8) uint64_t full[2], accf[kI8Slots], empty[kI8Slots], fin;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int bad_s;
    // row exponents e_s of supertile it at es_s[it % 4] (0: a flushed row;
    // the drain scales by 2^(e_s - 1028)).  A warp
    // writes those of supertile it + 4 after its drain of supertile it + 2,
    // whose last MMAs were issued only once every warp had drained weight 5
    // of supertile it + 1, so every warp has stored supertile it by then.
    // (With three buffers a warp could overwrite them while another still
    // stores supertile it: its drain of it + 1 waits only for weight 5 of it.)
    __shared__ __align__(8) int es_s[4][64];
    const PassDesc &d = dd.p;
    unsigned char *sW = sm, *sB = sm + kI8WBytes;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool issuer = warp == kI8DataWarps;
    if (s_u32(sm) & 1023u) {   // the swizzle pattern needs 1024-byte aligned operands
        if (tid == 0) atomicExch(err, 2);
        return;
    }
    if (tid == 0) {
        bad_s = 0;
        for (int b = 0; b < 2; ++b) mbar_init(&full[b], kI8DataWarps);
        for (int r = 0; r < kI8Slots; ++r) {
            mbar_init(&accf[r], 1);
            mbar_init(&empty[r], kI8DataWarps);
        }
        mbar_init(&fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (issuer) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&tmem_slot)),
                     "r"(kI8TmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // W's digit planes (already in the swizzled operand layout) into shared memory
    for (uint32_t i = tid; i < kI8WBytes / 16; i += kI8Threads)
        reinterpret_cast<uint4 *>(sW)[i] = reinterpret_cast<const uint4 *>(gW)[i];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");

    // data threads.  Split: row n = tid / 8, block indices 8 g .. 8 g + 7, at
    // lrow + sum of 2^lbp[b] over the bits b of the index's low three bits.
    // Drain: TMEM lane m = 32 q4 + lane (output i' = m / 2, re/im = m & 1),
    // columns n = 16 cgrp .. + 15; the lane stores n = 16 cgrp + 2 j + (m & 1)
    // at obase + sum of 2^onp[b] over the bits of j.  (lbp, onp: the state
    // bits of single tile bits, packed a byte each.)
    const uint32_t tmask = (1u << d.T) - 1, nmask = tmask & ~dd.blockmask;
    const int q4 = warp & 3, cgrp = warp >> 2;
    const uint32_t g = tid & 7, nrow = (uint32_t)tid >> 3;
    double sw = 0.0;   // W row scale of lane m
    uint64_t lrow = 0, obase = 0;
    uint32_t lbp = 0, onp = 0;
    auto bitoff = [](uint32_t packed, int b) { return 1ull << ((packed >> (8 * b)) & 63u); };
    if (!issuer) {
        const uint32_t m = 32u * q4 + lane;
        auto jn = [&](uint32_t v) { return pass_off(deposit_bits(v, nmask), d); };
        auto jb = [&](uint32_t v) { return pass_off(deposit_bits(v, dd.blockmask), d); };
        lrow = jn(nrow) + jb(8 * g);
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            lbp |= (uint32_t)(__ffsll((long long)jb(1u << b)) - 1) << (8 * b);
            onp |= (uint32_t)(__ffsll((long long)jn(2u << b)) - 1) << (8 * b);
        }
        obase = jb(m >> 1) + jn(16u * cgrp + (m & 1u));
        sw = reinterpret_cast<const double *>(gW + kI8OperandWords)[m];
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    // each CTA takes a contiguous range of supertiles
    const uint64_t o_lo = nsup * blockIdx.x / gridDim.x, o_hi = nsup * (blockIdx.x + 1) / gridDim.x;

    if (issuer) {
        if (lane == 0) {
            uint32_t it = 0;
            bool stop = false;
            const uint32_t wbase = s_u32(sW);
            for (uint64_t o = o_lo; o < o_hi && !stop && !bad_s; ++o, ++it) {
                const uint32_t b = it & 1u;
                if (!tc_wait(&full[b], (it >> 1) & 1u)) {
                    stop = true;
                    break;
                }
                tc_fence_after();
                const uint32_t planes = s_u32(sB + b * kI8BufBytes);
#pragma unroll 1
                for (int e = 0; e < kI8Weights; ++e) {   // weight wd: products (i, wd - i)
                    const int wd = kI8LowWeight + e, i0 = max(0, wd - (kI8Digits - 1));
                    const uint32_t gg = (uint32_t)kI8Weights * it + (uint32_t)e, slot = gg % kI8Slots;
                    if (gg >= (uint32_t)kI8Slots && !tc_wait(&empty[slot], ((gg / kI8Slots) - 1) & 1u)) {
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t acc = tmem + 64u * slot;
#pragma unroll 1
                    for (int i = i0; i <= min(kI8Digits - 1, wd); ++i) {
                        const int j = wd - i;
                        const uint32_t idesc = j == kI8Digits - 1 ? kI8IdescS : kI8IdescU;
                        const uint32_t aplane = wbase + (uint32_t)i * kI8WPlaneBytes;
                        const uint32_t bplane = planes + (uint32_t)j * kI8PlaneBytes;
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            const uint32_t en = (i != i0 || kk) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                    acc),
                                "l"(sw128_desc(aplane + 32u * kk)), "l"(sw128_desc(bplane + 32u * kk)), "r"(idesc),
                                "r"(en), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                                : "memory");
                        }
                    }
                    tc_commit(&accf[slot]);
                }
            }
            if (stop) bad_s = 1;
            // Teardown invariant: the TMEM is released only after every MMA
            // issued above has completed (one more commit tracks them all).
            tc_commit(&fin);
            if (!tc_wait(&fin, 0)) {
                bad_s = 1;
                atomicExch(err, 3);
            }
        }
        __syncwarp();
    } else {
        // the eight amplitudes of (row nrow, block indices 8 g ..) of supertile o
        auto load = [&](double2 (&x)[8], uint64_t o) {
            const double2 *p = s + pass_base(o, d) + lrow;
            if ((lbp & 63u) == 0) {   // block index bit 0 is state bit 0: pairs are 32-byte runs
#pragma unroll
                for (int a = 0; a < 8; a += 2) {
                    const double *q =
                        reinterpret_cast<const double *>(p + ((a & 2) ? bitoff(lbp, 1) : 0) + ((a & 4) ? bitoff(lbp, 2) : 0));
                    double r0, r1, r2, r3;
                    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                                 : "=d"(r0), "=d"(r1), "=d"(r2), "=d"(r3)
                                 : "l"(q));
                    x[a] = make_double2(r0, r1);
                    x[a + 1] = make_double2(r2, r3);
                }
            } else {
#pragma unroll
                for (int a = 0; a < 8; ++a)
                    x[a] = p[((a & 1) ? bitoff(lbp, 0) : 0) + ((a & 2) ? bitoff(lbp, 1) : 0) +
                             ((a & 4) ? bitoff(lbp, 2) : 0)];
            }
        };
        // registers -> seven digit planes (row nrow, K chunk g) and the row's scale
        auto split = [&](const double2 (&x)[8], unsigned char *planes, int *es_row) {
            uint32_t ek = 0;
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                ek = max(ek, (uint32_t)__double2hiint(x[a].x) & 0x7FF00000u);
                ek = max(ek, (uint32_t)__double2hiint(x[a].y) & 0x7FF00000u);
            }
            ek = max(ek, __shfl_xor_sync(0xffffffffu, ek, 1));
            ek = max(ek, __shfl_xor_sync(0xffffffffu, ek, 2));
            ek = max(ek, __shfl_xor_sync(0xffffffffu, ek, 4));
            const int es = (int)(ek >> 20);
            // rows below 2^-959 are flushed to zero (their scale 2^(1044 - es)
            // would not be a finite double)
            const bool live = es >= 64;
            const double scale = live ? __hiloint2double((2067 - es) << 20, 0) : 0.0;
            if (g == 0) es_row[nrow] = live ? es : 0;
            uint32_t lo[16], hi[16];
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                to_fixed(x[a].x, scale, lo[2 * a], hi[2 * a]);
                to_fixed(x[a].y, scale, lo[2 * a + 1], hi[2 * a + 1]);
            }
            uint32_t pl[kI8Digits][4];
#pragma unroll
            for (int qd = 0; qd < 4; ++qd) {
                uint32_t t[4];
                const uint32_t inl[4] = {lo[4 * qd], lo[4 * qd + 1], lo[4 * qd + 2], lo[4 * qd + 3]};
                bytes4x4(inl, t);
#pragma unroll
                for (int j = 0; j < 4; ++j) pl[j][qd] = t[j];
                const uint32_t inh[4] = {hi[4 * qd], hi[4 * qd + 1], hi[4 * qd + 2], hi[4 * qd + 3]};
                bytes4x4(inh, t);
#pragma unroll
                for (int j = 4; j < kI8Digits; ++j) pl[j][qd] = t[j - 4];
            }
            const uint32_t off = nrow * 128u + ((g ^ (nrow & 7u)) << 4);
#pragma unroll
            for (int j = 0; j < kI8Digits; ++j)
                *reinterpret_cast<uint4 *>(planes + (uint32_t)j * kI8PlaneBytes + off) =
                    make_uint4(pl[j][0], pl[j][1], pl[j][2], pl[j][3]);
        };
        auto wait_warp = [&](uint64_t *bb, uint32_t parity) -> uint32_t {
            uint32_t dn = 0;
            if (lane == 0) dn = tc_wait(bb, parity);
            return __shfl_sync(0xffffffffu, dn, 0);
        };
        auto arrive = [&](uint64_t *bb) {
            __syncwarp();
            if (lane == 0) mbar_arrive(bb);
        };
        // int32 accumulator a -> acc += a sc, exactly on the FP64 pipe:
        // 2^52 + (a + 2^31) has a + 2^31 as its low mantissa bits
        auto accumulate = [&](double (&acc)[16], const uint32_t (&r)[16], double sc) {
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const double a = __hiloint2double(0x43300000, (int)(r[c] ^ 0x80000000u)) - 4503601774854144.0;
                acc[c] = fma(a, sc, acc[c]);
            }
        };
        auto tmem_ld16 = [&](uint32_t taddr, uint32_t (&r)[16]) {
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                "%12, %13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
        };
        // the seven accumulators of supertile it (at o), combined and stored;
        // false if a wait ran out.  A commit covers every earlier MMA, so the
        // warp waits for every second weight and reads two.
        auto drain = [&](uint32_t it, uint64_t o) -> bool {
            double acc[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) acc[c] = 0.0;
            const uint32_t lanecol = tmem + ((32u * q4) << 16) + 16u * cgrp;
#pragma unroll 1
            for (int e = 0; e < kI8Weights; e += 2) {
                const int e1 = min(e + 1, kI8Weights - 1);
                const uint32_t g0 = (uint32_t)kI8Weights * it + (uint32_t)e, g1 = g0 + (uint32_t)(e1 - e);
                if (!wait_warp(&accf[g1 % kI8Slots], (g1 / kI8Slots) & 1u)) return false;
                tc_fence_after();
                // weight 2^(8 (d - 12)) times the W row scale, least significant first
                double sc = sw * __hiloint2double((1023 - 96 + 8 * (kI8LowWeight + e)) << 20, 0);
                for (uint32_t gk = g0; gk <= g1; ++gk, sc *= 256.0) {
                    uint32_t r[16];
                    tmem_ld16(lanecol + 64u * (gk % kI8Slots), r);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    tc_fence_before();
                    arrive(&empty[gk % kI8Slots]);
                    accumulate(acc, r, sc);
                }
            }
            // scale by the column and store: lane pairs (re, im) of i' exchange halves
            const int *es_row = es_s[it % 4];
            const uint32_t comp = lane & 1u;
            double2 *out = s + pass_base(o, d) + obase;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int2 e2 = *reinterpret_cast<const int2 *>(es_row + 16 * cgrp + 2 * j);
                const double s0 = e2.x ? __hiloint2double((e2.x - 5) << 20, 0) : 0.0;
                const double s1 = e2.y ? __hiloint2double((e2.y - 5) << 20, 0) : 0.0;
                const double v0 = acc[2 * j] * s0, v1 = acc[2 * j + 1] * s1;
                const double keep = comp ? v1 : v0, send = comp ? v0 : v1;
                const double recv = __shfl_xor_sync(0xffffffffu, send, 1);
                const uint64_t oj =
                    ((j & 1) ? bitoff(onp, 0) : 0) + ((j & 2) ? bitoff(onp, 1) : 0) + ((j & 4) ? bitoff(onp, 2) : 0);
                out[oj] = comp ? make_double2(recv, keep) : make_double2(keep, recv);
            }
            return true;
        };

        // per supertile: split the registers (supertile o) into plane buffer
        // it % 2 and hand it to the issuer, load supertile o + 1 into the
        // registers, then drain and store supertile o - 1 while the MMAs of
        // o run.  Buffer it % 2 was last read by the MMAs of supertile it - 2,
        // whose completion this warp saw while draining it.
        uint32_t it = 0;
        bool bad = false;
        double2 x[8];
        if (o_lo < o_hi) load(x, o_lo);
        for (uint64_t o = o_lo; o < o_hi; ++o, ++it) {
            if (__shfl_sync(0xffffffffu, bad_s, 0)) {
                bad = true;
                break;
            }
            split(x, sB + (it & 1u) * kI8BufBytes, es_s[it % 4]);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            arrive(&full[it & 1u]);
            if (o + 1 < o_hi) load(x, o + 1);
            if (it > 0 && !drain(it - 1, o - 1)) {
                bad = true;
                break;
            }
        }
        if (!bad && it > 0 && !drain(it - 1, o_hi - 1)) bad = true;
        if (bad && lane == 0) bad_s = 1;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (bad_s && tid == 0) atomicCAS(err, 0, 1);   // keeps a more specific code (3) set above
    if (issuer)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kI8TmemCols) : "memory");
}

// ---- host side ----------------------------------------------------------------

int launch_dense_i8(double2 *state, int n, const DenseDesc &dd, const uint32_t *dW, int *derr, cudaStream_t st) {
    if (n < kI8TileBits || dd.p.T != kI8TileBits || dd.p.L < 1 || __builtin_popcount(dd.blockmask) != kDenseQubits)
        return fail(QK_ERR_ARG, "complex128 tensor-core blocks need >= %d qubits", kI8TileBits);
    static std::atomic<uint64_t> smem_done{0};
    const cudaError_t ea = smem_limit_once(smem_done, (const void *)k_dense_i8, (int)kI8Smem);
    if (ea != cudaSuccess) return fail(QK_ERR_CUDA, "cudaFuncSetAttribute(k_dense_i8): %s", cudaGetErrorString(ea));
    const uint64_t nsup = 1ull << (n - kI8TileBits);
    const unsigned grid = (unsigned)std::min<uint64_t>(nsup, (uint64_t)device_sms());
    k_dense_i8<<<grid, kI8Threads, kI8Smem, st>>>(state, nsup, dd, dW, derr);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : fail(QK_ERR_CUDA, "k_dense_i8 launch: %s", cudaGetErrorString(e));
}

}  // namespace qk
