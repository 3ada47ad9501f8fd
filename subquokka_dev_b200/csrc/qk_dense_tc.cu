// Dense fused blocks on the 5th-generation tensor cores (complex64 states).
//
// A block is a 64 x 64 complex unitary U on six qubits (the product of
// consecutive gates, built on the host in FP64).  A pass applies one block to
// the whole state.  Each CTA owns one SM, loads the block's operand A once,
// and streams 4096-amplitude tiles (the block's six qubits plus six more
// tile bits, the lowest state bits first for coalescing):
//
//   tile as X[i][n]: i = block-qubit index (64), n = other tile bits (64)
//   real embedding, rows/cols interleaved (2i + re/im):
//     A[2i'+a][2i+b] = [[Ur, -Ui], [Ui, Ur]][a][b](i', i)      (128 x 128)
//     D[m][n] = sum_k A[m][k] B[n][k],  B[n][2i+b] = (re, im)_b X[i][n]
//   split precision (3 x BF16, FP32 accumulate in TMEM):
//     A = Ah + Al, B = Bh + Bl,  D = Ah Bh + Ah Bl + Al Bh   (K = 3 x 128)
//
// 24 tcgen05.mma (M128 N64 K16, kind::f16 with BF16 operands) per tile, issued
// by one thread, completion through tcgen05.commit -> mbarrier.  Operands sit
// in shared memory in the canonical K-major no-swizzle layout: 8-row x 16-byte
// core matrices, LBO = 128 B between K chunks, SBO = 2048 B between row
// groups.  The next tile is prefetched with cp.async during the contraction.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "qk_internal.h"
#include "qk_pass_device.cuh"

namespace qk {

constexpr int kTcThreads = 256;
constexpr int kTcTileBits = 12;
constexpr uint32_t kTcTile = 1u << kTcTileBits;       // amplitudes per tile
constexpr uint32_t kTcOpBytes = 128 * 128 * 2;        // one 128 x 128 bf16 operand
constexpr uint32_t kTcBBytes = 64 * 128 * 2;          // one 64 x 128 bf16 operand
constexpr uint32_t kTcTmemCols = 64;
constexpr uint32_t kTcSmem = 2 * kTcTile * 8 + 2 * kTcOpBytes + 2 * kTcBBytes + 256;
constexpr long long kTcWaitLimit = 20000000;          // mbarrier polls before giving up

struct DenseDesc {
    PassDesc p;         // tile bits (T = 12), L
    uint32_t blockmask; // tile-local bits that are the block's qubits
};

// byte offset of element (row r, k) of a K-major bf16 operand with 128 K columns
__host__ __device__ __forceinline__ uint32_t kmajor_off(uint32_t r, uint32_t k) {
    return (r >> 3) * 2048u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t s_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory position of tile element j: the 16-byte pair (j, j ^ 1) stays
// together (cp.async granule); the pair index is XORed with a fold of the
// higher index bits so that strided block-qubit accesses spread over banks.
__device__ __forceinline__ uint32_t tcz(uint32_t j) { return j ^ ((((j >> 4) ^ (j >> 7) ^ (j >> 10)) & 7u) << 1); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;   // leading byte offset: next K chunk
    d |= (uint64_t)((2048u >> 4) & 0x3FFFu) << 32;  // stride byte offset: next 8-row group
    d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
    return d;                                       // base offset 0, no swizzle
}

// kind::f16, A = B = BF16, D = F32, both K-major, M = 128, N = 64
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

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

__global__ void __launch_bounds__(kTcThreads, 1) k_dense_tc(float2 *__restrict__ s, uint64_t ntiles,
                                                            const __grid_constant__ DenseDesc dd,
                                                            const uint16_t *__restrict__ gA, int *__restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const PassDesc &d = dd.p;
    float2 *buf0 = reinterpret_cast<float2 *>(sm);
    float2 *buf1 = buf0 + kTcTile;
    unsigned char *Ah = sm + 2 * kTcTile * 8;
    unsigned char *Al = Ah + kTcOpBytes;
    unsigned char *Bh = Al + kTcOpBytes;
    unsigned char *Bl = Bh + kTcBBytes;
    uint16_t *jb = reinterpret_cast<uint16_t *>(Bl + kTcBBytes);
    uint16_t *jo = jb + 64;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // operand A (hi, lo) for the whole kernel, index tables, barrier, TMEM
    for (uint32_t i = tid; i < 2 * kTcOpBytes / 16; i += kTcThreads)
        reinterpret_cast<uint4 *>(Ah)[i] = reinterpret_cast<const uint4 *>(gA)[i];
    if (tid < 64) jb[tid] = (uint16_t)deposit_bits(tid, dd.blockmask);
    else if (tid < 128) jo[tid - 64] = (uint16_t)deposit_bits(tid - 64, (kTcTile - 1) & ~dd.blockmask);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&bar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&tmem_slot)),
                     "r"(kTcTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    // tile addressing: thread handles amplitude pairs p = tid + 256 u (u < 8),
    // elements j = 2p, 2p + 1 (tile bit 0 is state bit 0: 16-byte runs)
    const uint64_t g_t = pass_off(2 * tid, d);
    uint64_t g_u[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) g_u[b] = pass_off(512u << b, d);
    auto goff = [&](int u) {
        uint64_t x = g_t;
#pragma unroll
        for (int b = 0; b < 3; ++b)
            if ((u >> b) & 1) x |= g_u[b];
        return x;
    };
    auto prefetch = [&](float2 *buf, uint64_t base) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t j = 2 * (tid + 256 * u);
            const uint32_t dst = s_u32(buf + tcz(j));
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(s + (base | goff(u))) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    uint32_t phase = 0;
    uint64_t o = blockIdx.x;
    if (o < ntiles) prefetch(buf0, pass_base(o, d));
    for (int it = 0; o < ntiles; o += gridDim.x, ++it) {
        float2 *tl = (it & 1) ? buf1 : buf0;
        float2 *nx = (it & 1) ? buf0 : buf1;
        const uint64_t base = pass_base(o, d);
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        if (o + gridDim.x < ntiles) prefetch(nx, pass_base(o + gridDim.x, d));

        // B operand: row n = tid / 4, K columns 2i + b for i in [16 (tid % 4), +16)
        {
            const uint32_t n = tid >> 2, i0 = (tid & 3) * 16;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float hi[8], lo[8];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float2 x = tl[tcz(jb[i0 + 4 * c + q] | jo[n])];
                    const float xs[2] = {x.x, x.y};
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const float h = __bfloat162float(__float2bfloat16_rn(xs[b]));
                        hi[2 * q + b] = h;
                        lo[2 * q + b] = xs[b] - h;
                    }
                }
                const uint32_t off = kmajor_off(n, 2 * i0 + 8 * c);
                store_bf16x8(Bh + off, hi);
                store_bf16x8(Bl + off, lo);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
#pragma unroll 1
            for (int sp = 0; sp < 3; ++sp) {
                const uint32_t a = s_u32(sp < 2 ? Ah : Al), b = s_u32(sp == 1 ? Bl : Bh);
#pragma unroll 1
                for (int kk = 0; kk < 8; ++kk) {
                    const uint64_t ad = umma_desc(a + kk * 256), bd = umma_desc(b + kk * 256);
                    const uint32_t acc = (sp | kk) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                        "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s_u32(&bar))
                         : "memory");
        }
        // bounded wait for the contraction
        uint32_t done = 0;
        for (long long t = 0; t < kTcWaitLimit && !done; ++t) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(s_u32(&bar)), "r"(phase)
                : "memory");
        }
        phase ^= 1u;
        if (__syncthreads_or(!done)) {
            if (tid == 0) atomicExch(err, 1);
            break;
        }
        tc_fence_after();
        // D rows m = 32 (warp % 4) + lane, columns 32 (warp / 4) .. + 32
        {
            uint32_t r[32];
            const uint32_t taddr = tmem + (((uint32_t)(warp & 3) * 32u) << 16) + 32u * (uint32_t)(warp >> 2);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                  "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
                  "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                  "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const uint32_t m = (uint32_t)(warp & 3) * 32u + lane, ip = m >> 1, comp = m & 1;
            const uint32_t n0 = 32u * (uint32_t)(warp >> 2);
#pragma unroll
            for (int q = 0; q < 32; ++q)
                reinterpret_cast<float *>(&tl[tcz(jb[ip] | jo[n0 + q])])[comp] = __uint_as_float(r[q]);
        }
        tc_fence_before();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const uint32_t j = 2 * (tid + 256 * u);
            *reinterpret_cast<float4 *>(s + (base | goff(u))) = *reinterpret_cast<const float4 *>(tl + tcz(j));
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTmemCols) : "memory");
}

// ---- host side ----------------------------------------------------------------

static uint16_t bf16_rn(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7FFFu + lsb;
    return (uint16_t)(u >> 16);
}
static float bf16_to_f(uint16_t h) {
    const uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// A = real embedding of U (rows/cols interleaved re/im), split into bf16 hi +
// lo, each in the canonical K-major layout: 2 x 32 KiB.
void dense_block_operand(const DenseBlock &b, std::vector<uint16_t> &out) {
    out.assign(2 * 128 * 128, 0);
    unsigned char *hi = reinterpret_cast<unsigned char *>(out.data());
    unsigned char *lo = hi + kTcOpBytes;
    for (int ip = 0; ip < 64; ++ip)
        for (int i = 0; i < 64; ++i) {
            const double ur = b.u[2 * (ip * 64 + i)], ui = b.u[2 * (ip * 64 + i) + 1];
            const double v[2][2] = {{ur, -ui}, {ui, ur}};
            for (int a = 0; a < 2; ++a)
                for (int c = 0; c < 2; ++c) {
                    const float x = (float)v[a][c];
                    const uint16_t h = bf16_rn(x);
                    const uint16_t l = bf16_rn((float)(v[a][c] - (double)bf16_to_f(h)));
                    const uint32_t off = kmajor_off(2 * ip + a, 2 * i + c);
                    std::memcpy(hi + off, &h, 2);
                    std::memcpy(lo + off, &l, 2);
                }
        }
}

// tile bits of a block: its six qubits plus the lowest other state bits
DenseDesc dense_block_desc(const DenseBlock &b, int n) {
    DenseDesc dd;
    std::memset(&dd, 0, sizeof dd);
    std::vector<char> in(n, 0);
    for (int k = 0; k < kDenseQubits; ++k) in[b.q[k]] = 1;
    int cnt = kDenseQubits;
    for (int q = 0; q < n && cnt < kTcTileBits; ++q)
        if (!in[q]) { in[q] = 1; ++cnt; }
    int t = 0;
    for (int q = 0; q < n; ++q)
        if (in[q]) {
            for (int k = 0; k < kDenseQubits; ++k)
                if (b.q[k] == q) dd.blockmask |= 1u << t;
            dd.p.bpos[t++] = q;
        }
    dd.p.T = t;
    while (dd.p.L < dd.p.T && dd.p.bpos[dd.p.L] == dd.p.L) ++dd.p.L;
    return dd;
}

int launch_dense_tc(float2 *state, int n, const DenseDesc &dd, const uint16_t *dA, int *derr, cudaStream_t st) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaFuncSetAttribute(k_dense_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
        if (e != cudaSuccess) return fail(QK_ERR_CUDA, "cudaFuncSetAttribute(k_dense_tc): %s", cudaGetErrorString(e));
    }
    if (n < kTcTileBits || dd.p.T != kTcTileBits || dd.p.L < 1)
        return fail(QK_ERR_ARG, "tensor-core blocks need >= %d qubits", kTcTileBits);
    const uint64_t ntiles = 1ull << (n - kTcTileBits);
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sms);
    k_dense_tc<<<grid, kTcThreads, kTcSmem, st>>>(state, ntiles, dd, dA, derr);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : fail(QK_ERR_CUDA, "k_dense_tc launch: %s", cudaGetErrorString(e));
}

// from qk_pass.cu: one VSWAP as a permutation pass
int apply_perm_gate(void *state, int n, int dtype, const Op &op, cudaStream_t st);

int run_dense_blocks(void *state, int n, const std::vector<DenseBlock> &blocks, const uint16_t *dA, int *derr,
                     cudaStream_t st) {
    for (size_t k = 0; k < blocks.size(); ++k) {
        const DenseBlock &b = blocks[k];
        int rc = b.perm ? apply_perm_gate(state, n, QK_C64, b.perm_op, st)
                        : launch_dense_tc((float2 *)state, n, dense_block_desc(b, n), dA + k * 2 * 128 * 128, derr, st);
        if (rc) return rc;
    }
    return QK_OK;
}

}  // namespace qk
