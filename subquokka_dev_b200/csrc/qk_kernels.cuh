// Device code of the state-vector engine (sm_100a).
//
// The state is an array of 2^n interleaved complex amplitudes (double2 for
// complex128, float2 for complex64); qubit q is bit q of the index
// (src/MEM_Runner.cpp:79-99).  Each per-gate kernel is one HBM sweep that
// touches only the amplitudes the gate changes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "qk_internal.h"

namespace qk {

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

template <typename C> __host__ __device__ __forceinline__ C mk(double re, double im) {
    C r;
    r.x = (decltype(r.x))re;
    r.y = (decltype(r.y))im;
    return r;
}

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// a*b + c*d, as four fused multiply-adds per component
template <typename C> __device__ __forceinline__ C cmul2(C a, C b, C c, C d) {
    C r;
    r.x = fma(a.x, b.x, fma(-a.y, b.y, fma(c.x, d.x, -c.y * d.y)));
    r.y = fma(a.x, b.y, fma(a.y, b.x, fma(c.x, d.y, c.y * d.x)));
    return r;
}

template <typename C> __device__ __forceinline__ C cadd(C a, C b) {
    C r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}

// Insert a zero bit at position t: the reference's bit_string for one target
// (src/MEM_Runner.cpp:90-99).
__device__ __forceinline__ uint64_t ins0(uint64_t p, int t) {
    const uint64_t lo = (1ull << t) - 1;
    return ((p & ~lo) << 1) | (p & lo);
}

template <typename C> struct Mat2 { C m[4]; };
template <typename C> struct Mat4 { C m[16]; };
template <typename C> struct Diag4 { C d[4]; };

constexpr int kBlock = 256;  // threads per block of the sweep kernels
constexpr int kUnroll = 4;   // independent items per thread (loads in flight)

__device__ __forceinline__ uint64_t item0() {
    return (uint64_t)blockIdx.x * (kBlock * kUnroll) + threadIdx.x;
}

// Dense 2x2 on a low qubit t < 5: both amplitudes of a pair live in lanes of
// the same warp, so every lane loads one amplitude of a fully coalesced
// 32-amplitude run and fetches its partner with a warp shuffle.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_dense1_lane(C *__restrict__ s, uint64_t namp, int t, Mat2<C> m) {
    const uint64_t e0 = item0();
    const int bit = (threadIdx.x >> t) & 1;
    const C ma = bit ? m.m[3] : m.m[0];  // coefficient of my own amplitude
    const C mb = bit ? m.m[2] : m.m[1];  // coefficient of my partner's
    C v[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t e = e0 + (uint64_t)u * kBlock;
        v[u] = e < namp ? s[e] : mk<C>(0, 0);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        C w;
        w.x = __shfl_xor_sync(0xffffffffu, v[u].x, 1 << t);
        w.y = __shfl_xor_sync(0xffffffffu, v[u].y, 1 << t);
        v[u] = cmul2(ma, v[u], mb, w);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t e = e0 + (uint64_t)u * kBlock;
        if (e < namp) s[e] = v[u];
    }
}

// Dense 2x2 on qubit t >= 5: pair p -> (i0, i0 + 2^t); both halves are runs of
// >= 32 contiguous amplitudes, so both loads of a warp are coalesced.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_dense1_pair(C *__restrict__ s, uint64_t npairs, int t, Mat2<C> m) {
    const uint64_t p0 = item0();
    const uint64_t h = 1ull << t;
    C a[kUnroll], b[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < npairs) {
            const uint64_t i = ins0(p, t);
            a[u] = s[i];
            b[u] = s[i + h];
        }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < npairs) {
            const uint64_t i = ins0(p, t);
            s[i] = cmul2(m.m[0], a[u], m.m[1], b[u]);
            s[i + h] = cmul2(m.m[2], a[u], m.m[3], b[u]);
        }
    }
}

// Amplitudes with bit t set *= ph (Z, P): half the state is touched.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_phase1(C *__restrict__ s, uint64_t npairs, int t, C ph) {
    const uint64_t p0 = item0();
    const uint64_t h = 1ull << t;
    C a[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < npairs) a[u] = s[ins0(p, t) | h];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < npairs) s[ins0(p, t) | h] = cmul(a[u], ph);
    }
}

// Amplitude *= d[bit t] (RZ): flat, fully coalesced sweep.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_diag1(C *__restrict__ s, uint64_t namp, int t, C d0, C d1) {
    const uint64_t e0 = item0();
    C a[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t e = e0 + (uint64_t)u * kBlock;
        if (e < namp) a[u] = s[e];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t e = e0 + (uint64_t)u * kBlock;
        if (e < namp) s[e] = cmul(a[u], ((e >> t) & 1) ? d1 : d0);
    }
}

// Dense 4x4 on qubits qa < qb (U2); matrix index bit 0 = qa, bit 1 = qb.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_dense2(C *__restrict__ s, uint64_t nquads, int qa, int qb, Mat4<C> m) {
    const uint64_t p0 = item0();
    const uint64_t A = 1ull << qa, B = 1ull << qb;
#pragma unroll 2
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p >= nquads) continue;
        const uint64_t i = ins0(ins0(p, qa), qb);
        const C x0 = s[i], x1 = s[i + A], x2 = s[i + B], x3 = s[i + A + B];
        C y[4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
            y[r] = cadd(cmul2(m.m[4 * r + 0], x0, m.m[4 * r + 1], x1), cmul2(m.m[4 * r + 2], x2, m.m[4 * r + 3], x3));
        s[i] = y[0];
        s[i + A] = y[1];
        s[i + B] = y[2];
        s[i + A + B] = y[3];
    }
}

// Amplitudes with bits qa and qb both set *= ph (CP): a quarter of the state.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_phase2(C *__restrict__ s, uint64_t nquads, int qa, int qb, C ph) {
    const uint64_t p0 = item0();
    const uint64_t AB = (1ull << qa) | (1ull << qb);
    C a[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < nquads) a[u] = s[ins0(ins0(p, qa), qb) | AB];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < nquads) s[ins0(ins0(p, qa), qb) | AB] = cmul(a[u], ph);
    }
}

// Amplitude *= d[bit qa + 2 bit qb] (RZZ): flat sweep.
template <typename C>
__global__ void __launch_bounds__(kBlock) k_diag2(C *__restrict__ s, uint64_t namp, int qa, int qb, Diag4<C> d) {
    const uint64_t e0 = item0();
    C a[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t e = e0 + (uint64_t)u * kBlock;
        if (e < namp) a[u] = s[e];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t e = e0 + (uint64_t)u * kBlock;
        if (e < namp) s[e] = cmul(a[u], d.d[((e >> qa) & 1) | (((e >> qb) & 1) << 1)]);
    }
}

// Exchange |..1..0..> and |..0..1..> of qubits qa < qb (SWAP): half the state.
// Controlled X: swap the amplitude pairs of target qt where control qc is
// set (a quarter of the amplitudes are read and written twice over: S bytes).
template <typename C>
__global__ void __launch_bounds__(kBlock) k_cx(C *__restrict__ s, uint64_t nquads, int qc, int qt) {
    const uint64_t p0 = item0();
    const int lo = qc < qt ? qc : qt, hi = qc < qt ? qt : qc;
    const uint64_t Cb = 1ull << qc, Tb = 1ull << qt;
    C a[kUnroll], b[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < nquads) {
            const uint64_t i = ins0(ins0(p, lo), hi) | Cb;
            a[u] = s[i];
            b[u] = s[i | Tb];
        }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < nquads) {
            const uint64_t i = ins0(ins0(p, lo), hi) | Cb;
            s[i] = b[u];
            s[i | Tb] = a[u];
        }
    }
}

template <typename C>
__global__ void __launch_bounds__(kBlock) k_swap2(C *__restrict__ s, uint64_t nquads, int qa, int qb) {
    const uint64_t p0 = item0();
    const uint64_t A = 1ull << qa, B = 1ull << qb;
    C a[kUnroll], b[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < nquads) {
            const uint64_t i = ins0(ins0(p, qa), qb);
            a[u] = s[i | A];
            b[u] = s[i | B];
        }
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
        const uint64_t p = p0 + (uint64_t)u * kBlock;
        if (p < nquads) {
            const uint64_t i = ins0(ins0(p, qa), qb);
            s[i | A] = b[u];
            s[i | B] = a[u];
        }
    }
}

// |0...0>
template <typename C> __global__ void k_zero_state(C *s, uint64_t namp) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < namp; e += (uint64_t)gridDim.x * blockDim.x)
        s[e] = mk<C>(e == 0 ? 1.0 : 0.0, 0.0);
}

// complex128 <-> complex64 conversion for uploads/downloads of c64 states.
__global__ void k_c128_to_c64(const double2 *in, float2 *out, uint64_t namp);
__global__ void k_c64_to_c128(const float2 *in, double2 *out, uint64_t namp);

}  // namespace qk
