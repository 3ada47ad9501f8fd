// Host-side builders of the tensor-core operands and supertile layouts
// (qk_dense_tc.cu: complex64 blocks; qk_dense_i8.cu: complex128 blocks).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "qk_internal.h"
#include "qk_operand.h"

namespace qk {

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

// W = real embedding of U (rows/cols interleaved re/im), split into bf16 hi +
// lo, each in the canonical K-major layout: 2 x 32 KiB.
void dense_block_operand(const DenseBlock &b, std::vector<uint16_t> &out) {
    out.assign(2 * 128 * 128, 0);
    unsigned char *hi = reinterpret_cast<unsigned char *>(out.data());
    unsigned char *lo = hi + kBf16OperandBytes;
    for (int ip = 0; ip < 64; ++ip)
        for (int i = 0; i < 64; ++i) {
            const double ur = b.u[2 * (ip * 64 + i)], ui = b.u[2 * (ip * 64 + i) + 1];
            const double v[2][2] = {{ur, -ui}, {ui, ur}};
            for (int a = 0; a < 2; ++a)
                for (int c = 0; c < 2; ++c) {
                    const float x = (float)v[a][c];
                    const uint16_t h = bf16_rn(x);
                    const uint16_t l = bf16_rn((float)(v[a][c] - (double)bf16_to_f(h)));
                    const uint32_t off = sw128_off(2 * ip + a, 2 * i + c);
                    std::memcpy(hi + off, &h, 2);
                    std::memcpy(lo + off, &l, 2);
                }
        }
}

// tile bits of a block: its six qubits plus the lowest other state bits, up
// to max_tile_bits (13: 64 x 128 supertiles)
DenseDesc dense_block_desc(const DenseBlock &b, int n, int max_tile_bits) {
    DenseDesc dd;
    std::memset(&dd, 0, sizeof dd);
    std::vector<char> in(n, 0);
    for (int k = 0; k < kDenseQubits; ++k) in[b.q[k]] = 1;
    const int tbits = std::min(n, max_tile_bits);
    int cnt = kDenseQubits;
    for (int q = 0; q < n && cnt < tbits; ++q)
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

static int biased_exponent(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return (int)((u >> 52) & 0x7FF);
}

// Digit planes of W = the real embedding of U: row m's entries scaled by
// 2^(1076 - e_m) (e_m its largest biased exponent), rounded to integers and
// written as seven balanced base-256 digits; plane i is the A operand image
// (digit k of row m at sw128_i8_off(i, m, k)), followed by the row scales
// 2^(e_m - 1028).
void dense_i8_operand(const DenseBlock &b, std::vector<uint32_t> &out) {
    out.assign(kI8OperandBytes / 4, 0);
    unsigned char *bytes = reinterpret_cast<unsigned char *>(out.data());
    double *scale = reinterpret_cast<double *>(out.data() + kI8OperandWords);
    for (int m = 0; m < 128; ++m) {
        const int ip = m >> 1, a = m & 1;
        double row[128];
        int em = 0;
        for (int k = 0; k < 128; ++k) {
            const int i = k >> 1, c = k & 1;
            const double ur = b.u[2 * (ip * 64 + i)], ui = b.u[2 * (ip * 64 + i) + 1];
            row[k] = a == 0 ? (c == 0 ? ur : -ui) : (c == 0 ? ui : ur);
            em = std::max(em, biased_exponent(row[k]));
        }
        scale[m] = em > 0 ? std::ldexp(1.0, em - 1028) : 0.0;
        if (em == 0) continue;
        for (int k = 0; k < 128; ++k) {
            long long v = std::llrint(std::ldexp(row[k], 1076 - em));
            for (int i = 0; i < kI8Digits; ++i) {
                int dg;
                if (i < kI8Digits - 1) {
                    dg = (int)((v + 128) & 255) - 128;
                    v = (v - dg) / 256;
                } else {
                    dg = (int)v;   // |v| <= 65 after six balanced digits of a 55-bit value
                }
                bytes[sw128_i8_off((uint32_t)i, (uint32_t)m, (uint32_t)k)] = (unsigned char)(int8_t)dg;
            }
        }
    }
}

}  // namespace qk
