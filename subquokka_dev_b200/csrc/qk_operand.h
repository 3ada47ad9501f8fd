// Tensor-core operand layouts shared by the kernels and their host-side
// builders (csrc/qk_dense_host.cpp): byte offsets in the canonical K-major
// 128-byte-swizzle layout (rows of 128 bytes, the 16-byte chunk index XORed
// with the row index mod 8, 8-row groups 1024 bytes apart).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define QK_HD __host__ __device__ __forceinline__
#else
#define QK_HD inline
#endif

namespace qk {

constexpr uint32_t kBf16OperandBytes = 128 * 128 * 2;   // one 128 x 128 bf16 operand

// Byte offset of element (row r, k) of a 128-row x 128-K bf16 operand in the
// canonical K-major 128-byte-swizzle layout: two K atoms of 64 elements (16 KB
// each, row r at 128 r), the 16-byte chunk index XORed with r % 8 so that
// eight rows' chunks at one K fall into different banks.
QK_HD uint32_t sw128_off(uint32_t r, uint32_t k) {
    return (k >> 6) * 16384u + r * 128u + ((((k >> 3) & 7u) ^ (r & 7u)) << 4) + (k & 7u) * 2u;
}

// Byte offset of digit k of row m of the complex128 operand's digit plane i
// (128 rows of 128 one-byte digits, 16 KiB a plane).
QK_HD uint32_t sw128_i8_off(uint32_t i, uint32_t m, uint32_t k) {
    return i * 16384u + m * 128u + ((((k >> 4) ^ m) & 7u) << 4) + (k & 15u);
}

}  // namespace qk
