// Per-device facts the launchers need, cached without locks: the SM count,
// and whether a kernel's dynamic shared-memory limit has been raised on this
// device (cudaFuncSetAttribute applies to the current device only).
#pragma once

#include <atomic>
#include <cstdint>

#include <cuda_runtime.h>

namespace qk {

constexpr int kMaxDevices = 64;

inline int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

// SM count of the current device.
inline int device_sms() {
    static std::atomic<int> cache[kMaxDevices];
    const int dev = current_device();
    int s = (dev >= 0 && dev < kMaxDevices) ? cache[dev].load(std::memory_order_relaxed) : 0;
    if (!s) {
        cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
        if (s <= 0) s = 148;
        if (dev >= 0 && dev < kMaxDevices) cache[dev].store(s, std::memory_order_relaxed);
    }
    return s;
}

// Raise func's dynamic shared-memory limit to `bytes` once per device;
// `done` is one bit per device, a static of the caller's kernel instance.
inline cudaError_t smem_limit_once(std::atomic<uint64_t> &done, const void *func, int bytes) {
    const int dev = current_device();
    const uint64_t bit = (dev >= 0 && dev < kMaxDevices) ? 1ull << dev : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
    return e;
}

}  // namespace qk
