// qk_apply_fused_noalloc: the fused-pass path for callers that cannot
// allocate device memory.
//
// qk_plan_apply keeps each plan's pass programs and coefficients in device
// buffers it allocates with cudaMalloc.  Some callers cannot allow that: a
// serving process that has handed all of HBM to a memory pool or to its own
// state vectors, or a tight loop where a cudaMalloc / cudaFree (which can
// synchronise the whole device) would stall other streams.  This entry point
// keeps the programs of one call in a fixed array of QK_NOALLOC_SCRATCH_BYTES
// (1 MiB) that lives in this file as a __device__ variable, so the caller
// passes only its own state buffer and nothing is allocated on the device.
//
// Set-up: the first call on a device asks the runtime for the array's device
// address (cudaGetSymbolAddress, with that device current) and caches it;
// make that first call before any stream capture on the device.  The cached
// address belongs to the module the runtime loaded for that device, so the
// library must not be used across a cudaDeviceReset (the module, and with it
// the array, may come back at another address).  Every later call on any
// stream shares the one array, and each call overwrites it with its own
// programs: calls that overlap on the GPU (different streams, no ordering
// between them) race on it.  Calls on one stream are ordered and safe.
// Nothing in the array needs to start at zero: every byte a pass reads is
// written by the same call first.
//
// The programs are copied from host vectors that this call owns and frees on
// return, so the call waits for its copies to finish (cudaStreamSynchronize)
// before it returns -- the same rule as every other upload from a host
// temporary in this library.  A stream that is being captured cannot be
// synchronised and a captured copy would read freed memory at replay, so a
// call on a capturing stream is refused with QK_ERR_UNSUPPORTED.
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "qk_internal.h"

namespace qk {
int run_plan_at(void *state, int dtype, const HostPlan &hp, const TOp *ops, const void *coef, cudaStream_t st);
}  // namespace qk

using namespace qk;

namespace {

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[QK_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (host code only
// has a host-side stand-in for the symbol, never a device address).
int scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(QK_ERR_UNSUPPORTED, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(QK_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return QK_OK;
}

}  // namespace

extern "C" int qk_apply_fused_noalloc(void *state, int nqubits, int dtype, const qk_gate *gates, size_t n,
                                      void *cuda_stream) {
    if (!state || (!gates && n)) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 36) return fail(QK_ERR_ARG, "nqubits must be in [1, 36], got %d", nqubits);
    if (dtype != QK_C128 && dtype != QK_C64) return fail(QK_ERR_ARG, "unknown dtype %d", dtype);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(st, &cap);
    if (ce != cudaSuccess) return fail(QK_ERR_CUDA, "cudaStreamIsCapturing: %s", cudaGetErrorString(ce));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(QK_ERR_UNSUPPORTED,
                    "qk_apply_fused_noalloc copies its programs from host memory it frees on return and waits for "
                    "them, which a stream under capture cannot do");
    HostPlan hp;
    int rc = build_plan(gates, n, nqubits, default_plan_options(dtype, nqubits), hp);
    if (rc) return rc;
    const size_t ops_bytes = (hp.ops.size() * sizeof(TOp) + 255) & ~(size_t)255;
    const size_t ncoef = hp.coef.size() / 2;
    const size_t coef_bytes = ncoef * (dtype == QK_C128 ? sizeof(double2) : sizeof(float2));
    if (ops_bytes + coef_bytes > QK_NOALLOC_SCRATCH_BYTES)
        return fail(QK_ERR_ARG,
                    "circuit needs %zu bytes of pass programs and coefficients; qk_apply_fused_noalloc holds at "
                    "most %u (split the circuit, or use qk_plan_create / qk_plan_apply)",
                    ops_bytes + coef_bytes, (unsigned)QK_NOALLOC_SCRATCH_BYTES);
    void *base = nullptr;
    rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char *b = static_cast<unsigned char *>(base);
    std::vector<float> f;   // complex64 coefficients; must outlive the copy
    cudaError_t e = cudaSuccess;
    if (!hp.ops.empty()) e = cudaMemcpyAsync(b, hp.ops.data(), hp.ops.size() * sizeof(TOp), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && ncoef) {
        if (dtype == QK_C128) {
            e = cudaMemcpyAsync(b + ops_bytes, hp.coef.data(), coef_bytes, cudaMemcpyHostToDevice, st);
        } else {
            f.assign(hp.coef.begin(), hp.coef.end());
            e = cudaMemcpyAsync(b + ops_bytes, f.data(), coef_bytes, cudaMemcpyHostToDevice, st);
        }
    }
    // hp and f are freed on return: the copies finish first
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(QK_ERR_CUDA, "copy to scratch: %s", cudaGetErrorString(e));
    return run_plan_at(state, dtype, hp, reinterpret_cast<const TOp *>(b), b + ops_bytes, st);
}
