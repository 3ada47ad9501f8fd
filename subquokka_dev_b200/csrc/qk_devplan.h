// Device copy of a fused plan: pass programs and coefficients.
#pragma once

#include <cstddef>
#include <vector>

#include <cuda_runtime.h>

#include "qk_internal.h"

namespace qk {

// Device copy of a host plan (programs + coefficients in the state's type).
struct DevPlan {
    TOp *ops = nullptr;
    void *coef = nullptr;
    int32_t *gparams = nullptr;  // gradient slot -> parameter index (adjoint plans)
    size_t ops_cap = 0, coef_cap = 0, gparams_cap = 0;  // bytes
    void release() {
        if (ops) cudaFree(ops);
        if (coef) cudaFree(coef);
        if (gparams) cudaFree(gparams);
        ops = nullptr;
        coef = nullptr;
        gparams = nullptr;
        ops_cap = coef_cap = gparams_cap = 0;
    }
};

// Device memory a state handle keeps between adjoint calls: the lambda state
// and checkpoints, the accumulators and the pass programs.  Grow-only; freed
// with the state or by qk_sv_release_workspace.
struct Workspace {
    void *states = nullptr;      // lambda + checkpoints
    size_t states_cap = 0;       // bytes
    double *acc = nullptr;       // gradient / <H> / drift accumulators
    size_t acc_cap = 0;          // bytes
    std::vector<DevPlan> plans;  // device programs of the sweep's passes
    // device time and traffic of the last sweep (qk_sv_last_sweep)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0, last_bytes = 0;
    int last_fwd = 0, last_bwd = 0, last_other = 0;

    // Timing events, created on first use.
    cudaError_t events() {
        cudaError_t e = cudaSuccess;
        if (!ev0) e = cudaEventCreate(&ev0);
        if (e == cudaSuccess && !ev1) e = cudaEventCreate(&ev1);
        return e;
    }

    // Make room for `states_bytes` of states, `acc_bytes` of accumulators and
    // `nplans` device plans.  Returns a cudaError_t.
    cudaError_t reserve(size_t states_bytes, size_t acc_bytes, size_t nplans) {
        if (states_bytes > states_cap) {
            if (states) cudaFree(states);
            states = nullptr;
            states_cap = 0;
            cudaError_t e = cudaMalloc(&states, states_bytes);
            if (e != cudaSuccess) return e;
            states_cap = states_bytes;
        }
        if (acc_bytes > acc_cap) {
            if (acc) cudaFree(acc);
            acc = nullptr;
            acc_cap = 0;
            cudaError_t e = cudaMalloc(&acc, acc_bytes);
            if (e != cudaSuccess) return e;
            acc_cap = acc_bytes;
        }
        if (plans.size() < nplans) plans.resize(nplans);
        return cudaSuccess;
    }
    void release() {
        if (states) cudaFree(states);
        if (acc) cudaFree(acc);
        states = nullptr;
        acc = nullptr;
        states_cap = acc_cap = 0;
        for (auto &p : plans) p.release();
        plans.clear();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        ev0 = ev1 = nullptr;
    }
};

}  // namespace qk
