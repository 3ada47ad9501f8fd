// Device copy of a fused plan: pass programs and coefficients.
#pragma once

#include <cstddef>
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

}  // namespace qk
