// Expectation values of Pauli sums and adjoint gradients.
//
// The reference computes no observables and no gradients; these entry points
// are the engine's own (the variational workloads: a circuit of RX/RY/RZ
// rotations and fixed gates, H = sum of Pauli strings).
//
// Adjoint sweep (forward state uncomputed gate by gate, nothing stored but
// a few checkpoints):
//   psi = U_L..U_1 |psi0>, lambda = H psi, <H> = Re <psi|lambda>
//   for k = L..1:  g[p(k)] += Im <lambda|G_k|psi>   (U_k = exp(-i theta G_k / 2))
//                  psi <- U_k^dag psi, lambda <- U_k^dag lambda
// The gradient inner product is fused into the kernel that uncomputes both
// states, so a parameterised gate costs one read and one write of each.
// Forward states are kept at evenly spaced checkpoints; when the backward
// sweep reaches one, the uncomputed state is compared with it (drift) and
// replaced by it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include <cuda_runtime.h>

#include "qk_devplan.h"
#include "qk_device.h"
#include "qk_internal.h"
#include "qk_kernels.cuh"

namespace qk {

constexpr int kRedThreads = 256;
constexpr int kMaxGroupTerms = 64;

struct PauliGroup {
    uint64_t x;                       // X/Y part shared by the group
    int nterms;
    double coef[kMaxGroupTerms];      // real coefficient
    uint64_t z[kMaxGroupTerms];       // Z/Y part
    int ipow[kMaxGroupTerms];         // i^ipow from the Y factors (popcount(x & z) mod 4)
};

// factor(src) = sum_t coef_t i^ipow_t (-1)^popcount(src & z_t):
// (P psi)[src ^ x] = factor(src) psi[src]
__device__ __forceinline__ double2 group_factor(const PauliGroup &g, uint64_t src) {
    double re = 0, im = 0;
    for (int t = 0; t < g.nterms; ++t) {
        const double c = (__popcll(src & g.z[t]) & 1) ? -g.coef[t] : g.coef[t];
        switch (g.ipow[t] & 3) {
        case 0: re += c; break;
        case 1: im += c; break;
        case 2: re -= c; break;
        default: im -= c; break;
        }
    }
    return make_double2(re, im);
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[kRedThreads / 32];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (!l) red[w] = v;
    __syncthreads();
    v = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// acc += sum_j Re( conj(psi[j]) (P psi)[j] ) over one X-group:
// (P psi)[j] = factor(j ^ x) psi[j ^ x]
template <typename C>
__global__ void __launch_bounds__(kRedThreads) k_pauli_expval(const C *__restrict__ psi, uint64_t namp,
                                                              const __grid_constant__ PauliGroup g, double *acc) {
    double s = 0;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < namp; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t src = j ^ g.x;
        const C a = psi[j], b = psi[src];
        const double2 f = group_factor(g, src);
        // Re( conj(a) f b )
        const double br = (double)b.x * f.x - (double)b.y * f.y, bi = (double)b.x * f.y + (double)b.y * f.x;
        s += (double)a.x * br + (double)a.y * bi;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(acc, s);
}

// out[j] (+)= (P psi)[j] for one X-group
template <typename C>
__global__ void __launch_bounds__(kRedThreads) k_pauli_apply(C *__restrict__ out, const C *__restrict__ psi, uint64_t namp,
                                                             const __grid_constant__ PauliGroup g, int accumulate) {
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < namp; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t src = j ^ g.x;
        const C b = psi[src];
        const double2 f = group_factor(g, src);
        double re = (double)b.x * f.x - (double)b.y * f.y, im = (double)b.x * f.y + (double)b.y * f.x;
        if (accumulate) {
            const C o = out[j];
            re += o.x;
            im += o.y;
        }
        out[j] = mk<C>(re, im);
    }
}

// acc += Re <a|b>
template <typename C>
__global__ void __launch_bounds__(kRedThreads) k_dot_re(const C *__restrict__ a, const C *__restrict__ b, uint64_t namp,
                                                        double *acc) {
    double s = 0;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < namp; j += (uint64_t)gridDim.x * blockDim.x)
        s += (double)a[j].x * b[j].x + (double)a[j].y * b[j].y;
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(acc, s);
}

// acc += ||a - b||^2
template <typename C>
__global__ void __launch_bounds__(kRedThreads) k_dist2(const C *__restrict__ a, const C *__restrict__ b, uint64_t namp,
                                                       double *acc) {
    double s = 0;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < namp; j += (uint64_t)gridDim.x * blockDim.x) {
        const double dx = (double)a[j].x - b[j].x, dy = (double)a[j].y - b[j].y;
        s += dx * dx + dy * dy;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(acc, s);
}

// Im(conj(l) a)
template <typename C> __device__ __forceinline__ double im_dot(C l, C a) {
    return (double)l.x * a.y - (double)l.y * a.x;
}
template <typename C> __device__ __forceinline__ double re_dot(C l, C a) {
    return (double)l.x * a.x + (double)l.y * a.y;
}

// One parameterised rotation on qubit t, backward step: gradient
// Im<lambda|G|psi> (G = X, Y or Z by gen = 1, 2, 3) and both states
// multiplied by U^dag (u).
template <typename C>
__global__ void __launch_bounds__(kRedThreads) k_adj_rot(C *__restrict__ psi, C *__restrict__ lam, uint64_t npairs, int t,
                                                         Mat2<C> u, int gen, double *gacc) {
    const uint64_t h = 1ull << t;
    double s = 0;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i0 = ins0(p, t), i1 = i0 + h;
        const C a0 = psi[i0], a1 = psi[i1], l0 = lam[i0], l1 = lam[i1];
        if (gen == 1) s += im_dot(l0, a1) + im_dot(l1, a0);
        else if (gen == 2) s += re_dot(l1, a0) - re_dot(l0, a1);
        else s += im_dot(l0, a0) - im_dot(l1, a1);
        psi[i0] = cmul2(u.m[0], a0, u.m[1], a1);
        psi[i1] = cmul2(u.m[2], a0, u.m[3], a1);
        lam[i0] = cmul2(u.m[0], l0, u.m[1], l1);
        lam[i1] = cmul2(u.m[2], l0, u.m[3], l1);
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(gacc, s);
}

// from qk_engine.cu
int launch_gate_op(void *state, int n, int dtype, const Op &op, cudaStream_t st);

static int cuda_err(cudaError_t e, const char *what) {
    // An allocation failure is not sticky, but it stays as the thread's last
    // error; clear it so the next launch check does not report it again.
    if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? QK_ERR_OOM : QK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

static unsigned red_grid(uint64_t items) {
    const int sms = device_sms();
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + kRedThreads - 1) / kRedThreads, (uint64_t)sms * 8));
}

// Group Pauli terms by their X/Y mask.
static int group_terms(const qk_pauli_term *terms, size_t nterms, int n, std::vector<PauliGroup> &groups) {
    std::map<uint64_t, size_t> idx;
    const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1);
    for (size_t t = 0; t < nterms; ++t) {
        if ((terms[t].x_mask | terms[t].z_mask) & ~all)
            return fail(QK_ERR_QUBIT, "Pauli term %zu acts on a qubit >= %d", t, n);
        auto it = idx.find(terms[t].x_mask);
        if (it == idx.end() || groups[it->second].nterms == kMaxGroupTerms) {
            PauliGroup g;
            std::memset(&g, 0, sizeof g);
            g.x = terms[t].x_mask;
            groups.push_back(g);
            it = idx.insert_or_assign(terms[t].x_mask, groups.size() - 1).first;
        }
        PauliGroup &g = groups[it->second];
        g.coef[g.nterms] = terms[t].coeff;
        g.z[g.nterms] = terms[t].z_mask;
        g.ipow[g.nterms] = __builtin_popcountll(terms[t].x_mask & terms[t].z_mask) & 3;
        ++g.nterms;
    }
    return QK_OK;
}

template <typename C>
static int expval_t(const C *psi, int n, const std::vector<PauliGroup> &groups, double *dacc, cudaStream_t st) {
    const uint64_t namp = 1ull << n;
    for (const auto &g : groups) {
        k_pauli_expval<C><<<red_grid(namp), kRedThreads, 0, st>>>(psi, namp, g, dacc);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_err(e, "k_pauli_expval");
    }
    return QK_OK;
}

template <typename C>
static int apply_h_t(C *out, const C *psi, int n, const std::vector<PauliGroup> &groups, cudaStream_t st) {
    const uint64_t namp = 1ull << n;
    if (groups.empty()) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(C) * namp, st);
        return e == cudaSuccess ? QK_OK : cuda_err(e, "memset");
    }
    for (size_t i = 0; i < groups.size(); ++i) {
        k_pauli_apply<C><<<red_grid(namp), kRedThreads, 0, st>>>(out, psi, namp, groups[i], i > 0);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_err(e, "k_pauli_apply");
    }
    return QK_OK;
}

// generator of a trainable gate: 1 X (RX), 2 Y (RY), 3 Z (RZ), 0 not trainable
static int generator(const qk_gate &g) {
    return g.kind == QK_GATE_RX ? 1 : g.kind == QK_GATE_RY ? 2 : g.kind == QK_GATE_RZ ? 3 : 0;
}

template <typename C>
static int adjoint_t(C *psi, int n, int dtype, const qk_gate *gates, size_t ng, const int32_t *pidx, size_t nparams,
                     const std::vector<PauliGroup> &groups, int ncheck, double *expval, double *grad, double *drift,
                     Workspace &ws, cudaStream_t st) {
    const uint64_t namp = 1ull << n;
    const size_t bytes = sizeof(C) * namp;
    std::vector<Op> ops(ng);
    for (size_t i = 0; i < ng; ++i) {
        int rc = lower_gate(gates[i], ops[i]);
        if (rc) return rc;
        for (int k = 0; k < ops[i].nq; ++k)
            if (ops[i].q[k] < 0 || ops[i].q[k] >= n)
                return fail(QK_ERR_QUBIT, "gate %zu: qubit %d outside a %d-qubit state", i, ops[i].q[k], n);
        if (pidx && pidx[i] >= 0) {
            if ((size_t)pidx[i] >= nparams) return fail(QK_ERR_ARG, "gate %zu: parameter %d >= %zu", i, pidx[i], nparams);
            if (!generator(gates[i])) return fail(QK_ERR_UNSUPPORTED, "gate %zu: only RX, RY, RZ are trainable", i);
        }
    }
    // checkpoints: the state before gate c for evenly spaced c
    std::vector<size_t> cpos;
    if (ncheck < 0) ncheck = 0;
    if (ncheck > 0 && ng > 1) {
        for (int k = 1; k <= ncheck; ++k) {
            size_t c = (size_t)((double)ng * k / (ncheck + 1));
            if (c > 0 && c < ng && (cpos.empty() || c > cpos.back())) cpos.push_back(c);
        }
    }
    cudaError_t e = ws.reserve(bytes * (1 + cpos.size()), (nparams + 2) * sizeof(double), 0);
    if (e != cudaSuccess) return cuda_err(e, "cudaMalloc(adjoint workspace: lambda, checkpoints)");
    C *lam = static_cast<C *>(ws.states);
    C *ck = lam + namp;
    double *dacc = ws.acc;
    int rc = QK_OK;
    const size_t nacc = nparams + 2;  // grads, expval, drift
    e = ws.events();
    if (e == cudaSuccess) e = cudaEventRecord(ws.ev0, st);
    if (e != cudaSuccess) return cuda_err(e, "sweep timing events");
    ws.last_fwd = ws.last_bwd = (int)ng;   // one launch per gate each way
    ws.last_other = (int)(groups.size() + 1 + 3 * cpos.size());
    ws.last_bytes = 0;                     // not counted for the per-gate sweep
    e = cudaMemsetAsync(dacc, 0, nacc * sizeof(double), st);
    if (e != cudaSuccess) return cuda_err(e, "clear accumulators");

    // forward, saving checkpoints
    size_t nc = 0;
    for (size_t i = 0; i < ng; ++i) {
        if (nc < cpos.size() && cpos[nc] == i) {
            e = cudaMemcpyAsync(ck + nc * namp, psi, bytes, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_err(e, "checkpoint");
            ++nc;
        }
        rc = launch_gate_op(psi, n, dtype, ops[i], st);
        if (rc) return rc;
    }
    // lambda = H psi, <H> = Re<psi|lambda>
    rc = apply_h_t<C>(lam, psi, n, groups, st);
    if (rc) return rc;
    k_dot_re<C><<<red_grid(namp), kRedThreads, 0, st>>>(psi, lam, namp, dacc + nparams);
    // backward
    for (size_t i = ng; i-- > 0;) {
        Op inv = ops[i];
        invert_op(inv);
        const int p = pidx ? pidx[i] : -1;
        if (p >= 0) {
            Mat2<C> u;
            // RX/RY lower to dense 2x2, RZ to a diagonal: both as dense U^dag here
            if (inv.kind == OP_DENSE1) {
                for (int k = 0; k < 4; ++k) u.m[k] = mk<C>(inv.m[2 * k], inv.m[2 * k + 1]);
            } else {
                u.m[0] = mk<C>(inv.m[0], inv.m[1]);
                u.m[1] = mk<C>(0, 0);
                u.m[2] = mk<C>(0, 0);
                u.m[3] = mk<C>(inv.m[2], inv.m[3]);
            }
            const uint64_t np = namp / 2;
            k_adj_rot<C><<<red_grid(np), kRedThreads, 0, st>>>(psi, lam, np, inv.q[0], u, generator(gates[i]), dacc + p);
            e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_err(e, "k_adj_rot");
        } else {
            rc = launch_gate_op(psi, n, dtype, inv, st);
            if (!rc) rc = launch_gate_op(lam, n, dtype, inv, st);
            if (rc) return rc;
        }
        // psi now holds the state before gate i: compare with and restore from a checkpoint
        if (nc > 0 && cpos[nc - 1] == i) {
            --nc;
            k_dist2<C><<<red_grid(namp), kRedThreads, 0, st>>>(psi, ck + nc * namp, namp, dacc + nparams + 1);
            e = cudaMemcpyAsync(psi, ck + nc * namp, bytes, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_err(e, "restore checkpoint");
        }
    }
    e = cudaEventRecord(ws.ev1, st);
    if (e != cudaSuccess) return cuda_err(e, "sweep timing events");
    std::vector<double> h(nacc);
    e = cudaMemcpyAsync(h.data(), dacc, nacc * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "read results");
    {
        float ms = 0;
        ws.last_ms = cudaEventElapsedTime(&ms, ws.ev0, ws.ev1) == cudaSuccess ? ms : -1.0;
    }
    if (grad) std::memcpy(grad, h.data(), nparams * sizeof(double));
    if (expval) *expval = h[nparams];
    if (drift) *drift = std::sqrt(h[nparams + 1]);
    return QK_OK;
}

// fused passes (qk_pass.cu)
int upload_host_plan(const HostPlan &hp, DevPlan &dp, cudaStream_t st);
int run_forward_plan(void *state, const HostPlan &hp, const DevPlan &dp, cudaStream_t st);
int run_adjoint_plan(void *psi, void *lam, int dtype, const HostPlan &hp, const DevPlan &dp, double *ggrad,
                     cudaStream_t st);

// The same sweep with fused passes: the gates are cut into segments at the
// checkpoints; each segment runs forward as fused passes and backward as
// two-state adjoint passes (inverse gates on psi and lambda, gradients taken
// inside the passes).  At a segment start psi is compared with and restored
// from the checkpoint.
template <typename C>
static int adjoint_fused_t(C *psi, int n, int dtype, const qk_gate *gates, size_t ng, const int32_t *pidx,
                           size_t nparams, const std::vector<PauliGroup> &groups, int ncheck, double *expval,
                           double *grad, double *drift, Workspace &ws, cudaStream_t st) {
    const uint64_t namp = 1ull << n;
    const size_t bytes = sizeof(C) * namp;
    std::vector<size_t> cut{0};
    if (ncheck > 0 && ng > 1)
        for (int k = 1; k <= ncheck; ++k) {
            size_t c = (size_t)((double)ng * k / (ncheck + 1));
            if (c > cut.back() && c < ng) cut.push_back(c);
        }
    cut.push_back(ng);
    const size_t nseg = cut.size() - 1;
    std::vector<HostPlan> fwd(nseg), bwd(nseg);
    PlanOptions fo = default_plan_options(dtype, n), bo = default_adjoint_options(dtype, n);
    for (size_t sgi = 0; sgi < nseg; ++sgi) {
        int rc = build_plan(gates + cut[sgi], cut[sgi + 1] - cut[sgi], n, fo, fwd[sgi]);
        if (!rc) rc = build_adjoint_plan(gates + cut[sgi], cut[sgi + 1] - cut[sgi], pidx ? pidx + cut[sgi] : nullptr,
                                         n, bo, bwd[sgi]);
        if (rc) return rc;
        for (int32_t p : bwd[sgi].grad_params)
            if (p < 0 || (size_t)p >= nparams) return fail(QK_ERR_ARG, "parameter %d >= %zu", p, nparams);
    }
    const size_t nacc = nparams + 2;
    cudaError_t e = ws.reserve(bytes * nseg, nacc * sizeof(double), 2 * nseg);
    if (e != cudaSuccess) return cuda_err(e, "cudaMalloc(adjoint workspace: lambda, checkpoints)");
    C *lam = static_cast<C *>(ws.states);
    C *ck = lam + namp;
    double *dacc = ws.acc;
    for (size_t sgi = 0; sgi < nseg; ++sgi) {
        int rc = upload_host_plan(fwd[sgi], ws.plans[2 * sgi], st);
        if (!rc) rc = upload_host_plan(bwd[sgi], ws.plans[2 * sgi + 1], st);
        if (rc) return rc;
    }
    e = ws.events();
    if (e == cudaSuccess) e = cudaEventRecord(ws.ev0, st);
    if (e != cudaSuccess) return cuda_err(e, "sweep timing events");
    e = cudaMemsetAsync(dacc, 0, nacc * sizeof(double), st);
    if (e != cudaSuccess) return cuda_err(e, "clear accumulators");
    // algorithmic traffic: a forward pass reads and writes psi (2S), a
    // two-state pass psi and lambda (4S); lambda = H psi reads psi and writes
    // lambda (2S) and every further Pauli group re-reads lambda (3S); <H>
    // reads both (2S); each checkpoint copy, drift check and restore 2S
    ws.last_fwd = ws.last_bwd = ws.last_other = 0;
    for (size_t sgi = 0; sgi < nseg; ++sgi) {
        ws.last_fwd += (int)fwd[sgi].passes.size();
        ws.last_bwd += (int)bwd[sgi].passes.size();
    }
    const double S = (double)bytes;
    const double ng_h = groups.empty() ? 1.0 : (double)groups.size();
    ws.last_other = (int)(ng_h + 1 + 3 * (nseg - 1));
    ws.last_bytes = 2 * S * ws.last_fwd + 4 * S * ws.last_bwd + (groups.empty() ? S : 2 * S + 3 * S * (ng_h - 1)) +
                    2 * S + 3 * 2 * S * (double)(nseg - 1);
    // forward
    for (size_t sgi = 0; sgi < nseg; ++sgi) {
        if (sgi > 0) {
            e = cudaMemcpyAsync(ck + (sgi - 1) * namp, psi, bytes, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_err(e, "checkpoint");
        }
        int rc = run_forward_plan(psi, fwd[sgi], ws.plans[2 * sgi], st);
        if (rc) return rc;
    }
    int rc = apply_h_t<C>(lam, psi, n, groups, st);
    if (rc) return rc;
    k_dot_re<C><<<red_grid(namp), kRedThreads, 0, st>>>(psi, lam, namp, dacc + nparams);
    // backward
    for (size_t sgi = nseg; sgi-- > 0;) {
        rc = run_adjoint_plan(psi, lam, dtype, bwd[sgi], ws.plans[2 * sgi + 1], dacc, st);
        if (rc) return rc;
        if (sgi > 0) {
            k_dist2<C><<<red_grid(namp), kRedThreads, 0, st>>>(psi, ck + (sgi - 1) * namp, namp, dacc + nparams + 1);
            e = cudaMemcpyAsync(psi, ck + (sgi - 1) * namp, bytes, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_err(e, "restore checkpoint");
        }
    }
    e = cudaEventRecord(ws.ev1, st);
    if (e != cudaSuccess) return cuda_err(e, "sweep timing events");
    std::vector<double> h(nacc);
    e = cudaMemcpyAsync(h.data(), dacc, nacc * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "read results");
    {
        float ms = 0;
        ws.last_ms = cudaEventElapsedTime(&ms, ws.ev0, ws.ev1) == cudaSuccess ? ms : -1.0;
    }
    if (grad) std::memcpy(grad, h.data(), nparams * sizeof(double));
    if (expval) *expval = h[nparams];
    if (drift) *drift = std::sqrt(h[nparams + 1]);
    return QK_OK;
}

}  // namespace qk

using namespace qk;

// state accessors defined in qk_engine.cu
namespace qk {
cudaStream_t state_stream(const qk_sv *sv);
void *state_ptr(const qk_sv *sv);
int state_qubits(const qk_sv *sv);
int state_dtype(const qk_sv *sv);
Workspace &state_workspace(qk_sv *sv);
}  // namespace qk

extern "C" {

int qk_expval_pauli(qk_sv *sv, const qk_pauli_term *terms, size_t nterms, double *out) {
    if (!sv || !out || (!terms && nterms)) return fail(QK_ERR_ARG, "null argument");
    const int n = state_qubits(sv);
    std::vector<PauliGroup> groups;
    int rc = group_terms(terms, nterms, n, groups);
    if (rc) return rc;
    cudaStream_t st = state_stream(sv);
    Workspace &ws = state_workspace(sv);
    cudaError_t e = ws.reserve(0, sizeof(double), 0);
    if (e != cudaSuccess) return cuda_err(e, "cudaMalloc(accumulator)");
    double *dacc = ws.acc;
    e = cudaMemsetAsync(dacc, 0, sizeof(double), st);
    if (e != cudaSuccess) return cuda_err(e, "clear accumulator");
    rc = state_dtype(sv) == QK_C128 ? expval_t<double2>((const double2 *)state_ptr(sv), n, groups, dacc, st)
                                    : expval_t<float2>((const float2 *)state_ptr(sv), n, groups, dacc, st);
    if (!rc) {
        e = cudaMemcpyAsync(out, dacc, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_err(e, "read expectation");
    }
    return rc;
}

int qk_adjoint_grad(qk_sv *sv, const qk_gate *gates, size_t ngates, const int32_t *param_index, size_t nparams,
                    const qk_pauli_term *terms, size_t nterms, int checkpoints, double *expval, double *grad,
                    double *drift) {
    if (!sv || (!gates && ngates) || (!terms && nterms) || (!grad && nparams))
        return fail(QK_ERR_ARG, "null argument");
    const int n = state_qubits(sv);
    std::vector<PauliGroup> groups;
    int rc = group_terms(terms, nterms, n, groups);
    if (rc) return rc;
    if (checkpoints < 0) checkpoints = std::min<int>(8, (int)std::ceil(std::sqrt((double)ngates)));
    const int dtype = state_dtype(sv);
    cudaStream_t st = state_stream(sv);
    if (dtype == QK_C128)
        return adjoint_t<double2>((double2 *)state_ptr(sv), n, dtype, gates, ngates, param_index, nparams, groups,
                                  checkpoints, expval, grad, drift, state_workspace(sv), st);
    return adjoint_t<float2>((float2 *)state_ptr(sv), n, dtype, gates, ngates, param_index, nparams, groups,
                             checkpoints, expval, grad, drift, state_workspace(sv), st);
}

int qk_adjoint_grad_fused(qk_sv *sv, const qk_gate *gates, size_t ngates, const int32_t *param_index, size_t nparams,
                          const qk_pauli_term *terms, size_t nterms, int checkpoints, double *expval, double *grad,
                          double *drift) {
    if (!sv || (!gates && ngates) || (!terms && nterms) || (!grad && nparams))
        return fail(QK_ERR_ARG, "null argument");
    const int n = state_qubits(sv);
    std::vector<PauliGroup> groups;
    int rc = group_terms(terms, nterms, n, groups);
    if (rc) return rc;
    if (checkpoints < 0) checkpoints = std::min<int>(8, (int)std::ceil(std::sqrt((double)ngates)) / 4);
    const int dtype = state_dtype(sv);
    cudaStream_t st = state_stream(sv);
    if (dtype == QK_C128)
        return adjoint_fused_t<double2>((double2 *)state_ptr(sv), n, dtype, gates, ngates, param_index, nparams,
                                        groups, checkpoints, expval, grad, drift, state_workspace(sv), st);
    return adjoint_fused_t<float2>((float2 *)state_ptr(sv), n, dtype, gates, ngates, param_index, nparams, groups,
                                   checkpoints, expval, grad, drift, state_workspace(sv), st);
}

}  // extern "C"
