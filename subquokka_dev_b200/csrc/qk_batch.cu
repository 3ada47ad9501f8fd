// Batched variational circuits: many circuits of different sizes, forward
// + <H> + adjoint gradients, as one CUDA graph.
//
// Every circuit gets a forward plan and an adjoint plan (fused passes).  Step
// k of the batch is ONE persistent launch of k_pass_batch that runs the k-th
// pass of every circuit that has one: the work items are the tiles of all
// those circuits, split into contiguous ranges, one per CTA.  Resetting the
// states, applying H, the expectation values and the drift check are batched
// kernels driven by a block -> circuit table.  The whole sequence is captured
// once into a CUDA graph; a parameter update rewrites the pinned host copy of
// the coefficients, which the graph's first node copies to the device.
//
// The reference has no counterpart (no gradients, no batching).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "qk_devplan.h"
#include "qk_device.h"
#include "qk_internal.h"
#include "qk_pass_device.cuh"

namespace qk {

template <typename C> struct BatchEntry {
    C *s, *s2;                 // psi, lambda (adjoint steps)
    const TOp *prog;           // the pass's program (already offset)
    const C *coef;             // its coefficients (already offset)
    const int32_t *gparams;    // its gradient slots -> parameter index
    double *ggrad;             // the circuit's gradient array
    uint64_t tile0, ntiles;    // global item range of this entry
    PassDesc d;                // prog0 = coef0 = grad0 = 0
};

// One persistent launch over the k-th pass of every circuit.
template <typename C, int R, int NS>
__global__ void __launch_bounds__(pass_max_threads<C, R, NS>()) k_pass_batch(const BatchEntry<C> *__restrict__ tab,
                                                                            int nent, uint64_t total, uint64_t chunk) {
    constexpr int LOG2R = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : R == 16 ? 4 : 5;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ PassDesc sd;
    const uint64_t beg = (uint64_t)blockIdx.x * chunk;
    const uint64_t end = beg + chunk < total ? beg + chunk : total;
    if (beg >= end) return;
    const uint32_t NT = blockDim.x;
    // first entry holding item beg
    int lo = 0, hi = nent - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (tab[mid].tile0 <= beg) lo = mid;
        else hi = mid - 1;
    }
    int e = lo, loaded = -1;
    uint32_t N = 0;
    C *tl = nullptr, *tw = nullptr;
    TOp *prog = nullptr;
    C *coef = nullptr;
    double *gsm = nullptr;
    TileAddr<C, LOG2R> ta;
    for (uint64_t it = beg; it < end; ++it) {
        while (it >= tab[e].tile0 + tab[e].ntiles) ++e;
        if (e != loaded) {
            __syncthreads();
            if constexpr (NS == 2) {
                if (loaded >= 0)
                    for (int i = threadIdx.x; i < sd.ngrad; i += NT) atomicAdd(tab[loaded].ggrad + tab[loaded].gparams[i], gsm[i]);
            }
            __syncthreads();
            if (threadIdx.x == 0) sd = tab[e].d;
            __syncthreads();
            N = 1u << sd.T;
            tl = reinterpret_cast<C *>(smem_raw);
            tw = tl + N;
            prog = reinterpret_cast<TOp *>(tl + (size_t)N * NS);
            coef = reinterpret_cast<C *>(prog + sd.nprog);
            gsm = reinterpret_cast<double *>(coef + sd.ncoef);
            for (int i = threadIdx.x; i < sd.nprog; i += NT) prog[i] = tab[e].prog[i];
            for (int i = threadIdx.x; i < sd.ncoef; i += NT) coef[i] = tab[e].coef[i];
            if constexpr (NS == 2)
                for (int i = threadIdx.x; i < sd.ngrad; i += NT) gsm[i] = 0.0;
            ta.init(sd, NT);
            loaded = e;
        }
        C *s = tab[e].s, *s2 = tab[e].s2;
        const uint64_t base = pass_base(it - tab[e].tile0, sd);
        __syncthreads();  // previous tile's stores have read the buffers
#pragma unroll
        for (int u = 0; u < R; ++u) {
            cp_async_amp(tl + ta.sidx(u), s + (base | ta.g(u)));
            if constexpr (NS == 2) cp_async_amp(tw + ta.sidx(u), s2 + (base | ta.g(u)));
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        run_program<C, R, NS, false>(tl, tw, base, sd, prog, coef, gsm, N);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < R; ++u) {
            s[base | ta.g(u)] = tl[ta.sidx(u)];
            if constexpr (NS == 2) s2[base | ta.g(u)] = tw[ta.sidx(u)];
        }
    }
    if constexpr (NS == 2) {
        __syncthreads();
        for (int i = threadIdx.x; i < sd.ngrad; i += NT) atomicAdd(tab[loaded].ggrad + tab[loaded].gparams[i], gsm[i]);
    }
}

// ---- batched element-wise kernels (block -> circuit table) ------------------

constexpr int kBatchThreads = 256;
constexpr uint32_t kBatchChunk = 8192;  // amplitudes per block

struct BatchState {
    void *psi, *lam;
    uint64_t namp;
    int term0, nterm;       // slice of the term table
    double *expval, *drift;  // per-circuit outputs (device)
};

struct BatchTerm {
    double coef;
    uint64_t x, z;
    int ipow;
};

__device__ __forceinline__ double batch_block_sum(double v) {
    __shared__ double red[kBatchThreads / 32];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (!l) red[w] = v;
    __syncthreads();
    v = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// mode 0: psi = |0...0>, clear the circuit's outputs
// mode 1: lambda = H psi, expval += Re <psi|lambda>
// mode 2: drift += || psi - |0...0> ||^2
template <typename C>
__global__ void __launch_bounds__(kBatchThreads) k_batch_elem(const BatchState *__restrict__ st,
                                                              const BatchTerm *__restrict__ terms,
                                                              const int *__restrict__ blk_circ,
                                                              const uint32_t *__restrict__ blk_first, int mode) {
    const BatchState S = st[blk_circ[blockIdx.x]];
    C *psi = (C *)S.psi, *lam = (C *)S.lam;
    const uint64_t j0 = (uint64_t)blk_first[blockIdx.x] * kBatchChunk;
    const uint64_t j1 = j0 + kBatchChunk < S.namp ? j0 + kBatchChunk : S.namp;
    double acc = 0;
    for (uint64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        if (mode == 0) {
            psi[j] = mk<C>(j == 0 ? 1.0 : 0.0, 0.0);
        } else if (mode == 1) {
            double re = 0, im = 0;
            for (int t = S.term0; t < S.term0 + S.nterm; ++t) {
                const BatchTerm T = terms[t];
                const uint64_t src = j ^ T.x;
                const C b = psi[src];
                const double c = (__popcll(src & T.z) & 1) ? -T.coef : T.coef;
                double fr = 0, fi = 0;
                switch (T.ipow & 3) {
                case 0: fr = c; break;
                case 1: fi = c; break;
                case 2: fr = -c; break;
                default: fi = -c; break;
                }
                re += fr * b.x - fi * b.y;
                im += fr * b.y + fi * b.x;
            }
            lam[j] = mk<C>(re, im);
            const C a = psi[j];
            acc += (double)a.x * re + (double)a.y * im;
        } else {
            const C a = psi[j];
            const double dx = (double)a.x - (j == 0 ? 1.0 : 0.0), dy = a.y;
            acc += dx * dx + dy * dy;
        }
    }
    if (mode == 0) {
        if (j0 == 0 && threadIdx.x == 0) {
            *S.expval = 0.0;
            *S.drift = 0.0;
        }
        return;
    }
    acc = batch_block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(mode == 1 ? S.expval : S.drift, acc);
}

static int cuda_err(cudaError_t e, const char *what) {
    // An allocation failure is not sticky, but it stays as the thread's last
    // error; clear it so the next launch check does not report it again.
    if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? QK_ERR_OOM : QK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace qk

using namespace qk;

struct qk_batch {
    int ncirc = 0, dtype = QK_C64;
    PlanOptions fo{}, bo{};
    std::vector<int> n;                        // qubits per circuit
    std::vector<std::vector<qk_gate>> gates;   // per circuit (angles rebound by set_params)
    std::vector<std::vector<int32_t>> pidx;    // per circuit
    std::vector<size_t> poff;                  // parameter offsets
    size_t nparams = 0;
    std::vector<HostPlan> fplan, bplan;
    // device memory
    std::vector<void *> psi, lam;
    DevPlan fdev, bdev;                        // all circuits' programs, concatenated
    std::vector<size_t> f_op0, f_c0, b_op0, b_c0, b_g0;  // per-circuit offsets into the concatenation
    void *coef_host = nullptr;                 // pinned: forward + backward coefficients, state type
    size_t fcoef_bytes = 0, bcoef_bytes = 0;
    double *d_out = nullptr;                   // grads | expvals | drift
    double *h_out = nullptr;                   // pinned copy
    BatchState *d_states = nullptr;
    BatchTerm *d_terms = nullptr;
    int *d_blk_circ = nullptr;
    uint32_t *d_blk_first = nullptr;
    int nblk = 0;
    std::vector<void *> d_tables;              // per-step entry tables
    struct Step {
        int ns;              // 1 forward, 2 adjoint
        const void *tab;
        int nent;
        uint64_t total;
        size_t smem;
        int T, r;
    };
    std::vector<Step> steps;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t launches = 0;
    // qk_batch_timing: events around the last graph launch, algorithmic bytes of one run
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0, alg_bytes = 0;

    // programs, step tables, coefficient buffer and graph (rebuilt per tile shape)
    void free_plans() {
        fdev.release();
        bdev.release();
        for (void *p : d_tables) cudaFree(p);
        d_tables.clear();
        if (coef_host) cudaFreeHost(coef_host);
        coef_host = nullptr;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        steps.clear();
    }
    void free_device() {
        free_plans();
        for (void *p : psi) if (p) cudaFree(p);
        for (void *p : lam) if (p) cudaFree(p);
        psi.clear();
        lam.clear();
        if (d_out) cudaFree(d_out);
        if (d_states) cudaFree(d_states);
        if (d_terms) cudaFree(d_terms);
        if (d_blk_circ) cudaFree(d_blk_circ);
        if (d_blk_first) cudaFree(d_blk_first);
        if (h_out) cudaFreeHost(h_out);
        d_out = nullptr;
        d_states = nullptr;
        d_terms = nullptr;
        d_blk_circ = nullptr;
        d_blk_first = nullptr;
        h_out = nullptr;
    }
    ~qk_batch() {
        free_device();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace qk {

// Coefficients of all plans, in the state type, into the pinned host buffer.
static void fill_coefficients(qk_batch *b) {
    const size_t cs = b->dtype == QK_C128 ? 16 : 8;
    unsigned char *h = static_cast<unsigned char *>(b->coef_host);
    auto put = [&](const std::vector<double> &c, size_t off) {
        if (b->dtype == QK_C128) std::memcpy(h + off, c.data(), c.size() * sizeof(double));
        else
            for (size_t i = 0; i < c.size(); ++i) reinterpret_cast<float *>(h + off)[i] = (float)c[i];
    };
    for (int c = 0; c < b->ncirc; ++c) {
        put(b->fplan[c].coef, b->f_c0[c] * cs);
        put(b->bplan[c].coef, b->fcoef_bytes + b->b_c0[c] * cs);
    }
}

template <typename C>
static int build_tables(qk_batch *b) {
    // step tables: step k = k-th pass of every circuit
    size_t fmax = 0, bmax = 0;
    for (int c = 0; c < b->ncirc; ++c) {
        fmax = std::max(fmax, b->fplan[c].passes.size());
        bmax = std::max(bmax, b->bplan[c].passes.size());
    }
    const TOp *fops = b->fdev.ops, *bops = b->bdev.ops;
    const C *fcoef = (const C *)b->fdev.coef, *bcoef = (const C *)b->bdev.coef;
    double *grads = b->d_out;
    // algorithmic traffic of one run: per circuit of S bytes, a forward pass
    // 2S, a two-state pass 4S, the reset S, lambda = H psi 2S (psi read,
    // lambda written), the drift check S
    b->alg_bytes = 0;
    for (int c = 0; c < b->ncirc; ++c) {
        const double S = (double)sizeof(C) * (double)(1ull << b->n[c]);
        b->alg_bytes += S * (2.0 * b->fplan[c].passes.size() + 4.0 * b->bplan[c].passes.size() + 4.0);
    }
    for (int ns = 1; ns <= 2; ++ns) {
        const size_t kmax = ns == 1 ? fmax : bmax;
        for (size_t k = 0; k < kmax; ++k) {
            std::vector<BatchEntry<C>> tab;
            uint64_t total = 0;
            size_t prog_bytes = 0;
            int T = -1;
            for (int c = 0; c < b->ncirc; ++c) {
                const HostPlan &hp = ns == 1 ? b->fplan[c] : b->bplan[c];
                if (k >= hp.passes.size()) continue;
                PassDesc d = hp.passes[k];
                if (d.perm) return fail(QK_ERR_UNSUPPORTED, "batched circuits cannot contain VSWAP gates");
                if (T < 0) T = d.T;
                if (d.T != T) return fail(QK_ERR_ARG, "batched passes need one tile size (circuit %d)", c);
                BatchEntry<C> en;
                std::memset(&en, 0, sizeof en);
                en.s = (C *)b->psi[c];
                en.s2 = ns == 2 ? (C *)b->lam[c] : nullptr;
                const size_t op0 = ns == 1 ? b->f_op0[c] : b->b_op0[c];
                const size_t c0 = ns == 1 ? b->f_c0[c] : b->b_c0[c];
                en.prog = (ns == 1 ? fops : bops) + op0 + d.prog0;
                en.coef = (ns == 1 ? fcoef : bcoef) + c0 + d.coef0;
                en.gparams = ns == 2 ? b->bdev.gparams + b->b_g0[c] + d.grad0 : nullptr;
                en.ggrad = grads + b->poff[c];
                en.tile0 = total;
                en.ntiles = 1ull << (b->n[c] - d.T);
                d.prog0 = d.coef0 = d.grad0 = 0;
                en.d = d;
                tab.push_back(en);
                total += en.ntiles;
                prog_bytes = std::max(prog_bytes, d.nprog * sizeof(TOp) + d.ncoef * sizeof(C) +
                                                      (ns == 2 ? d.ngrad * sizeof(double) : 0));
            }
            if (tab.empty()) continue;
            void *dt = nullptr;
            cudaError_t e = cudaMalloc(&dt, tab.size() * sizeof(BatchEntry<C>));
            if (e == cudaSuccess)
                e = cudaMemcpy(dt, tab.data(), tab.size() * sizeof(BatchEntry<C>), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return cuda_err(e, "batch step table");
            b->d_tables.push_back(dt);
            qk_batch::Step s;
            s.ns = ns;
            s.tab = dt;
            s.nent = (int)tab.size();
            s.total = total;
            s.T = T;
            s.r = ns == 1 ? b->fo.reg_bits : b->bo.reg_bits;
            s.smem = ((size_t)sizeof(C) << T) * ns + prog_bytes;
            if (s.smem > (220u << 10)) return fail(QK_ERR_ARG, "batched pass needs %zu bytes of shared memory", s.smem);
            b->steps.push_back(s);
        }
    }
    return QK_OK;
}

template <typename C, int R, int NS>
static int launch_batch_step(const qk_batch::Step &s, cudaStream_t st) {
    static std::atomic<uint64_t> smem_done{0};
    const cudaError_t ea = smem_limit_once(smem_done, (const void *)k_pass_batch<C, R, NS>, 220 << 10);
    if (ea != cudaSuccess) return cuda_err(ea, "cudaFuncSetAttribute(k_pass_batch)");
    const int sms = device_sms();
    const unsigned threads = (1u << s.T) / R;
    int mb = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mb, k_pass_batch<C, R, NS>, (int)threads, s.smem);
    if (mb < 1) mb = 1;
    const uint64_t ctas = std::min<uint64_t>(s.total, (uint64_t)sms * mb);
    const uint64_t chunk = (s.total + ctas - 1) / ctas;
    const unsigned grid = (unsigned)((s.total + chunk - 1) / chunk);
    k_pass_batch<C, R, NS><<<grid, threads, s.smem, st>>>((const BatchEntry<C> *)s.tab, s.nent, s.total, chunk);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QK_OK : cuda_err(e, "k_pass_batch launch");
}

template <typename C>
static int launch_step(const qk_batch::Step &s, cudaStream_t st) {
    if (s.ns == 1) {
        switch (s.r) {
        case 2: return launch_batch_step<C, 4, 1>(s, st);
        case 3: return launch_batch_step<C, 8, 1>(s, st);
        case 4: return launch_batch_step<C, 16, 1>(s, st);
        }
    } else {
        switch (s.r) {
        case 2: return launch_batch_step<C, 4, 2>(s, st);
        case 3: return launch_batch_step<C, 8, 2>(s, st);
        case 4:
            if constexpr (sizeof(C) == sizeof(float2)) return launch_batch_step<C, 16, 2>(s, st);
            break;
        }
    }
    return fail(QK_ERR_ARG, "reg_bits %d unsupported in batched passes", s.r);
}

// Enqueue one whole batch evaluation on b->stream (captured into the graph).
template <typename C>
static int enqueue(qk_batch *b) {
    cudaStream_t st = b->stream;
    size_t launches = 0;
    cudaError_t e = cudaMemcpyAsync(b->fdev.coef, b->coef_host, b->fcoef_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->bdev.coef, (unsigned char *)b->coef_host + b->fcoef_bytes, b->bcoef_bytes,
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_out, 0, b->nparams * sizeof(double), st);
    if (e != cudaSuccess) return cuda_err(e, "batch coefficients");
    k_batch_elem<C><<<b->nblk, kBatchThreads, 0, st>>>(b->d_states, b->d_terms, b->d_blk_circ, b->d_blk_first, 0);
    ++launches;
    bool h_done = false;
    for (const auto &s : b->steps) {
        if (s.ns == 2 && !h_done) {
            k_batch_elem<C><<<b->nblk, kBatchThreads, 0, st>>>(b->d_states, b->d_terms, b->d_blk_circ, b->d_blk_first, 1);
            ++launches;
            h_done = true;
        }
        int rc = launch_step<C>(s, st);
        if (rc) return rc;
        ++launches;
    }
    if (!h_done) {
        k_batch_elem<C><<<b->nblk, kBatchThreads, 0, st>>>(b->d_states, b->d_terms, b->d_blk_circ, b->d_blk_first, 1);
        ++launches;
    }
    k_batch_elem<C><<<b->nblk, kBatchThreads, 0, st>>>(b->d_states, b->d_terms, b->d_blk_circ, b->d_blk_first, 2);
    ++launches;
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_out, b->d_out, (b->nparams + 2 * b->ncirc) * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_err(e, "batch enqueue");
    b->launches = launches;
    return QK_OK;
}

// Build every circuit's plans (host threads, one circuit at a time each).
static int build_all_plans(qk_batch *b) {
    b->fplan.assign(b->ncirc, HostPlan());
    b->bplan.assign(b->ncirc, HostPlan());
    std::vector<int> rcs(b->ncirc, QK_OK);
    std::vector<std::string> errs(b->ncirc);
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int c = next++; c < b->ncirc; c = next++) {
            PlanOptions fo = b->fo, bo = b->bo;
            fo.tile_bits = std::min(fo.tile_bits, b->n[c]);
            bo.tile_bits = std::min(bo.tile_bits, b->n[c]);
            int rc = build_plan(b->gates[c].data(), b->gates[c].size(), b->n[c], fo, b->fplan[c]);
            if (!rc)
                rc = build_adjoint_plan(b->gates[c].data(), b->gates[c].size(), b->pidx[c].data(), b->n[c], bo,
                                        b->bplan[c]);
            if (rc) {
                rcs[c] = rc;
                errs[c] = qk_last_error();
            }
        }
    };
    const int nt = std::max(1, std::min<int>(b->ncirc, (int)std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    for (int c = 0; c < b->ncirc; ++c)
        if (rcs[c]) return fail(rcs[c], "circuit %d: %s", c, errs[c].c_str());
    return QK_OK;
}

// Build plans, upload programs and coefficients (states are allocated once).
static int prepare(qk_batch *b) {
    b->free_plans();
    const int dt = b->dtype;
    const size_t cs = dt == QK_C128 ? 16 : 8;
    int prc = build_all_plans(b);
    if (prc) return prc;
    // concatenate programs
    HostPlan fall, ball;
    b->f_op0.assign(b->ncirc, 0);
    b->f_c0.assign(b->ncirc, 0);
    b->b_op0.assign(b->ncirc, 0);
    b->b_c0.assign(b->ncirc, 0);
    b->b_g0.assign(b->ncirc, 0);
    for (int c = 0; c < b->ncirc; ++c) {
        b->f_op0[c] = fall.ops.size();
        b->f_c0[c] = fall.coef.size() / 2;
        fall.ops.insert(fall.ops.end(), b->fplan[c].ops.begin(), b->fplan[c].ops.end());
        fall.coef.insert(fall.coef.end(), b->fplan[c].coef.begin(), b->fplan[c].coef.end());
        b->b_op0[c] = ball.ops.size();
        b->b_c0[c] = ball.coef.size() / 2;
        b->b_g0[c] = ball.grad_params.size();
        ball.ops.insert(ball.ops.end(), b->bplan[c].ops.begin(), b->bplan[c].ops.end());
        ball.coef.insert(ball.coef.end(), b->bplan[c].coef.begin(), b->bplan[c].coef.end());
        ball.grad_params.insert(ball.grad_params.end(), b->bplan[c].grad_params.begin(), b->bplan[c].grad_params.end());
    }
    fall.dtype = ball.dtype = dt;
    cudaError_t e;
    auto alloc = [&](void **p, size_t bytes) {
        e = cudaMalloc(p, std::max<size_t>(bytes, 16));
        return e == cudaSuccess;
    };
    // programs (coefficients are copied by the graph from the pinned buffer)
    b->fcoef_bytes = std::max<size_t>(fall.coef.size() / 2, 1) * cs;
    b->bcoef_bytes = std::max<size_t>(ball.coef.size() / 2, 1) * cs;
    if (!alloc((void **)&b->fdev.ops, fall.ops.size() * sizeof(TOp)) || !alloc(&b->fdev.coef, b->fcoef_bytes) ||
        !alloc((void **)&b->bdev.ops, ball.ops.size() * sizeof(TOp)) || !alloc(&b->bdev.coef, b->bcoef_bytes) ||
        !alloc((void **)&b->bdev.gparams, ball.grad_params.size() * sizeof(int32_t)))
        return cuda_err(e, "cudaMalloc(batch programs)");
    e = cudaMemcpy(b->fdev.ops, fall.ops.data(), fall.ops.size() * sizeof(TOp), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->bdev.ops, ball.ops.data(), ball.ops.size() * sizeof(TOp), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !ball.grad_params.empty())
        e = cudaMemcpy(b->bdev.gparams, ball.grad_params.data(), ball.grad_params.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_err(e, "upload batch programs");
    e = cudaMallocHost(&b->coef_host, b->fcoef_bytes + b->bcoef_bytes);
    if (e != cudaSuccess) return cuda_err(e, "cudaMallocHost(coefficients)");
    fill_coefficients(b);
    if (!b->psi.empty()) return QK_OK;
    // states, outputs
    b->psi.assign(b->ncirc, nullptr);
    b->lam.assign(b->ncirc, nullptr);
    for (int c = 0; c < b->ncirc; ++c)
        if (!alloc(&b->psi[c], cs << b->n[c]) || !alloc(&b->lam[c], cs << b->n[c])) return cuda_err(e, "cudaMalloc(batch states)");
    const size_t nout = b->nparams + 2 * b->ncirc;
    if (!alloc((void **)&b->d_out, nout * sizeof(double))) return cuda_err(e, "cudaMalloc(batch outputs)");
    e = cudaMallocHost((void **)&b->h_out, nout * sizeof(double));
    if (e != cudaSuccess) return cuda_err(e, "cudaMallocHost(outputs)");
    return QK_OK;
}

}  // namespace qk

// Hamiltonians and block tables (kept from creation; independent of plans).
struct qk_batch_host_terms {
    std::vector<BatchTerm> terms;
    std::vector<int> term0, nterm;
};

namespace qk {

static int upload_elem_tables(qk_batch *b, const qk_batch_host_terms &ht) {
    const size_t cs = b->dtype == QK_C128 ? 16 : 8;
    (void)cs;
    std::vector<BatchState> sts(b->ncirc);
    std::vector<int> bc;
    std::vector<uint32_t> bf;
    for (int c = 0; c < b->ncirc; ++c) {
        sts[c].psi = b->psi[c];
        sts[c].lam = b->lam[c];
        sts[c].namp = 1ull << b->n[c];
        sts[c].term0 = ht.term0[c];
        sts[c].nterm = ht.nterm[c];
        sts[c].expval = b->d_out + b->nparams + c;
        sts[c].drift = b->d_out + b->nparams + b->ncirc + c;
        const uint64_t nb = (sts[c].namp + kBatchChunk - 1) / kBatchChunk;
        for (uint64_t k = 0; k < nb; ++k) {
            bc.push_back(c);
            bf.push_back((uint32_t)k);
        }
    }
    b->nblk = (int)bc.size();
    cudaError_t e = cudaMalloc(&b->d_states, sts.size() * sizeof(BatchState));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_terms, std::max<size_t>(1, ht.terms.size()) * sizeof(BatchTerm));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_blk_circ, bc.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_blk_first, bf.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_states, sts.data(), sts.size() * sizeof(BatchState), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !ht.terms.empty())
        e = cudaMemcpy(b->d_terms, ht.terms.data(), ht.terms.size() * sizeof(BatchTerm), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_blk_circ, bc.data(), bc.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(b->d_blk_first, bf.data(), bf.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? QK_OK : cuda_err(e, "batch tables");
}

static int capture(qk_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_err(e, "cudaStreamBeginCapture");
    int rc = b->dtype == QK_C128 ? enqueue<double2>(b) : enqueue<float2>(b);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_err(e, "cudaStreamEndCapture");
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    return e == cudaSuccess ? QK_OK : cuda_err(e, "cudaGraphInstantiate");
}

}  // namespace qk

namespace {

int full_prepare(qk_batch *b, const qk_batch_host_terms &ht) {
    const bool first = b->psi.empty();
    int rc = prepare(b);
    if (!rc) rc = b->dtype == QK_C128 ? build_tables<double2>(b) : build_tables<float2>(b);
    if (!rc && first) rc = upload_elem_tables(b, ht);
    if (!rc) rc = capture(b);
    return rc;
}

float time_graph(qk_batch *b, int reps) {
    cudaEvent_t a, z;
    cudaEventCreate(&a);
    cudaEventCreate(&z);
    cudaGraphLaunch(b->exec, b->stream);  // warm-up
    cudaEventRecord(a, b->stream);
    for (int i = 0; i < reps; ++i) cudaGraphLaunch(b->exec, b->stream);
    cudaEventRecord(z, b->stream);
    float ms = -1;
    if (cudaEventSynchronize(z) == cudaSuccess) cudaEventElapsedTime(&ms, a, z);
    cudaEventDestroy(a);
    cudaEventDestroy(z);
    return ms / reps;
}

}  // namespace

struct qk_batch_full : qk_batch {
    qk_batch_host_terms ht;
};

extern "C" {

int qk_batch_create(int ncirc, const int32_t *nqubits, const qk_gate *gates, const size_t *gate_counts,
                    const int32_t *param_index, const size_t *param_counts, const qk_pauli_term *terms,
                    const size_t *term_counts, const qk_batch_opts *opts, qk_batch **out) {
    if (!out || ncirc <= 0 || !nqubits || !gates || !gate_counts || !param_counts || !term_counts || (!terms))
        return fail(QK_ERR_ARG, "null argument");
    auto *b = new qk_batch_full();
    b->ncirc = ncirc;
    b->dtype = opts ? opts->dtype : QK_C64;
    if (b->dtype != QK_C128 && b->dtype != QK_C64) {
        delete b;
        return fail(QK_ERR_ARG, "unknown dtype");
    }
    size_t g0 = 0, t0 = 0;
    int nmin = 64;
    for (int c = 0; c < ncirc; ++c) {
        if (nqubits[c] < 1 || nqubits[c] > 30) {
            delete b;
            return fail(QK_ERR_ARG, "circuit %d: %d qubits (1..30)", c, nqubits[c]);
        }
        nmin = std::min(nmin, (int)nqubits[c]);
        b->n.push_back(nqubits[c]);
        b->gates.emplace_back(gates + g0, gates + g0 + gate_counts[c]);
        b->pidx.emplace_back(gate_counts[c], -1);
        if (param_index)
            for (size_t i = 0; i < gate_counts[c]; ++i) b->pidx.back()[i] = param_index[g0 + i];
        b->poff.push_back(b->nparams);
        b->nparams += param_counts[c];
        for (size_t i = 0; i < gate_counts[c]; ++i)
            if (b->pidx.back()[i] >= (int32_t)param_counts[c]) {
                const int bad = b->pidx.back()[i];
                delete b;
                return fail(QK_ERR_ARG, "circuit %d gate %zu: parameter %d >= %zu", c, i, bad, param_counts[c]);
            }
        b->ht.term0.push_back((int)b->ht.terms.size());
        b->ht.nterm.push_back((int)term_counts[c]);
        for (size_t t = 0; t < term_counts[c]; ++t) {
            const qk_pauli_term &pt = terms[t0 + t];
            if ((pt.x_mask | pt.z_mask) >> nqubits[c]) {
                delete b;
                return fail(QK_ERR_QUBIT, "circuit %d term %zu acts beyond %d qubits", c, t, nqubits[c]);
            }
            b->ht.terms.push_back({pt.coeff, pt.x_mask, pt.z_mask, __builtin_popcountll(pt.x_mask & pt.z_mask) & 3});
        }
        g0 += gate_counts[c];
        t0 += term_counts[c];
    }
    b->fo = default_plan_options(b->dtype, nmin);
    b->bo = default_adjoint_options(b->dtype, nmin);
    // one kernel instance for all circuits: programs without real-op forms
    b->fo.plain_ops = b->bo.plain_ops = 1;
    if (b->dtype == QK_C64) {
        // the batch's many small states: 1024-amplitude adjoint tiles with 8
        // amplitudes a thread (256 circuits of 14-22 qubits: 261 ms against
        // 310 ms with the single-circuit default of 2048 and 16)
        b->bo.tile_bits = std::min(10, nmin);
        b->bo.reg_bits = std::min(3, b->bo.tile_bits);
    }
    if (opts && opts->tile_bits) b->fo.tile_bits = std::min(opts->tile_bits, nmin);
    if (opts && opts->reg_bits) b->fo.reg_bits = opts->reg_bits;
    if (opts && opts->adj_tile_bits) b->bo.tile_bits = std::min(opts->adj_tile_bits, nmin);
    if (opts && opts->adj_reg_bits) b->bo.reg_bits = opts->adj_reg_bits;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return cuda_err(e, "cudaStreamCreate");
    }
    int rc = QK_OK;
    if (opts && opts->autotune) {
        // try tile shapes on the real batch, keep the fastest forward and adjoint
        struct Cand { int T, r; };
        const std::vector<Cand> fc = b->dtype == QK_C64 ? std::vector<Cand>{{11, 4}, {12, 3}, {12, 4}, {13, 4}}
                                                        : std::vector<Cand>{{11, 4}, {12, 3}, {11, 3}};
        const std::vector<Cand> bc = b->dtype == QK_C64 ? std::vector<Cand>{{10, 3}, {11, 3}, {12, 3}}
                                                        : std::vector<Cand>{{11, 3}, {11, 2}, {10, 2}};
        float best = 1e30f;
        PlanOptions bf = b->fo, bb = b->bo;
        for (const auto &f : fc)
            for (const auto &k : bc) {
                if (f.T > nmin || k.T > nmin) continue;
                b->fo.tile_bits = f.T;
                b->fo.reg_bits = f.r;
                b->bo.tile_bits = k.T;
                b->bo.reg_bits = k.r;
                if (full_prepare(b, b->ht)) continue;
                const float ms = time_graph(b, 2);
                if (ms > 0 && ms < best) {
                    best = ms;
                    bf = b->fo;
                    bb = b->bo;
                }
            }
        b->fo = bf;
        b->bo = bb;
    }
    rc = full_prepare(b, b->ht);
    if (rc) {
        delete b;
        return rc;
    }
    *out = b;
    return QK_OK;
}

int qk_batch_run(qk_batch *b, double *expvals, double *grads, double *drift) {
    if (!b) return fail(QK_ERR_ARG, "null batch");
    cudaError_t e = cudaSuccess;
    if (!b->ev0) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess && !b->ev1) e = cudaEventCreate(&b->ev1);
    if (e == cudaSuccess) e = cudaEventRecord(b->ev0, b->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(b->exec, b->stream);
    if (e == cudaSuccess) e = cudaEventRecord(b->ev1, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_err(e, "batch run");
    float ms = 0;
    b->last_ms = cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess ? ms : -1.0;
    if (grads) std::memcpy(grads, b->h_out, b->nparams * sizeof(double));
    if (expvals) std::memcpy(expvals, b->h_out + b->nparams, b->ncirc * sizeof(double));
    if (drift)
        for (int c = 0; c < b->ncirc; ++c) drift[c] = std::sqrt(std::max(0.0, b->h_out[b->nparams + b->ncirc + c]));
    return QK_OK;
}

int qk_batch_set_params(qk_batch *b, const double *params) {
    if (!b || (!params && b->nparams)) return fail(QK_ERR_ARG, "null argument");
    for (int c = 0; c < b->ncirc; ++c)
        for (size_t i = 0; i < b->gates[c].size(); ++i)
            if (b->pidx[c][i] >= 0) b->gates[c][i].param = params[b->poff[c] + b->pidx[c][i]];
    // same gate structure -> same plans; only the coefficients change
    std::vector<size_t> fsz(b->ncirc), bsz(b->ncirc);
    for (int c = 0; c < b->ncirc; ++c) {
        fsz[c] = b->fplan[c].coef.size();
        bsz[c] = b->bplan[c].coef.size();
    }
    int rc = build_all_plans(b);
    if (rc) return rc;
    for (int c = 0; c < b->ncirc; ++c)
        if (b->fplan[c].coef.size() != fsz[c] || b->bplan[c].coef.size() != bsz[c])
            return fail(QK_ERR_ARG, "circuit %d: new parameters changed the plan", c);
    // the graph reads the pinned buffer when it runs: wait for a run in flight
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_err(e, "batch sync");
    fill_coefficients(b);
    return QK_OK;
}

int qk_batch_timing(const qk_batch *b, double *device_ms, double *alg_bytes) {
    if (!b) return fail(QK_ERR_ARG, "null batch");
    if (device_ms) *device_ms = b->last_ms;
    if (alg_bytes) *alg_bytes = b->alg_bytes;
    return QK_OK;
}

int qk_batch_stats(const qk_batch *b, int *steps, int *launches, int *tile_bits, int *reg_bits, int *adj_tile_bits,
                   int *adj_reg_bits) {
    if (!b) return fail(QK_ERR_ARG, "null batch");
    if (steps) *steps = (int)b->steps.size();
    if (launches) *launches = (int)b->launches;
    if (tile_bits) *tile_bits = b->fo.tile_bits;
    if (reg_bits) *reg_bits = b->fo.reg_bits;
    if (adj_tile_bits) *adj_tile_bits = b->bo.tile_bits;
    if (adj_reg_bits) *adj_reg_bits = b->bo.reg_bits;
    return QK_OK;
}

void qk_batch_destroy(qk_batch *b) { delete static_cast<qk_batch_full *>(b); }

}  // extern "C"
