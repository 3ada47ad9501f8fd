// States larger than HBM: the state in pinned host memory, the gates on the
// GPU, chunk by chunk (the GPU form of the reference's IO runner,
// src/IO_Runner.cpp:309-488, which keeps the state in files and runs each
// 2^chunk_qbit piece on the host cores).
//
// Layout: host amplitude k at index k, qubit q = bit q (the in-memory layout,
// never permuted).  A circuit is cut into segments.  Each segment has a set
// of L "local" qubits that holds every qubit its gates touch; a sweep of the
// segment visits the 2^(n-L) chunks -- the amplitudes that share one value
// of the n - L other bits -- and for each one gathers its 2^L amplitudes into
// a device buffer (local bit i = the i-th lowest local qubit), runs the
// segment's fused plan on it, and scatters it back to the same host places.
// The reference moves amplitudes between files to bring a qubit into its
// chunk (VSWAP); here a qubit joins the local set by a change of the gather
// addresses, so a segment costs one read and one write of the state over the
// host link however many qubits it exchanges.
//
// Gather: the lowest r bits of the local set are the state's bits 0..r-1, so
// each chunk is 2^(L-r) runs of 2^r contiguous amplitudes; the next block of
// consecutive local bits above them becomes the rows of one
// cudaMemcpy2DAsync, any further local bits a loop of such copies.
//
// Pipeline: three device buffers and three streams.  Chunk c is copied in on
// the copy-in stream (after the buffer's previous chunk has been copied
// out), run on the compute stream, copied out on the copy-out stream; events
// order the three.  A segment's copy-ins wait for the previous segment's
// last copy-out, since two segments' chunks overlap in host memory.
//
// Segments (host, greedy): a segment starts from the qubits of the first
// pending gate and grows, one qubit at a time, by the qubit that lets the
// most pending gates join (a gate joins when all its qubits are local and
// no earlier pending gate that stays behind shares a qubit with it), ties
// to the lowest qubit, which keeps the gather runs long; when no qubit adds
// a gate, the lowest free qubit is taken.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "qk_devplan.h"
#include "qk_internal.h"

namespace qk {
int run_forward_plan(void *state, const HostPlan &hp, const DevPlan &dp, cudaStream_t st);
int upload_host_plan(const HostPlan &hp, DevPlan &dp, cudaStream_t st);

namespace {

int cuda_e(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation) (void)cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? QK_ERR_OOM : QK_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

uint64_t gate_mask(const qk_gate &g) {
    uint64_t m = 0;
    for (int i = 0; i < g.nq; ++i) m |= 1ull << g.q[i];
    return m;
}

int popc(uint64_t x) { return __builtin_popcountll(x); }

// Gates (indices into `pend`) that join a segment with local set `mask`.
size_t count_joining(const std::vector<uint64_t> &masks, const std::vector<size_t> &pend, uint64_t mask) {
    uint64_t blocked = 0;
    size_t k = 0;
    for (size_t i : pend) {
        const uint64_t m = masks[i];
        if ((m & ~mask) == 0 && (m & blocked) == 0) ++k;
        else blocked |= m;
    }
    return k;
}

}  // namespace

struct OocSegment {
    uint64_t local = 0;             // local qubits
    std::vector<size_t> gates;      // indices into the circuit, in execution order
};

int ooc_segments(const qk_gate *gates, size_t ng, int n, int L, std::vector<OocSegment> &segs) {
    segs.clear();
    std::vector<uint64_t> masks(ng);
    for (size_t i = 0; i < ng; ++i) {
        masks[i] = gate_mask(gates[i]);
        if (popc(masks[i]) > L) return fail(QK_ERR_ARG, "gate %zu touches more qubits than a chunk holds", i);
        for (int k = 0; k < gates[i].nq; ++k)
            if (gates[i].q[k] < 0 || gates[i].q[k] >= n)
                return fail(QK_ERR_QUBIT, "gate %zu: qubit %d outside a %d-qubit state", i, gates[i].q[k], n);
    }
    const uint64_t all = n >= 64 ? ~0ull : (1ull << n) - 1;
    std::vector<size_t> pend(ng);
    for (size_t i = 0; i < ng; ++i) pend[i] = i;
    while (!pend.empty()) {
        uint64_t mask = masks[pend[0]];
        while (popc(mask) < L) {
            const size_t base = count_joining(masks, pend, mask);
            int best = -1;
            size_t best_k = base;
            for (int q = 0; q < n; ++q) {
                if (mask >> q & 1) continue;
                const size_t k = count_joining(masks, pend, mask | 1ull << q);
                if (k > best_k) { best_k = k; best = q; }
            }
            if (best < 0) best = __builtin_ctzll(all & ~mask);   // lowest free qubit
            mask |= 1ull << best;
        }
        OocSegment s;
        s.local = mask;
        std::vector<size_t> rest;
        uint64_t blocked = 0;
        for (size_t i : pend) {
            const uint64_t m = masks[i];
            if ((m & ~mask) == 0 && (m & blocked) == 0) s.gates.push_back(i);
            else { blocked |= m; rest.push_back(i); }
        }
        segs.push_back(std::move(s));
        pend.swap(rest);
    }
    return QK_OK;
}

}  // namespace qk

using namespace qk;

struct qk_hsv {
    int n = 0, L = 0, dtype = QK_C128;
    size_t es = 16;                  // bytes per amplitude
    void *host = nullptr;            // pinned, 2^n amplitudes
    void *dbuf[3] = {nullptr, nullptr, nullptr};
    cudaStream_t s_in = nullptr, s_run = nullptr, s_out = nullptr;
    cudaEvent_t in_done[3] = {}, run_done[3] = {}, out_done[3] = {};
    cudaEvent_t t0 = nullptr, t1 = nullptr, seg_done = nullptr;
    double last_ms = 0, last_bytes = 0;
    int last_segments = 0;
    size_t max_pitch = 0;            // cudaDevAttrMaxPitch
    std::vector<DevPlan> plans;

    ~qk_hsv() {
        if (s_in) cudaStreamSynchronize(s_in);
        if (s_run) cudaStreamSynchronize(s_run);
        if (s_out) cudaStreamSynchronize(s_out);
        for (auto &p : plans) p.release();
        for (int b = 0; b < 3; ++b) {
            if (dbuf[b]) cudaFree(dbuf[b]);
            if (in_done[b]) cudaEventDestroy(in_done[b]);
            if (run_done[b]) cudaEventDestroy(run_done[b]);
            if (out_done[b]) cudaEventDestroy(out_done[b]);
        }
        for (cudaEvent_t e : {t0, t1, seg_done})
            if (e) cudaEventDestroy(e);
        for (cudaStream_t s : {s_in, s_run, s_out})
            if (s) cudaStreamDestroy(s);
        if (host) cudaFreeHost(host);
    }
};

namespace {

uint64_t deposit(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    while (mask) {
        const uint64_t low = mask & (0 - mask);
        if (v & 1) r |= low;
        v >>= 1;
        mask ^= low;
    }
    return r;
}

// Copy one chunk between host and device.  local: the local bit set (L
// bits, the lowest r of them the state's bits 0..r-1); base: host index of
// the chunk's first amplitude (its outer bits).  to_device: gather, else
// scatter.
int copy_chunk(qk_hsv *h, void *dev, uint64_t local, uint64_t base, bool to_device, cudaStream_t st) {
    const size_t es = h->es;
    int r = 0;
    while (r < 64 && (local >> r & 1)) ++r;
    const uint64_t upper = local & ~((r >= 64 ? ~0ull : (1ull << r) - 1));
    // rows: the next block of consecutive local bits above bit r
    int r0 = upper ? __builtin_ctzll(upper) : 0, hrows = 0;
    while (upper && (upper >> (r0 + hrows) & 1)) ++hrows;
    const uint64_t rest = upper & ~(((1ull << hrows) - 1) << r0);
    const size_t width = es << r;
    const size_t spitch = es << r0;             // host stride of one row
    const size_t rows = upper ? (size_t)1 << hrows : 1;
    const size_t nrest = (size_t)1 << popc(rest);
    if (nrest > 65536) return fail(QK_ERR_UNSUPPORTED, "chunk gather of %zu copies: too fragmented", nrest);
    unsigned char *hb = static_cast<unsigned char *>(h->host);
    unsigned char *db = static_cast<unsigned char *>(dev);
    // a 2D copy takes pitches up to the device's limit; past it (rows of
    // GiB), one plain copy per row
    const bool two_d = rows > 1 && spitch <= h->max_pitch && width <= h->max_pitch;
    const size_t per = two_d ? 1 : rows;
    for (size_t j = 0; j < nrest; ++j) {
        const uint64_t hoff = base | deposit(j, rest);
        const size_t doff = (j * rows) << r;     // device index of the first row
        for (size_t t = 0; t < per; ++t) {
            unsigned char *hp = hb + (hoff + ((uint64_t)t << r0)) * es, *dp = db + (doff + (t << r)) * es;
            cudaError_t e;
            if (to_device)
                e = two_d ? cudaMemcpy2DAsync(dp, width, hp, spitch, width, rows, cudaMemcpyHostToDevice, st)
                          : cudaMemcpyAsync(dp, hp, width, cudaMemcpyHostToDevice, st);
            else
                e = two_d ? cudaMemcpy2DAsync(hp, spitch, dp, width, width, rows, cudaMemcpyDeviceToHost, st)
                          : cudaMemcpyAsync(hp, dp, width, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return cuda_e(e, to_device ? "chunk gather" : "chunk scatter");
        }
    }
    return QK_OK;
}

}  // namespace

extern "C" {

int qk_hsv_create(int nqubits, int chunk_qubits, int dtype, qk_hsv **out) {
    if (!out) return fail(QK_ERR_ARG, "null output");
    *out = nullptr;
    if (dtype != QK_C128 && dtype != QK_C64) return fail(QK_ERR_ARG, "unknown dtype %d", dtype);
    if (nqubits < 2 || nqubits > 40) return fail(QK_ERR_ARG, "nqubits must be in [2, 40], got %d", nqubits);
    if (chunk_qubits < 1 || chunk_qubits > nqubits)
        return fail(QK_ERR_ARG, "chunk_qubits must be in [1, %d], got %d", nqubits, chunk_qubits);
    qk_hsv *h = new qk_hsv();
    h->n = nqubits;
    h->L = chunk_qubits;
    h->dtype = dtype;
    h->es = dtype == QK_C128 ? 16 : 8;
    cudaError_t e = cudaHostAlloc(&h->host, h->es << nqubits, cudaHostAllocPortable);
    for (int b = 0; e == cudaSuccess && b < 3; ++b) e = cudaMalloc(&h->dbuf[b], h->es << chunk_qubits);
    for (cudaStream_t *s : {&h->s_in, &h->s_run, &h->s_out})
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
    for (int b = 0; e == cudaSuccess && b < 3; ++b) {
        e = cudaEventCreateWithFlags(&h->in_done[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->run_done[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->out_done[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreate(&h->t0);
    if (e == cudaSuccess) e = cudaEventCreate(&h->t1);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->seg_done, cudaEventDisableTiming);
    int dev = 0, mp = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&mp, cudaDevAttrMaxPitch, dev);
    h->max_pitch = mp > 0 ? (size_t)mp : 0;
    if (e != cudaSuccess) {
        const int rc = cuda_e(e, "host state / chunk buffers");
        delete h;
        return rc;
    }
    *out = h;
    return qk_hsv_reset(h);
}

int qk_hsv_reset(qk_hsv *h) {
    if (!h) return fail(QK_ERR_ARG, "null state");
    // |0...0>, zeroed by host threads (a large pinned buffer)
    const size_t bytes = h->es << h->n;
    const unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            const size_t a = bytes * t / nt, b = bytes * (t + 1) / nt;
            std::memset(static_cast<unsigned char *>(h->host) + a, 0, b - a);
        });
    for (auto &x : th) x.join();
    if (h->dtype == QK_C128) static_cast<double *>(h->host)[0] = 1.0;
    else static_cast<float *>(h->host)[0] = 1.0f;
    return QK_OK;
}

void *qk_hsv_data(qk_hsv *h) { return h ? h->host : nullptr; }

int qk_hsv_apply_gates(qk_hsv *h, const qk_gate *gates, size_t ng) {
    if (!h || (!gates && ng)) return fail(QK_ERR_ARG, "null argument");
    std::vector<OocSegment> segs;
    int rc = ooc_segments(gates, ng, h->n, h->L, segs);
    if (rc) return rc;
    // plans: each segment's gates on its local bits (local bit i = i-th lowest local qubit)
    std::vector<HostPlan> hps(segs.size());
    const PlanOptions po = default_plan_options(h->dtype, h->L);
    for (size_t s = 0; s < segs.size(); ++s) {
        int rank[64];
        for (int q = 0, k = 0; q < h->n; ++q) rank[q] = (segs[s].local >> q & 1) ? k++ : -1;
        std::vector<qk_gate> g;
        g.reserve(segs[s].gates.size());
        for (size_t i : segs[s].gates) {
            qk_gate x = gates[i];
            for (int k = 0; k < x.nq; ++k) x.q[k] = rank[x.q[k]];
            g.push_back(x);
        }
        rc = build_plan(g.data(), g.size(), h->L, po, hps[s]);
        if (rc) return rc;
    }
    if (h->plans.size() < segs.size()) h->plans.resize(segs.size());
    for (size_t s = 0; s < segs.size(); ++s) {
        rc = upload_host_plan(hps[s], h->plans[s], h->s_run);
        if (rc) return rc;
    }
    const uint64_t all = h->n >= 64 ? ~0ull : (1ull << h->n) - 1;
    const uint64_t nchunks = 1ull << (h->n - h->L);
    cudaError_t e = cudaEventRecord(h->t0, h->s_in);
    if (e != cudaSuccess) return cuda_e(e, "timing");
    uint64_t k = 0;   // chunk counter over the whole circuit (buffer k % 3)
    for (size_t s = 0; s < segs.size(); ++s) {
        const uint64_t outer = all & ~segs[s].local;
        if (s > 0) {   // this segment's gathers overlap the last segment's scatters
            e = cudaEventRecord(h->seg_done, h->s_out);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(h->s_in, h->seg_done, 0);
            if (e != cudaSuccess) return cuda_e(e, "segment order");
        }
        for (uint64_t c = 0; c < nchunks; ++c, ++k) {
            const int b = (int)(k % 3);
            const uint64_t base = deposit(c, outer);
            if (k >= 3) {   // the buffer's previous chunk has left the device
                e = cudaStreamWaitEvent(h->s_in, h->out_done[b], 0);
                if (e != cudaSuccess) return cuda_e(e, "buffer reuse");
            }
            rc = copy_chunk(h, h->dbuf[b], segs[s].local, base, true, h->s_in);
            if (rc) return rc;
            e = cudaEventRecord(h->in_done[b], h->s_in);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(h->s_run, h->in_done[b], 0);
            if (e != cudaSuccess) return cuda_e(e, "copy-in order");
            rc = run_forward_plan(h->dbuf[b], hps[s], h->plans[s], h->s_run);
            if (rc) return rc;
            e = cudaEventRecord(h->run_done[b], h->s_run);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(h->s_out, h->run_done[b], 0);
            if (e != cudaSuccess) return cuda_e(e, "compute order");
            rc = copy_chunk(h, h->dbuf[b], segs[s].local, base, false, h->s_out);
            if (rc) return rc;
            e = cudaEventRecord(h->out_done[b], h->s_out);
            if (e != cudaSuccess) return cuda_e(e, "copy-out order");
        }
    }
    e = cudaEventRecord(h->t1, h->s_out);
    if (e == cudaSuccess) e = cudaEventSynchronize(h->t1);
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->t0, h->t1);
    if (e != cudaSuccess) return cuda_e(e, "out-of-core sweep");
    h->last_ms = ms;
    h->last_segments = (int)segs.size();
    h->last_bytes = 2.0 * (double)(h->es << h->n) * (double)segs.size();
    return QK_OK;
}

int qk_hsv_stats(const qk_hsv *h, int *segments, double *device_ms, double *link_bytes) {
    if (!h) return fail(QK_ERR_ARG, "null state");
    if (segments) *segments = h->last_segments;
    if (device_ms) *device_ms = h->last_ms;
    if (link_bytes) *link_bytes = h->last_bytes;
    return QK_OK;
}

int qk_ooc_segments(const qk_gate *gates, size_t ng, int nqubits, int chunk_qubits, uint64_t *local_masks,
                    int32_t *segment_sizes, int32_t *order, size_t cap, size_t *nsegments) {
    if ((!gates && ng) || !nsegments) return fail(QK_ERR_ARG, "null argument");
    if (nqubits < 1 || nqubits > 63 || chunk_qubits < 1 || chunk_qubits > nqubits)
        return fail(QK_ERR_ARG, "bad sizes");
    std::vector<OocSegment> segs;
    int rc = ooc_segments(gates, ng, nqubits, chunk_qubits, segs);
    if (rc) return rc;
    *nsegments = segs.size();
    if (segs.size() > cap) return QK_OK;   // sizes only
    size_t k = 0;
    for (size_t s = 0; s < segs.size(); ++s) {
        if (local_masks) local_masks[s] = segs[s].local;
        if (segment_sizes) segment_sizes[s] = (int32_t)segs[s].gates.size();
        for (size_t i : segs[s].gates)
            if (order) order[k++] = (int32_t)i;
    }
    return QK_OK;
}

void qk_hsv_destroy(qk_hsv *h) { delete h; }

}  // extern "C"
