// Contexts and asynchronous host-buffer batches of banded SW.
//
// A context owns, on one device, 1 to 8 slots; each slot has a stream, an
// event, a pinned staging buffer and a device arena.  gmf_batch_submit packs
// the caller's host arrays into the slot's staging buffer (every array at a
// 256-byte boundary), copies them to the arena in one host-to-device copy,
// runs gmf_banded_sw on the slot's stream with the arena as inputs, outputs
// and workspace, and copies the fixed-size outputs back into staging in one
// device-to-host copy.  Completion (gmf_batch_poll / gmf_batch_wait) copies
// the CIGAR words the batch produced and hands everything to the caller's
// host buffers.  With several slots, the copies of one batch overlap the
// kernels of another.
//
// Memory: every slot may hold up to memory_budget / slots bytes of device
// memory; an arena grows (never shrinks) when a batch needs more.  Growing
// frees the old arena, which waits for the device, so steady traffic of
// similar batches allocates only during its first batches.

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_set>
#include <vector>

#include "gmf_common.cuh"

namespace {

constexpr int CTX_MAX_SLOTS = 8;
constexpr size_t AL = 256;
inline size_t al(size_t x) { return (x + AL - 1) & ~(AL - 1); }

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    char* host = nullptr;  // pinned staging
    size_t host_bytes = 0;
    char* dev = nullptr;   // device arena
    size_t dev_bytes = 0;
    int64_t ticket = -1;   // batch in flight, -1 when free
    // the batch in flight
    int32_t n = 0;
    bool tb = false;
    gmf_host_sw_results out{};
    size_t out_at = 0;     // offset of the fixed-size outputs (arena and staging alike)
    size_t cigar_at = 0;   // offset of the CIGAR words in the arena
    int64_t cigar_cap = 0;
};

// Offsets of one batch's pieces in a slot (same layout in staging and arena).
struct Layout {
    size_t q, qo, t, to, hb, off, order, go;  // inputs
    size_t in_end;
    size_t score, qe, te, qs, ts, counts, cstart, clen, used, err;  // outputs
    size_t out_end;
    size_t cigar, ws, ws_bytes, total;
};

}  // namespace

struct gmf_ctx {
    int device = 0;
    size_t budget = 0;
    std::mutex mu;
    Slot slots[CTX_MAX_SLOTS];
    int n_slots = 0;
    int64_t next_ticket = 1;
    int next_slot = 0;
    std::unordered_set<int64_t> completed;  // finished by a submit that needed the slot
};

namespace {

int finalize(Slot& s) {
    GMF_CUDA_TRY(cudaEventSynchronize(s.done));
    const int32_t n = s.n;
    const char* h = s.host + s.out_at;
    // staging holds the outputs back to back in the order of Layout
    size_t o = 0;
    auto take = [&](void* dst, size_t bytes) {
        if (dst && bytes) std::memcpy(dst, h + o, bytes);
        o += al(bytes);
    };
    take(s.out.score, 4 * (size_t)n);
    take(s.out.query_end, 4 * (size_t)n);
    take(s.out.target_end, 4 * (size_t)n);
    take(s.tb ? s.out.query_start : nullptr, 4 * (size_t)n);
    take(s.tb ? s.out.target_start : nullptr, 4 * (size_t)n);
    take(s.tb ? s.out.op_counts : nullptr, 16 * (size_t)n);
    take(s.tb ? s.out.cigar_start : nullptr, 8 * (size_t)n);
    take(s.tb ? s.out.cigar_len : nullptr, 4 * (size_t)n);
    unsigned long long used = 0;
    std::memcpy(&used, h + o, sizeof(used));
    o += al(8);
    int32_t err = 0;
    std::memcpy(&err, h + o, sizeof(err));
    if (s.out.error_flags) *s.out.error_flags = err;
    const long long words = std::min<long long>((long long)used, s.cigar_cap);
    if (s.out.cigar_used) *s.out.cigar_used = (int64_t)words;
    if (s.tb && words > 0) {  // on the slot's own stream: other slots' work goes on
        GMF_CUDA_TRY(cudaMemcpyAsync(s.out.cigar, s.dev + s.cigar_at, 4 * (size_t)words, cudaMemcpyDeviceToHost,
                                     s.stream));
        GMF_CUDA_TRY(cudaStreamSynchronize(s.stream));
    }
    s.ticket = -1;
    return GMF_OK;
}

// memcpy split over host threads for large copies (one thread copies a few
// GB/s; the staging of a large batch is hundreds of MB).
void par_memcpy(char* dst, const char* src, size_t n) {
    constexpr size_t PIECE = 16u << 20;
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const size_t parts = std::min<size_t>(hw, (n + PIECE - 1) / PIECE);
    if (parts <= 1) {
        if (n) std::memcpy(dst, src, n);
        return;
    }
    const size_t step = (n + parts - 1) / parts;
    std::vector<std::thread> ts;
    ts.reserve(parts - 1);
    for (size_t i = 1; i < parts; ++i) {
        const size_t a = i * step, b = std::min(n, a + step);
        if (a >= b) continue;
        try {
            ts.emplace_back([=] { std::memcpy(dst + a, src + a, b - a); });
        } catch (...) {  // no thread to spare: copy this piece here
            std::memcpy(dst + a, src + a, b - a);
        }
    }
    std::memcpy(dst, src, std::min(n, step));
    for (auto& t : ts) t.join();
}

int check_host(const gmf_host_pairs* p, const gmf_sw_params* prm, const gmf_host_sw_results* r) {
    if (!p || !prm || !r || p->n_pairs < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (!r->score || !r->query_end || !r->target_end || !r->error_flags || !r->cigar_used)
        return GMF_ERR_INVALID_ARGUMENT;
    if (r->cigar && (!r->query_start || !r->target_start || !r->cigar_start || !r->cigar_len ||
                     r->cigar_capacity < 0))
        return GMF_ERR_INVALID_ARGUMENT;
    if (p->n_pairs == 0) return GMF_OK;
    if (!p->query_off || !p->target_off || !p->half_band || !p->band_offset) return GMF_ERR_INVALID_ARGUMENT;
    if (p->query_off[0] != 0 || p->target_off[0] != 0) return GMF_ERR_INVALID_ARGUMENT;
    for (int32_t i = 0; i < p->n_pairs; ++i) {
        if (p->query_off[i + 1] < p->query_off[i] || p->target_off[i + 1] < p->target_off[i])
            return GMF_ERR_INVALID_ARGUMENT;
        if (p->query_off[i + 1] - p->query_off[i] > GMF_MAX_SEQ_LEN ||
            p->target_off[i + 1] - p->target_off[i] > GMF_MAX_SEQ_LEN)
            return GMF_ERR_LIMIT;
        if (p->half_band[i] < 0 || p->half_band[i] > GMF_MAX_HALF_BAND) return GMF_ERR_LIMIT;
    }
    if ((p->query_off[p->n_pairs] > 0 && !p->query) || (p->target_off[p->n_pairs] > 0 && !p->target))
        return GMF_ERR_INVALID_ARGUMENT;
    if (p->xdrop_group_off) {
        if (p->n_xdrop_groups < 0 || p->xdrop_group_off[0] != 0 ||
            p->xdrop_group_off[p->n_xdrop_groups] != p->n_pairs)
            return GMF_ERR_INVALID_ARGUMENT;
        for (int32_t g = 0; g < p->n_xdrop_groups; ++g)
            if (p->xdrop_group_off[g + 1] < p->xdrop_group_off[g]) return GMF_ERR_INVALID_ARGUMENT;
    }
    return GMF_OK;
}

// Longest-first processing order by DP area, bucketed by powers of two (a
// scheduling hint only: results never depend on it).
void lpt_order(const gmf_host_pairs* p, int32_t* order) {
    const int32_t n = p->n_pairs;
    std::vector<int32_t> count(65, 0);
    std::vector<uint8_t> bucket((size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        const unsigned long long area =
            (unsigned long long)(p->query_off[i + 1] - p->query_off[i]) * (2ull * p->half_band[i] + 1) + 1;
        const int b = 63 - __builtin_clzll(area);
        bucket[(size_t)i] = (uint8_t)b;
        ++count[64 - b];
    }
    std::vector<int32_t> start(65, 0);
    for (int b = 1; b < 65; ++b) start[b] = start[b - 1] + count[b - 1];
    for (int32_t i = 0; i < n; ++i) order[start[64 - bucket[(size_t)i]]++] = i;
}

}  // namespace

static int ctx_destroy(gmf_ctx* c);

static int ctx_create(int device, int32_t slots, size_t memory_budget, gmf_ctx** out) {
    if (!out || slots < 1 || slots > CTX_MAX_SLOTS) return GMF_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    GMF_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return GMF_ERR_INVALID_ARGUMENT;
    GMF_CUDA_TRY(cudaSetDevice(device));
    gmf_ctx* c = new (std::nothrow) gmf_ctx();
    if (!c) return GMF_ERR_HOST;
    c->device = device;
    c->budget = memory_budget;
    c->n_slots = slots;
    for (int i = 0; i < slots; ++i) {
        Slot& s = c->slots[i];
        if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
            ctx_destroy(c);
            return GMF_ERR_CUDA;
        }
    }
    *out = c;
    return GMF_OK;
}

static int ctx_destroy(gmf_ctx* c) {
    if (!c) return GMF_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    for (Slot& s : c->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        if (s.dev) cudaFree(s.dev);
        if (s.host) cudaFreeHost(s.host);
        if (s.done) cudaEventDestroy(s.done);
        if (s.stream) cudaStreamDestroy(s.stream);
    }
    delete c;
    return GMF_OK;
}

static int batch_submit(gmf_ctx* c, const gmf_host_pairs* p, const gmf_sw_params* prm,
                        const gmf_host_sw_results* r, int64_t* ticket) {
    if (!c || !ticket) return GMF_ERR_INVALID_ARGUMENT;
    GMF_TRY(check_host(p, prm, r));
    std::lock_guard<std::mutex> lock(c->mu);
    GMF_CUDA_TRY(cudaSetDevice(c->device));
    const int32_t n = p->n_pairs;
    const bool tb = r->cigar != nullptr;
    // a slot: the next one in turn, finishing its batch first if it has one
    Slot& s = c->slots[c->next_slot];
    c->next_slot = (c->next_slot + 1) % c->n_slots;
    if (s.ticket >= 0) {
        const int64_t t = s.ticket;
        GMF_TRY(finalize(s));
        c->completed.insert(t);
    }
    // layout
    const long long nq = n ? p->query_off[n] : 0, nt = n ? p->target_off[n] : 0;
    std::vector<int32_t> qlen((size_t)std::max(n, 1)), tlen((size_t)std::max(n, 1));
    for (int32_t i = 0; i < n; ++i) {
        qlen[(size_t)i] = (int32_t)(p->query_off[i + 1] - p->query_off[i]);
        tlen[(size_t)i] = (int32_t)(p->target_off[i + 1] - p->target_off[i]);
    }
    int32_t max_hb = 0;
    for (int32_t i = 0; i < n; ++i) max_hb = std::max(max_hb, p->half_band[i]);
    const long long cap = tb ? std::min<long long>(r->cigar_capacity, nq + nt + n) : 0;
    const int ng = p->xdrop_group_off ? p->n_xdrop_groups : 0;
    Layout L{};
    size_t o = 0;
    auto put = [&](size_t bytes) {
        const size_t at = o;
        o += al(bytes);
        return at;
    };
    L.q = put((size_t)std::max(nq, 1ll));
    L.qo = put(8 * ((size_t)n + 1));
    L.t = put((size_t)std::max(nt, 1ll));
    L.to = put(8 * ((size_t)n + 1));
    L.hb = put(4 * (size_t)n);
    L.off = put(4 * (size_t)n);
    L.order = put(4 * (size_t)n);
    L.go = put(4 * ((size_t)ng + 1));
    L.in_end = o;
    L.score = put(4 * (size_t)n);
    L.qe = put(4 * (size_t)n);
    L.te = put(4 * (size_t)n);
    L.qs = put(4 * (size_t)n);
    L.ts = put(4 * (size_t)n);
    L.counts = put(16 * (size_t)n);
    L.cstart = put(8 * (size_t)n);
    L.clen = put(4 * (size_t)n);
    L.used = put(8);
    L.err = put(4);
    L.out_end = o;
    L.cigar = put(4 * (size_t)std::max(cap, 1ll));
    L.ws_bytes = gmf_banded_sw_workspace_bytes(n, qlen.data(), tlen.data(), p->half_band, tb ? 1 : 0);
    L.ws = put(L.ws_bytes);
    L.total = o;
    const size_t share = c->budget / (size_t)c->n_slots;
    if (c->budget && L.total > share) return GMF_ERR_LIMIT;
    // grow the slot's buffers (its previous batch is finished)
    if (s.dev_bytes < L.total) {
        if (s.dev) GMF_CUDA_TRY(cudaFree(s.dev));
        s.dev = nullptr;
        s.dev_bytes = 0;
        const size_t want = c->budget ? std::min(L.total + L.total / 4, share) : L.total + L.total / 4;
        GMF_CUDA_TRY(cudaMalloc(&s.dev, want));
        s.dev_bytes = want;
    }
    if (s.host_bytes < L.out_end) {
        if (s.host) GMF_CUDA_TRY(cudaFreeHost(s.host));
        s.host = nullptr;
        s.host_bytes = 0;
        const size_t want = L.out_end + L.out_end / 4;
        GMF_CUDA_TRY(cudaHostAlloc(&s.host, want, cudaHostAllocDefault));
        s.host_bytes = want;
    }
    // stage the inputs and copy them over in one piece
    char* h = s.host;
    if (nq) par_memcpy(h + L.q, reinterpret_cast<const char*>(p->query), (size_t)nq);
    std::memcpy(h + L.qo, p->query_off, 8 * ((size_t)n + 1));
    if (nt) par_memcpy(h + L.t, reinterpret_cast<const char*>(p->target), (size_t)nt);
    std::memcpy(h + L.to, p->target_off, 8 * ((size_t)n + 1));
    std::memcpy(h + L.hb, p->half_band, 4 * (size_t)n);
    std::memcpy(h + L.off, p->band_offset, 4 * (size_t)n);
    lpt_order(p, reinterpret_cast<int32_t*>(h + L.order));
    if (ng) std::memcpy(h + L.go, p->xdrop_group_off, 4 * ((size_t)ng + 1));
    GMF_CUDA_TRY(cudaMemcpyAsync(s.dev, h, L.in_end, cudaMemcpyHostToDevice, s.stream));
    // the batched form on the slot's stream
    char* d = s.dev;
    gmf_pairs dp{};
    dp.n_pairs = n;
    dp.query = reinterpret_cast<const int8_t*>(d + L.q);
    dp.query_off = reinterpret_cast<const int64_t*>(d + L.qo);
    dp.target = reinterpret_cast<const int8_t*>(d + L.t);
    dp.target_off = reinterpret_cast<const int64_t*>(d + L.to);
    dp.half_band = reinterpret_cast<const int32_t*>(d + L.hb);
    dp.band_offset = reinterpret_cast<const int32_t*>(d + L.off);
    dp.order = reinterpret_cast<const int32_t*>(d + L.order);
    dp.max_half_band = max_hb;
    dp.xdrop_group_off = ng ? reinterpret_cast<const int32_t*>(d + L.go) : nullptr;
    dp.n_xdrop_groups = ng;
    gmf_sw_results dr{};
    dr.score = reinterpret_cast<int32_t*>(d + L.score);
    dr.query_end = reinterpret_cast<int32_t*>(d + L.qe);
    dr.target_end = reinterpret_cast<int32_t*>(d + L.te);
    dr.query_start = tb ? reinterpret_cast<int32_t*>(d + L.qs) : nullptr;
    dr.target_start = tb ? reinterpret_cast<int32_t*>(d + L.ts) : nullptr;
    dr.op_counts = tb ? reinterpret_cast<int32_t*>(d + L.counts) : nullptr;
    dr.cigar = tb ? reinterpret_cast<uint32_t*>(d + L.cigar) : nullptr;
    dr.cigar_capacity = cap;
    dr.cigar_start = tb ? reinterpret_cast<int64_t*>(d + L.cstart) : nullptr;
    dr.cigar_len = tb ? reinterpret_cast<int32_t*>(d + L.clen) : nullptr;
    dr.cigar_used = reinterpret_cast<unsigned long long*>(d + L.used);
    dr.error_flags = reinterpret_cast<int32_t*>(d + L.err);
    if (n > 0) {
        GMF_TRY(gmf_banded_sw(&dp, prm, &dr, d + L.ws, L.ws_bytes, (gmf_stream_t)s.stream));
    } else {
        GMF_CUDA_TRY(cudaMemsetAsync(d + L.used, 0, 8, s.stream));
        GMF_CUDA_TRY(cudaMemsetAsync(d + L.err, 0, 4, s.stream));
    }
    GMF_CUDA_TRY(cudaMemcpyAsync(h + L.score, d + L.score, L.out_end - L.score, cudaMemcpyDeviceToHost, s.stream));
    GMF_CUDA_TRY(cudaEventRecord(s.done, s.stream));
    s.n = n;
    s.tb = tb;
    s.out = *r;
    s.out_at = L.score;
    s.cigar_at = L.cigar;
    s.cigar_cap = cap;
    s.ticket = c->next_ticket++;
    *ticket = s.ticket;
    return GMF_OK;
}

static int complete(gmf_ctx* c, int64_t ticket, bool block) {
    if (!c) return GMF_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(c->mu);
    auto it = c->completed.find(ticket);
    if (it != c->completed.end()) {
        c->completed.erase(it);
        return GMF_OK;
    }
    GMF_CUDA_TRY(cudaSetDevice(c->device));
    for (Slot& s : c->slots) {
        if (s.ticket != ticket) continue;
        if (!block) {
            const cudaError_t e = cudaEventQuery(s.done);
            if (e == cudaErrorNotReady) return GMF_ERR_NOT_READY;
            if (e != cudaSuccess) return GMF_ERR_CUDA;
        }
        return finalize(s);
    }
    return GMF_ERR_INVALID_ARGUMENT;  // unknown, or already completed
}

// No C++ exception leaves the library: a failed host allocation, thread or
// lock becomes GMF_ERR_HOST.
template <class F>
static int guarded(F&& f) noexcept {
    try {
        return f();
    } catch (...) {
        return GMF_ERR_HOST;
    }
}

extern "C" int gmf_ctx_create(int device, int32_t slots, size_t memory_budget, gmf_ctx** out) {
    return guarded([&] { return ctx_create(device, slots, memory_budget, out); });
}

extern "C" int gmf_ctx_destroy(gmf_ctx* c) {
    return guarded([&] { return ctx_destroy(c); });
}

extern "C" int gmf_batch_submit(gmf_ctx* c, const gmf_host_pairs* p, const gmf_sw_params* prm,
                                const gmf_host_sw_results* r, int64_t* ticket) {
    return guarded([&] { return batch_submit(c, p, prm, r, ticket); });
}

extern "C" int gmf_batch_poll(gmf_ctx* c, int64_t ticket) {
    return guarded([&] { return complete(c, ticket, false); });
}

extern "C" int gmf_batch_wait(gmf_ctx* c, int64_t ticket) {
    return guarded([&] { return complete(c, ticket, true); });
}
