// C ABI of the banded SW kernels: the batched form (device classifier + one
// persistent, work-queue-driven kernel per pair class) and the plain form
// (one warp per pair, int32, one launch).
//
// Batched form:
//   1. sw_classify_kernel sorts the pairs (in the caller's processing order,
//      e.g. longest first) into per-class lists in the workspace: int16x2 with
//      8 / 16 / 32 lanes per pair chosen by band width, or int32 when a score
//      could leave int16.  No host synchronisation: the compute kernels read
//      the list lengths on the device.
//   2. For each class a grid of (SMs x resident blocks) warps pulls pairs from
//      the class list with an atomic head counter until the list is empty, so
//      uneven pairs balance dynamically.
// Results never depend on the class, the order or the batch: every path
// computes the same integer DP and the same traceback decisions.

#include <algorithm>
#include <atomic>
#include <mutex>

#include "sw_common.cuh"

namespace gmf {

__host__ __device__ inline unsigned long long sw32_tb_words_api(int qlen, int W) {
    const long long P = W + 1 > 64 ? W + 1 : 64;
    const long long nstrips = (qlen + 31) / 32;
    const long long last = (nstrips - 1) * P + 2 * ((qlen - 1) & 31) + W - 1;
    return (unsigned long long)((last >> 3) + 1) * 32ull;
}


// The biased 16x2 form is exact when no 16-bit value can wrap and no
// traceback difference leaves 15 bits.  On the gcd-scaled scoring (match m,
// largest penalty p), biased cells lie in [p, smax + 4p + 2] with smax =
// m * (min(qlen, tlen) + 1); the step's cells, including those it masks
// afterwards, stay below smax + 4p + 2 + m, and every difference the
// traceback flags test (H - diag, H - F, F - (H_up - open), E - (M_left -
// open), E - (E_left - ext)) is at most smax + 4p + 2 + m.  Flags are bit 15
// of difference + 0x7fff, exact while that sum stays below 2^16.
__host__ __device__ inline int max_penalty(int mism, int go, int ge) {
    const int m = mism > go ? mism : go;
    return m > ge ? m : ge;
}
__host__ __device__ inline int gcd_int(int a, int b) {
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}
// g of the scaled scoring: gcd of every parameter that enters a cell value
__host__ __device__ inline int score_gcd(int match, int mism, int go, int ge) {
    return gcd_int(gcd_int(match, mism), gcd_int(go, ge));
}
__host__ __device__ inline bool fits_int16(int qlen, int tlen, int m16, int x16, int o16, int e16) {
    const long long smax = (long long)m16 * ((qlen < tlen ? qlen : tlen) + 1);
    const int p = max_penalty(x16, o16, e16);
    return p <= 2048 && m16 <= 2048 && smax + 4LL * p + 2 + m16 <= 32768;
}

// Class of a pair.  Narrow bands share a warp (8 or 16 lanes per pair); wide
// bands get a warp; long pairs with wide bands get 2, 4 or 8 warps of one CTA
// when their period lets that many warps run concurrently (P >= NW * (4*32 +
// 4)) and the pair has at least two strips per warp.  Each cooperative class
// covers one period range [NW * 132, 2 * NW * 132) (the 8-warp class up to
// COOP_PMAX); shorter pairs in those ranges take one warp.
__host__ __device__ inline int sw_class(int qlen, int tlen, int hb, int match, int mism, int go, int ge,
                                        int l8w, int l16w, const int* cmin) {
    if (!fits_int16(qlen, tlen, match, mism, go, ge)) return CLS_I32;  // scaled scoring (SwArgs m16...)
    const int W = 2 * hb + 1;
    if (W <= l8w) return CLS_I16_L8;
    if (W <= l16w) return CLS_I16_L16;
    const int P = sw16_period(W, 32);
    const int strips = (qlen + 63) / 64;
    // each cooperative class holds one period range (its rings are sized for it)
    if (P >= 8 * 132 && P <= COOP_PMAX) return (cmin[2] > 0 && strips >= cmin[2]) ? CLS_I16_C8 : CLS_I16_L32;
    if (P >= 4 * 132 && P < 8 * 132) return (cmin[1] > 0 && strips >= cmin[1]) ? CLS_I16_C4 : CLS_I16_L32;
    if (P >= 2 * 132 && P < 4 * 132) return (cmin[0] > 0 && strips >= cmin[0]) ? CLS_I16_C2 : CLS_I16_L32;
    return CLS_I16_L32;
}

__global__ void sw_classify_kernel(SwArgs a) {
    const int lane = threadIdx.x & 31;
    for (int i0 = blockIdx.x * blockDim.x; i0 < a.n_pairs; i0 += gridDim.x * blockDim.x) {
        const int idx = i0 + threadIdx.x;
        int p = -1, cls = -1;
        if (idx < a.n_pairs) {
            p = a.order ? a.order[idx] : idx;
            const int ql = (int)(a.q_off[p + 1] - a.q_off[p]);
            const int tl = (int)(a.t_off[p + 1] - a.t_off[p]);
            cls = sw_class(ql, tl, a.hb[p], a.m16, a.x16, a.o16, a.e16, a.l8w, a.l16w, a.cmin);
        }
        const unsigned lt = (1u << lane) - 1u;
#pragma unroll
        for (int c = 0; c < N_CLASSES; ++c) {
            const unsigned b = __ballot_sync(FULL_MASK, cls == c);
            if (!b) continue;
            int base = 0;
            const int leader = __ffs(b) - 1;
            if (lane == leader) base = atomicAdd(&a.queue[N_CLASSES + c], __popc(b));
            base = __shfl_sync(FULL_MASK, base, leader);
            if (cls == c) a.lists[(size_t)c * a.n_pairs + base + __popc(b & lt)] = p;
        }
    }
}

static size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// Queue heads and counts, the class lists, and the per-pair traceback
// location (base word, layout tag) the deferred walk reads.
static size_t queue_bytes(int n_pairs) {
    // heads/counts, class lists, walk records (base, tag), group x-drop records (row maxima, carry)
    return round_up(2 * N_CLASSES * sizeof(int32_t), 256) + round_up((size_t)N_CLASSES * n_pairs * 4, 256) +
           round_up((size_t)n_pairs * 8, 256) + round_up((size_t)n_pairs * 4, 256) +
           round_up((size_t)n_pairs * 8, 256) + round_up((size_t)n_pairs * 4, 256);
}

// Side streams of the batched form, one per pair class.  The class kernels
// are forked onto them from the caller's stream and joined back before the
// walk, so a class whose long pairs are draining shares the GPU with the next
// class instead of idling it.  Each caller stream gets its own set (created
// on its first call, up to kSideSets per device; later callers share the
// last set), so calls from different streams -- the workers of a serving
// loop -- never queue behind each other on a side stream.
constexpr int N_SIDE = N_CLASSES;
struct SideStreams {
    cudaStream_t owner;  // the caller stream this set serves
    cudaStream_t s[N_SIDE];
    cudaEvent_t fork;
    cudaEvent_t join[N_SIDE];
    bool ready;
};
constexpr int kMaxSideDevices = 64;
constexpr int kSideSets = 16;
std::mutex g_side_mu;  // guards side streams, tuning, and every fork/launch/join sequence
SideStreams g_side[kMaxSideDevices][kSideSets];

// Scheduling knobs per device (see gmf_sw_tuning).
struct Tuning {
    gmf_sw_tuning t;
    bool set;
};
Tuning g_tuning[kMaxSideDevices];

static gmf_sw_tuning default_tuning() {
    gmf_sw_tuning t;
    t.l8_max_w = 61;
    t.l16_max_w = 125;
    t.coop_min_strips[0] = 4;
    t.coop_min_strips[1] = 8;
    t.coop_min_strips[2] = 16;
    t.warps_per_block = 4;
    t.side_streams = 1;
    return t;
}

static int current_tuning(gmf_sw_tuning* out) {  // caller holds g_side_mu
    int dev = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxSideDevices) return GMF_ERR_LIMIT;
    *out = g_tuning[dev].set ? g_tuning[dev].t : default_tuning();
    return GMF_OK;
}

static int side_streams(cudaStream_t owner, SideStreams** out) {  // caller holds g_side_mu
    int dev = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxSideDevices) return GMF_ERR_LIMIT;
    SideStreams* sets = g_side[dev];
    int k = 0;
    while (k < kSideSets - 1 && sets[k].ready && sets[k].owner != owner) ++k;
    SideStreams& ss = sets[k];
    if (!ss.ready) {
        for (int i = 0; i < N_SIDE; ++i) {
            GMF_CUDA_TRY(cudaStreamCreateWithFlags(&ss.s[i], cudaStreamNonBlocking));
            GMF_CUDA_TRY(cudaEventCreateWithFlags(&ss.join[i], cudaEventDisableTiming));
        }
        GMF_CUDA_TRY(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming));
        ss.owner = owner;
        ss.ready = true;
    }
    *out = &ss;
    return GMF_OK;
}

static int ring_entries(int d_max) {
    int r = 1;
    while (r < d_max + 1) r <<= 1;
    return r;
}

static int check_common(const gmf_pairs* pairs, const gmf_sw_params* params, const gmf_sw_results* res) {
    if (!pairs || !params || !res) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->n_pairs < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->max_half_band < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->max_half_band > GMF_MAX_HALF_BAND) return GMF_ERR_LIMIT;
    const int lim = 1 << 20;
    if (params->match_score <= 0 || params->match_score > lim || params->mismatch_penalty < 0 ||
        params->mismatch_penalty > lim || params->gap_open < 0 || params->gap_open > lim ||
        params->gap_extend < 0 || params->gap_extend > lim)
        return GMF_ERR_INVALID_ARGUMENT;
    if (!res->score || !res->query_end || !res->target_end || !res->cigar_used || !res->error_flags)
        return GMF_ERR_INVALID_ARGUMENT;
    if (res->cigar && (!res->cigar_start || !res->cigar_len || res->cigar_capacity < 0))
        return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->n_pairs > 0 && (!pairs->query || !pairs->query_off || !pairs->target ||
                               !pairs->target_off || !pairs->half_band || !pairs->band_offset))
        return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->xdrop_group_off && pairs->n_xdrop_groups < 0) return GMF_ERR_INVALID_ARGUMENT;
    return GMF_OK;
}

// Test hook of the bounded waits (gmf_sw_test_coop_wait): 0 = the default limit.
static std::atomic<int> g_test_spin_limit{0};
static std::atomic<int> g_test_stall{0};

static void fill_args(SwArgs& a, const gmf_pairs* pairs, const gmf_sw_params* params,
                      const gmf_sw_results* res) {
    const int lim = g_test_spin_limit.load();
    a.coop_spin_limit = lim > 0 ? lim : COOP_WAIT_LIMIT;
    a.coop_stall = g_test_stall.load();
    a.q = pairs->query;
    a.q_off = pairs->query_off;
    a.t = pairs->target;
    a.t_off = pairs->target_off;
    a.hb = pairs->half_band;
    a.boff = pairs->band_offset;
    a.order = pairs->order;
    a.n_pairs = pairs->n_pairs;
    a.match = params->match_score;
    a.mismatch = params->mismatch_penalty;
    a.gap_open = params->gap_open;
    a.gap_extend = params->gap_extend;
    a.x_drop = params->x_drop;
    a.l8w = 61;  // defaults; the batched form replaces them with the device's tuning
    a.l16w = 125;
    a.cmin[0] = 4;
    a.cmin[1] = 8;
    a.cmin[2] = 16;
    a.max_hb = pairs->max_half_band;
    const int g = score_gcd(params->match_score, params->mismatch_penalty, params->gap_open, params->gap_extend);
    a.g16 = g;
    a.m16 = params->match_score / g;
    a.x16 = params->mismatch_penalty / g;
    a.o16 = params->gap_open / g;
    a.e16 = params->gap_extend / g;
    const int pmax = max_penalty(a.x16, a.o16, a.e16);
    a.zero16 = 4 * pmax + 2;
    a.neg16 = 2 * pmax;
    const unsigned one2 = 0x00010001u;
    K16& k = a.k16;
    k.Z = (unsigned)a.zero16;
    k.NEGV = (unsigned)a.neg16;
    k.Z2 = k.Z * one2;
    k.NEG2 = k.NEGV * one2;
    k.GO2 = (unsigned)a.o16 * one2;
    k.GE2 = (unsigned)a.e16 * one2;
    k.MATCH2 = (unsigned)a.m16 * one2;
    k.NGE2 = ((0x10000u - (unsigned)a.e16) & 0xFFFFu) * one2;
    k.MX = (unsigned)(a.m16 + a.x16);
    k.EB2 = (0x8000u - (unsigned)a.e16) * one2;
    k.ONE = 1u;
    k.NEG1 = 0xFFFFFFFFu;
    k.G = g;
    a.score = res->score;
    a.q_end = res->query_end;
    a.t_end = res->target_end;
    a.q_start = res->query_start;
    a.t_start = res->target_start;
    a.op_counts = res->op_counts;
    a.cigar = res->cigar;
    a.cigar_cap = res->cigar_capacity;
    a.cigar_start = res->cigar_start;
    a.cigar_len = res->cigar_len;
    a.cigar_used = res->cigar_used;
    a.err = res->error_flags;
}

static int e_mode_of(const gmf_sw_params* p) {
    return p->gap_open > p->gap_extend ? 0 : (p->gap_open == p->gap_extend ? 1 : 2);
}

struct DevInfo {
    int sms = 148;
    int smem_optin = 227 * 1024;
};

static int dev_info(DevInfo& di) {
    int dev = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    GMF_CUDA_TRY(cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev));
    GMF_CUDA_TRY(cudaDeviceGetAttribute(&di.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    return GMF_OK;
}

// Warps per block that fit the per-warp shared memory.
static int warps_per_block(size_t per_warp, const DevInfo& di, int cap = 4) {
    int wpb = cap < 1 ? 1 : (cap > 4 ? 4 : cap);
    while (wpb > 1 && per_warp * wpb > (size_t)di.smem_optin) --wpb;
    return per_warp > (size_t)di.smem_optin ? 0 : wpb;
}

// Group x-drop (alignment/extension.py L139-193 on a batch of several pairs):
// the row loop stops after the first row on which every member satisfies
// (max row max so far) - row max > x_drop, a member's rows past its query
// reading as 0; each member's best is then the first strictly larger row max
// over the rows up to that one.  One warp per group of two or more members
// (a pair alone already stopped on its own rows), rows in chunks of 32: a
// prefix max over the lanes plus the member's carry gives the running max.
__global__ void __launch_bounds__(128) sw_xdrop_group_kernel(SwArgs a) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    for (int g = gw; g < a.n_xg; g += nw) {
        const int lo = max(a.xg_off[g], 0), hi = min(a.xg_off[g + 1], a.n_pairs);
        if (hi - lo <= 1) continue;
        int max_rows = 0;
        for (int p = lo; p < hi; ++p) max_rows = max(max_rows, (int)(a.q_off[p + 1] - a.q_off[p]));
        for (int p = lo + lane; p < hi; p += 32) a.rm_seen[p] = 0;
        __syncwarp();
        // pass 1: the last row the batch considers
        int stop = max_rows - 1;
        for (int r0 = 0; r0 < max_rows; r0 += 32) {
            const int r = r0 + lane;
            unsigned all = __ballot_sync(FULL_MASK, r < max_rows);
            for (int p = lo; p < hi; ++p) {
                const unsigned long long rb_at = a.rm_base[p];
                const int ql = (int)(a.q_off[p + 1] - a.q_off[p]);
                const int2* rm = rb_at == ~0ull ? nullptr : reinterpret_cast<const int2*>(a.pool + rb_at);
                const int rb = (rm && r < ql) ? rm[r].x : 0;
                int pm = rb;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(FULL_MASK, pm, o);
                    if (lane >= o) pm = imax(pm, u);
                }
                pm = imax(pm, a.rm_seen[p]);
                all &= __ballot_sync(FULL_MASK, pm - rb > a.x_drop);
                const int carry = __shfl_sync(FULL_MASK, pm, 31);
                __syncwarp();
                if (lane == 0) a.rm_seen[p] = carry;
                __syncwarp();
            }
            if (all) {
                stop = r0 + __ffs((int)all) - 1;
                break;
            }
        }
        // pass 2: each member's best over rows [0, min(stop, qlen-1)]
        for (int p = lo; p < hi; ++p) {
            const unsigned long long rb_at = a.rm_base[p];
            if (rb_at == ~0ull) continue;  // no rows: the class kernel's empty result stands
            const int2* rm = reinterpret_cast<const int2*>(a.pool + rb_at);
            const int ql = (int)(a.q_off[p + 1] - a.q_off[p]);
            const int last = imin(stop, ql - 1);
            int bh = 0, bi = 0, bd = 0;
            for (int r0 = 0; r0 <= last; r0 += 32) {
                const int r = r0 + lane;
                const int2 v = r <= last ? rm[r] : make_int2(-1, 0);
                int cv = v.x, cl = lane;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const int ov = __shfl_xor_sync(FULL_MASK, cv, o);
                    const int ol = __shfl_xor_sync(FULL_MASK, cl, o);
                    if (ov > cv || (ov == cv && ol < cl)) {
                        cv = ov;
                        cl = ol;
                    }
                }
                const int cd = __shfl_sync(FULL_MASK, v.y, cl);
                if (cv > bh) {
                    bh = cv;
                    bi = r0 + cl + 1;
                    bd = cd;
                }
            }
            if (lane == 0) {
                const int hb = a.hb[p], off = a.boff[p];
                a.score[p] = bh;
                a.q_end[p] = bh > 0 ? bi : 0;
                a.t_end[p] = bh > 0 ? bi + off - hb + bd : 0;
            }
        }
    }
}

static int launch_xdrop_groups(const SwArgs& a, int sms, cudaStream_t stream) {
    const long long warps = std::min<long long>(a.n_xg, (long long)sms * 16);
    sw_xdrop_group_kernel<<<(int)((warps + 3) / 4), 128, 0, stream>>>(a);
    return cuda_status(cudaGetLastError());
}

}  // namespace gmf

using namespace gmf;

extern "C" size_t gmf_banded_sw_workspace_bytes(int32_t n_pairs, const int32_t* qlen,
                                                const int32_t* tlen, const int32_t* half_band,
                                                int32_t with_traceback) {
    size_t words = 0;
    if (n_pairs > 0 && qlen && tlen && half_band) {
        for (int32_t p = 0; p < n_pairs; ++p) {
            const int ql = std::max(qlen[p], 0), tl = std::max(tlen[p], 0);
            const int W = 2 * std::max(half_band[p], 0) + 1;
            words += 2 * (size_t)ql + 8;  // row maxima (x-drop) + alignment padding
            if (with_traceback && ql > 0) {
                // the larger of the int32 and int16x2 layouts, whichever class the pair gets
                unsigned long long tb = sw32_tb_words_api(ql, W);
                for (int L = 8; L <= 32; L <<= 1) tb = std::max(tb, sw16_tb_words_l(ql, W, L));
                words += tb + (size_t)ql + tl + 1;
            }
        }
    }
    return 256 + queue_bytes(std::max(n_pairs, 0)) + round_up(words * 4, 256);
}

static int sw_prepare(const gmf_pairs* pairs, const gmf_sw_params* params, const gmf_sw_results* res,
                      void* workspace, size_t workspace_bytes, cudaStream_t stream, SwArgs& a) {
    GMF_TRY(check_common(pairs, params, res));
    const size_t qb = queue_bytes(pairs->n_pairs);
    if (!workspace || workspace_bytes < 256 + qb) return GMF_ERR_WORKSPACE;
    GMF_BIND_STREAM(stream);
    GMF_CUDA_TRY(cudaMemsetAsync(workspace, 0, 256 + round_up(2 * N_CLASSES * sizeof(int32_t), 256), stream));
    GMF_CUDA_TRY(cudaMemsetAsync(res->cigar_used, 0, sizeof(unsigned long long), stream));
    GMF_CUDA_TRY(cudaMemsetAsync(res->error_flags, 0, sizeof(int32_t), stream));
    fill_args(a, pairs, params, res);
    char* w = (char*)workspace;
    a.counters = (unsigned long long*)w;
    a.queue = (int32_t*)(w + 256);
    a.lists = (int32_t*)(w + 256 + round_up(2 * N_CLASSES * sizeof(int32_t), 256));
    char* tb = (char*)a.lists + round_up((size_t)N_CLASSES * pairs->n_pairs * 4, 256);
    a.tb_base = (unsigned long long*)tb;
    a.tb_tag = (int32_t*)(tb + round_up((size_t)pairs->n_pairs * 8, 256));
    a.defer_walk = 0;
    if (pairs->n_pairs > 0)
        GMF_CUDA_TRY(cudaMemsetAsync(a.tb_tag, 0xFF, (size_t)pairs->n_pairs * 4, stream));
    char* rm = tb + round_up((size_t)pairs->n_pairs * 8, 256) + round_up((size_t)pairs->n_pairs * 4, 256);
    const bool groups = params->x_drop > 0 && pairs->xdrop_group_off && pairs->n_xdrop_groups > 0 &&
                        pairs->n_pairs > 0;
    a.xg_off = groups ? pairs->xdrop_group_off : nullptr;
    a.n_xg = groups ? pairs->n_xdrop_groups : 0;
    a.rm_base = groups ? (unsigned long long*)rm : nullptr;
    a.rm_seen = groups ? (int32_t*)(rm + round_up((size_t)pairs->n_pairs * 8, 256)) : nullptr;
    if (groups) GMF_CUDA_TRY(cudaMemsetAsync(a.rm_base, 0xFF, (size_t)pairs->n_pairs * 8, stream));
    a.pool = (uint32_t*)(w + 256 + qb);
    a.pool_cap = (workspace_bytes - 256 - qb) / 4;
    return GMF_OK;
}

extern "C" int gmf_banded_sw(const gmf_pairs* pairs, const gmf_sw_params* params,
                             const gmf_sw_results* res, void* workspace, size_t workspace_bytes,
                             gmf_stream_t stream_) {
    const cudaStream_t stream = (cudaStream_t)stream_;
    SwArgs a;
    GMF_TRY(sw_prepare(pairs, params, res, workspace, workspace_bytes, stream, a));
    if (pairs->n_pairs == 0) return GMF_OK;
    DevInfo di;
    GMF_TRY(dev_info(di));
    const bool tb = res->cigar != nullptr;
    const bool xd = params->x_drop > 0;
    const int em = e_mode_of(params);
    a.defer_walk = tb ? 1 : 0;
    std::lock_guard<std::mutex> lock(g_side_mu);
    gmf_sw_tuning tun;
    GMF_TRY(current_tuning(&tun));
    a.l8w = tun.l8_max_w;
    a.l16w = tun.l16_max_w;
    for (int i = 0; i < 3; ++i) a.cmin[i] = tun.coop_min_strips[i];

    const int cls_blocks = std::min((pairs->n_pairs + 255) / 256, di.sms * 4);
    sw_classify_kernel<<<cls_blocks, 256, 0, stream>>>(a);
    GMF_CUDA_TRY(cudaGetLastError());

    const int Wmax = 2 * pairs->max_half_band + 1;
    const int Pmax = sw16_period(Wmax, 32);
    // every class kernel goes to its own side stream (or, untuned-off, to the
    // caller's stream), longest classes first
    SideStreams* ss = nullptr;
    const bool fork = tun.side_streams != 0;
    if (fork) {
        GMF_TRY(side_streams(stream, &ss));
        GMF_CUDA_TRY(cudaEventRecord(ss->fork, stream));
    }
    int used = 0;
    auto next_stream = [&](cudaStream_t* out) -> int {
        if (!fork) {
            *out = stream;
            return GMF_OK;
        }
        GMF_CUDA_TRY(cudaStreamWaitEvent(ss->s[used], ss->fork, 0));
        *out = ss->s[used++];
        return GMF_OK;
    };
    // cooperative classes: the 2- and 4-warp ones with a ring of P + 8 entries
    // per warp for the largest period the class can hold, the 8-warp one with
    // back-pressure and a fixed ring
    const int coop_cls[3] = {CLS_I16_C8, CLS_I16_C4, CLS_I16_C2};
    const int coop_pmin[3] = {8 * 132, 4 * 132, 2 * 132};
    const int coop_pcap[3] = {COOP_PMAX, 8 * 132 - 4, 4 * 132 - 4};
    const int coop_knob[3] = {2, 1, 0};  // coop_min_strips index of C8, C4, C2
    for (int c = 0; c < 3; ++c) {
        if (Pmax < coop_pmin[c] || tun.coop_min_strips[coop_knob[c]] <= 0) continue;  // class empty
        SwArgs ac = a;
        // the 8-warp class bounds each warp's lead over its reader (1024 entries
        // cover periods up to COOP_PMAX); the others hold a whole period
        ac.ring = coop_cls[c] == CLS_I16_C8 ? 1024 : ring_entries(std::min(Pmax, coop_pcap[c]) + 7);
        if ((size_t)sw16_coop_warps(coop_cls[c]) * ac.ring * 4 > (size_t)di.smem_optin) return GMF_ERR_LIMIT;
        cudaStream_t s;
        GMF_TRY(next_stream(&s));
        GMF_TRY(launch_sw16_coop(ac, coop_cls[c], tb, xd, em, s));
    }
    // one-warp and shared-warp classes (a class only ever holds pairs up to
    // its own band limit), widest first
    const int cls_wmax[3] = {std::min(Wmax, tun.l8_max_w), std::min(Wmax, tun.l16_max_w), Wmax};
    const int lanes[3] = {8, 16, 32};
    for (int c = 2; c >= 0; --c) {
        const int L = lanes[c];
        SwArgs ac = a;
        ac.ring = ring_entries(std::max(3, sw16_period(cls_wmax[c], L) - 4 * L - 1));
        const int wpb = warps_per_block((size_t)sw16_smem_per_warp(c, ac.ring), di, tun.warps_per_block);
        if (wpb == 0) return GMF_ERR_LIMIT;
        const int grid = di.sms * std::max(1, 16 / wpb);
        cudaStream_t s;
        GMF_TRY(next_stream(&s));
        GMF_TRY(launch_sw16(ac, c, tb, xd, em, grid, wpb, s));
    }
    SwArgs a32 = a;
    a32.ring = ring_entries(std::max(64, Wmax + 1) - 64);
    const int wpb = warps_per_block((size_t)sw32_smem_per_warp(a32.ring), di, tun.warps_per_block);
    if (wpb == 0) return GMF_ERR_LIMIT;
    {
        cudaStream_t s;
        GMF_TRY(next_stream(&s));
        GMF_TRY(launch_sw32(a32, tb, xd, em, true, di.sms * std::max(1, 12 / wpb), wpb, s));
    }
    for (int i = 0; fork && i < used; ++i) {
        GMF_CUDA_TRY(cudaEventRecord(ss->join[i], ss->s[i]));
        GMF_CUDA_TRY(cudaStreamWaitEvent(stream, ss->join[i], 0));
    }
    if (a.n_xg > 0) GMF_TRY(launch_xdrop_groups(a, di.sms, stream));
    return tb ? launch_sw_walk(a, stream) : GMF_OK;
}

extern "C" int gmf_banded_sw_plain(const gmf_pairs* pairs, const gmf_sw_params* params,
                                   const gmf_sw_results* res, void* workspace, size_t workspace_bytes,
                                   gmf_stream_t stream_) {
    const cudaStream_t stream = (cudaStream_t)stream_;
    SwArgs a;
    GMF_TRY(sw_prepare(pairs, params, res, workspace, workspace_bytes, stream, a));
    if (pairs->n_pairs == 0) return GMF_OK;
    DevInfo di;
    GMF_TRY(dev_info(di));
    const int Wmax = 2 * pairs->max_half_band + 1;
    a.ring = ring_entries(std::max(64, Wmax + 1) - 64);
    const int wpb = warps_per_block((size_t)sw32_smem_per_warp(a.ring), di);
    if (wpb == 0) return GMF_ERR_LIMIT;
    const int grid = (pairs->n_pairs + wpb - 1) / wpb;
    const bool tb = res->cigar != nullptr;
    if (a.n_xg == 0) return launch_sw32(a, tb, params->x_drop > 0, e_mode_of(params), false, grid, wpb, stream);
    // x-drop groups: the group pass settles each member's best before the walk
    a.defer_walk = tb ? 1 : 0;
    GMF_TRY(launch_sw32(a, tb, true, e_mode_of(params), false, grid, wpb, stream));
    GMF_TRY(launch_xdrop_groups(a, di.sms, stream));
    return tb ? launch_sw_walk(a, stream) : GMF_OK;
}

extern "C" int gmf_sw_get_tuning(gmf_sw_tuning* t) {
    if (!t) return GMF_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_side_mu);
    return current_tuning(t);
}

extern "C" int gmf_sw_set_tuning(const gmf_sw_tuning* t) {
    if (!t) return GMF_ERR_INVALID_ARGUMENT;
    const int wmax = 2 * GMF_MAX_HALF_BAND + 1;
    if (t->l8_max_w < 0 || t->l8_max_w > wmax || t->l16_max_w < t->l8_max_w || t->l16_max_w > wmax)
        return GMF_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < 3; ++i)
        if (t->coop_min_strips[i] < 0 || t->coop_min_strips[i] > (1 << 24)) return GMF_ERR_INVALID_ARGUMENT;
    if (t->warps_per_block < 1 || t->warps_per_block > 4 || (t->side_streams != 0 && t->side_streams != 1))
        return GMF_ERR_INVALID_ARGUMENT;
    int dev = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxSideDevices) return GMF_ERR_LIMIT;
    std::lock_guard<std::mutex> lock(g_side_mu);
    g_tuning[dev].t = *t;
    g_tuning[dev].set = true;
    return GMF_OK;
}

extern "C" int gmf_sw_test_coop_wait(int32_t spin_limit, int32_t stall_writers) {
    if (spin_limit < 0 || (stall_writers != 0 && stall_writers != 1)) return GMF_ERR_INVALID_ARGUMENT;
    g_test_spin_limit.store(spin_limit);
    g_test_stall.store(stall_writers);
    return GMF_OK;
}
