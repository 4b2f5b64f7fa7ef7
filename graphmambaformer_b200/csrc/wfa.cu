// Unit-cost global wavefront alignment (edit distance + CIGAR).
//
// Semantics (graphmambaformer/alignment/extension.py L308-463,
// WavefrontAligner): diagonal k = i - j, offset = query bases consumed.
// Wavefront 0 is the match run from (0, 0); wavefront s takes, per diagonal
// k in [-s, s], the largest of three candidates of wavefront s-1 --
// substitution (k, +1), insertion (k-1, +1), deletion (k+1, +0) -- each
// rejected on its own when it leaves the matrix (offset outside [0, n] or
// column outside [0, m]), then extends through the run of matching codes (a
// code matches iff equal, >= 0 and != 5).  The alignment is complete at the
// first s whose diagonal n - m reaches n; the distance bound is tested after
// that check, so a pair exactly at the bound succeeds.  n == 0 or m == 0 is
// answered directly (distance max(n, m), CIGAR I n D m).  The traceback walks
// back from (s, n - m), taking at each score the first largest of the
// unclipped candidates X, I, D; the gap between that candidate and the
// diagonal's reach is a run of matches (never negative).
//
// Layout:
//   forward kernel  persistent blocks pull pairs 8 at a time, in the caller's
//                   order.  A pair is computed by one warp, or by the whole
//                   block when it is long (a side of 4000 codes in the first
//                   pass, distance 96 in the second): the team's threads take
//                   the diagonals of a wavefront in turn and extend each one
//                   4 codes per step (a sliding window of aligned words of
//                   both sequences, byte compares).  The two live wavefronts
//                   sit in shared memory (scores up to 255 for a warp, 2050
//                   for a block) and move to a global slot beyond.  The
//                   second pass also stores wavefront s at s*s + s + k.
//   walk kernel     one thread per pair: two passes over the history (count,
//                   then write the run-length words back to front).

#include "gmf_common.cuh"

namespace {

constexpr int WFA_WARPS = 8;                          // warps per block
constexpr int WFA_SMEM_S = 255;                       // wavefronts up to this score in shared memory
constexpr int WFA_SMEM_WF = 2 * WFA_SMEM_S + 3;       // ints per shared wavefront
constexpr int WFA_MAX_BLOCKS_PER_SM = 4;
constexpr int WFA_BLOCK_S = (WFA_WARPS * WFA_SMEM_WF - 3) / 2;  // block-wide wavefronts: scores up to 2050
constexpr int WFA_LONG_LEN = 4000;  // first pass: a pair with a side this long gets a whole block
constexpr int WFA_LONG_D = 96;      // second pass: a pair at this distance gets a whole block

struct Seq {
    const uint32_t* w;  // aligned words covering the whole buffer
    int nw;
    long long base;     // byte offset of the buffer's first code from w
    __device__ unsigned ld(long long i) const {
        i = i < 0 ? 0 : (i >= nw ? nw - 1 : i);
        return __ldg(w + i);
    }
};

__host__ __device__ inline Seq make_seq(const int8_t* buf, long long total) {
    Seq s;
    const uintptr_t a = (uintptr_t)buf & ~(uintptr_t)3;
    s.w = reinterpret_cast<const uint32_t*>(a);
    s.base = (long long)((uintptr_t)buf - a);
    const long long nw = total > 0 ? ((s.base + total - 1) >> 2) + 1 : 1;
    s.nw = nw > 0x7fffffffll ? 0x7fffffff : (int)nw;
    return s;
}

struct WfaArgs {
    int n_pairs;
    const int8_t* q;
    const long long* q_off;
    const int8_t* t;
    const long long* t_off;
    const int* order;
    Seq Q, T;
    int max_distance;
    int eff;               // largest distance any pair can reach: min(max_distance, longest side)
    int* spill;            // 2 * (2*eff + 3) ints per warp, or null when eff <= WFA_SMEM_S
    unsigned* work;        // pair counter
    int* distance;         // forward without history: written; with history: read
    // history (align only)
    int* hist;
    long long hist_cap;    // ints
    unsigned long long* hist_used;
    long long* hist_off;   // per pair: offset into hist, -1 when absent
    int* err;
    int long_len, long_d;  // whole-block pairs: a side of long_len codes (first pass), distance long_d (second)
};

__device__ __forceinline__ int clip_cand(int v, int k, int n, int m) {
    const int col = v - k;
    return (v < 0 || v > n || col < 0 || col > m) ? -1 : v;
}

// Offset after the run of matches from query position i on diagonal k.  Both
// sequences are read as a sliding window of aligned words (one new word per
// sequence per 4 codes, loaded one step ahead of the compare).
__device__ __forceinline__ int wfa_extend(const Seq& Q, long long q0, const Seq& T, long long t0, int n, int m,
                                          int i, int k) {
    if (i < 0) return i;
    const int j = i - k;
    if (j < 0 || i >= n || j >= m) return i;
    const long long bq = Q.base + q0 + i, bt = T.base + t0 + j;
    long long wq = bq >> 2, wt = bt >> 2;
    const int sq = (int)(bq & 3) * 8, st = (int)(bt & 3) * 8;
    unsigned qa = Q.ld(wq), qb = Q.ld(wq + 1), ta = T.ld(wt), tb = T.ld(wt + 1);
    const int lim = min(n - i, m - j);
    int adv = 0;
    for (;;) {
        const unsigned qn = Q.ld(wq + 2), tn = T.ld(wt + 2);
        const unsigned a = __funnelshift_r(qa, qb, sq), b = __funnelshift_r(ta, tb, st);
        const unsigned bad = __vcmpne4(a, b) | __vcmpeq4(a, 0x05050505u) | __vcmpgeu4(a, 0x80808080u);
        const int r = bad ? (__ffs((int)bad) - 1) >> 3 : 4;
        adv += r;
        if (r < 4 || adv >= lim) break;
        qa = qb;
        qb = qn;
        ta = tb;
        tb = tn;
        ++wq;
        ++wt;
    }
    return i + min(adv, lim);
}

// A pair is computed by one warp, or by the whole block when it is long.
struct WarpTeam {
    int rank;
    static constexpr int SIZE = 32;
    __device__ void sync() const { __syncwarp(); }
    __device__ bool sync_any(bool x) const {
        __syncwarp();
        return __any_sync(gmf::FULL_MASK, x);
    }
    __device__ long long bcast0(long long v, long long*) const { return __shfl_sync(gmf::FULL_MASK, v, 0); }
};

struct BlockTeam {
    int rank;
    static constexpr int SIZE = WFA_WARPS * 32;
    __device__ void sync() const { __syncthreads(); }
    __device__ bool sync_any(bool x) const { return __syncthreads_or(x) != 0; }
    __device__ long long bcast0(long long v, long long* scratch) const {
        if (rank == 0) *scratch = v;
        __syncthreads();
        const long long r = *scratch;
        __syncthreads();
        return r;
    }
};

// The wavefronts of one pair up to completion; returns the distance, or -1
// once `limit` is reached without completing.  `sm` holds two wavefronts of
// scores up to `sm_s`; beyond that they move to `gl` (two of 2*eff+3).  With
// `hist`, wavefront s is also stored at hist[s*s + s + k].
template <bool HIST, class Team>
__device__ int wfa_forward(const WfaArgs& A, long long q0, long long t0, int n, int m, int limit, int* sm, int sm_s,
                           int* gl, int* hist, const Team& tm, long long* scratch) {
    const int final_k = n - m;
    long long h0 = 0;
    if (tm.rank == 0) h0 = wfa_extend(A.Q, q0, A.T, t0, n, m, 0, 0);
    h0 = tm.bcast0(h0, scratch);
    if (HIST && tm.rank == 0) hist[0] = (int)h0;
    if (final_k == 0 && h0 >= n) return 0;
    int* prev = sm;
    int* cur = sm + 2 * sm_s + 3;
    int cen = sm_s + 1;
    if (tm.rank == 0) prev[cen] = (int)h0;
    tm.sync();
    bool shared = true;
    for (int s = 1;; ++s) {
        if (s - 1 >= limit || s > A.eff) return -1;  // s <= max(n, m) <= eff always holds
        if (shared && s > sm_s) {  // move the live wavefront to the global slot
            const int gcen = A.eff + 1;
            for (int k = -(s - 1) + tm.rank; k <= s - 1; k += Team::SIZE) gl[k + gcen] = prev[k + cen];
            tm.sync();
            prev = gl;
            cur = gl + 2 * A.eff + 3;
            cen = gcen;
            shared = false;
        }
        const int ps = s - 1;
        bool done = false;
        for (int base = -s; base <= s; base += Team::SIZE) {
            const int k = base + tm.rank;
            if (k <= s) {
                int sub = (k >= -ps && k <= ps) ? prev[k + cen] : -1;
                int ins = (k - 1 >= -ps && k - 1 <= ps) ? prev[k - 1 + cen] : -1;
                int del = (k + 1 >= -ps && k + 1 <= ps) ? prev[k + 1 + cen] : -1;
                sub = clip_cand(sub >= 0 ? sub + 1 : -1, k, n, m);
                ins = clip_cand(ins >= 0 ? ins + 1 : -1, k, n, m);
                del = clip_cand(del, k, n, m);
                const int best = max(max(sub, ins), del);
                const int r = wfa_extend(A.Q, q0, A.T, t0, n, m, best, k);
                cur[k + cen] = r;
                if (HIST) hist[(long long)s * s + s + k] = r;
                done |= (k == final_k) && r >= n;
            }
        }
        if (tm.sync_any(done)) return s;
        int* tmp = prev;
        prev = cur;
        cur = tmp;
    }
}

// One pair: its distance (first pass) or its history (second pass).
template <bool HIST, class Team>
__device__ void wfa_pair(const WfaArgs& A, int p, int* sm, int sm_s, int* gl, const Team& tm, long long* scratch) {
    const long long q0 = A.q_off[p], t0 = A.t_off[p];
    const int n = (int)(A.q_off[p + 1] - q0), m = (int)(A.t_off[p + 1] - t0);
    if (!HIST) {
        int d;
        if (n == 0 || m == 0)
            d = max(n, m);
        else
            d = wfa_forward<false>(A, q0, t0, n, m, A.max_distance, sm, sm_s, gl, nullptr, tm, scratch);
        if (tm.rank == 0) A.distance[p] = d;
        return;
    }
    const int d = A.distance[p];
    long long off = -1;
    if (d > A.eff) {
        if (tm.rank == 0) atomicOr(A.err, (int)GMF_SWF_WORKSPACE);
    } else if (d >= 0 && n > 0 && m > 0) {
        const long long need = (long long)(d + 1) * (d + 1);
        if (tm.rank == 0) {
            const unsigned long long o = atomicAdd(A.hist_used, (unsigned long long)need);
            if ((long long)o + need <= A.hist_cap)
                off = (long long)o;
            else
                atomicOr(A.err, (int)GMF_SWF_WORKSPACE);
        }
        off = tm.bcast0(off, scratch);
        if (off >= 0) {
            const int got = wfa_forward<true>(A, q0, t0, n, m, d, sm, sm_s, gl, A.hist + off, tm, scratch);
            if (got != d) off = -1;  // cannot happen: the pass is deterministic
        }
    }
    if (tm.rank == 0) A.hist_off[p] = off;
}

__device__ __forceinline__ bool wfa_is_long(const WfaArgs& A, int p, bool hist) {
    if (hist) return A.distance[p] >= A.long_d;
    const long long n = A.q_off[p + 1] - A.q_off[p], m = A.t_off[p + 1] - A.t_off[p];
    return (n > m ? n : m) >= A.long_len;
}

// Blocks pull positions of the caller's order.  A block takes one position
// and, when its pair is long, computes it with all its warps (wavefronts in
// the block's shared memory up to score 2050); otherwise it takes 7 more
// positions and its warps compute one pair each (a long pair among those
// goes first, block-wide).  With a longest-first order every long pair gets a
// block of its own.
template <bool HIST>
__global__ void __launch_bounds__(WFA_WARPS * 32) wfa_forward_kernel(WfaArgs A) {
    __shared__ int s_wf[WFA_WARPS * 2 * WFA_SMEM_WF];
    __shared__ int s_pos[WFA_WARPS];
    __shared__ long long s_scratch;
    const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
    const long long slot = 2 * (2ll * A.eff + 3);
    int* gl_warp = A.spill ? A.spill + ((long long)blockIdx.x * WFA_WARPS + wib) * slot : nullptr;
    int* gl_block = A.spill ? A.spill + (long long)blockIdx.x * WFA_WARPS * slot : nullptr;
    const unsigned n = (unsigned)A.n_pairs;
    for (;;) {
        if (tid == 0) {
            const unsigned first = atomicAdd(A.work, 1u);
            s_pos[0] = first < n ? (int)first : -1;
            for (int e = 1; e < WFA_WARPS; ++e) s_pos[e] = -1;
            if (first < n) {
                const int p = A.order ? A.order[first] : (int)first;
                if (!wfa_is_long(A, p, HIST)) {
                    const unsigned more = atomicAdd(A.work, (unsigned)(WFA_WARPS - 1));
                    for (int e = 1; e < WFA_WARPS; ++e)
                        if (more + e - 1 < n) s_pos[e] = (int)(more + e - 1);
                }
            }
        }
        __syncthreads();
        if (s_pos[0] < 0) break;
        bool any_long = false;
        for (int e = 0; e < WFA_WARPS; ++e) {
            if (s_pos[e] < 0) continue;
            const int p = A.order ? A.order[s_pos[e]] : s_pos[e];
            if (wfa_is_long(A, p, HIST)) {
                wfa_pair<HIST>(A, p, s_wf, WFA_BLOCK_S, gl_block, BlockTeam{tid}, &s_scratch);
                any_long = true;
            }
        }
        if (any_long) __syncthreads();
        if (s_pos[wib] >= 0) {
            const int p = A.order ? A.order[s_pos[wib]] : s_pos[wib];
            if (!wfa_is_long(A, p, HIST))
                wfa_pair<HIST>(A, p, s_wf + wib * 2 * WFA_SMEM_WF, WFA_SMEM_S, gl_warp, WarpTeam{lane}, nullptr);
        }
        __syncthreads();
    }
}

struct WalkArgs {
    int n_pairs;
    const long long* q_off;
    const long long* t_off;
    const int* distance;
    const int* hist;
    const long long* hist_off;
    int* op_counts;
    uint32_t* cigar;
    long long cigar_cap;
    long long* cigar_start;
    int* cigar_len;
    unsigned long long* cigar_used;
    int* err;
};

// Run-length emitter in back-to-front order.
struct Emit {
    uint32_t* out;  // null in the counting pass
    long long end;  // one past the pair's last word
    long long words;
    int cur_op, cur_len;
    int n_eq, n_x, n_i, n_d;
    __device__ void init(uint32_t* o, long long e) {
        out = o;
        end = e;
        words = 0;
        cur_op = -1;
        cur_len = 0;
        n_eq = n_x = n_i = n_d = 0;
    }
    __device__ void flush() {
        if (cur_len > 0) {
            if (out) out[end - 1 - words] = ((uint32_t)cur_len << 4) | (uint32_t)cur_op;
            ++words;
        }
        cur_len = 0;
    }
    __device__ void put(int op, int len) {
        if (len <= 0) return;
        n_eq += op == gmf::OP_EQ ? len : 0;
        n_x += op == gmf::OP_X ? len : 0;
        n_i += op == gmf::OP_I ? len : 0;
        n_d += op == gmf::OP_D ? len : 0;
        if (op != cur_op) {
            flush();
            cur_op = op;
        }
        cur_len += len;
    }
};

// Returns false when the walk meets a diagonal without a valid predecessor
// (cannot happen for a history the forward pass completed at distance d;
// checked so that a bad distance never reads outside the pair's history).
__device__ bool wfa_walk(const int* H, int d, int final_k, Emit& e) {
    int k = final_k;
    if (k < -d || k > d) return false;
    for (int s = d; s >= 1; --s) {
        const int reach = H[(long long)s * s + s + k];
        const long long pb = (long long)(s - 1) * (s - 1);
        const int ps = s - 1;
        int v[3];
        const int pk[3] = {k, k - 1, k + 1};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int x = pk[c];
            const int o = (x >= -ps && x <= ps) ? H[pb + ps + x] : -1;
            v[c] = o >= 0 ? (c < 2 ? o + 1 : o) : -1;
        }
        int b = 0;
        if (v[1] > v[b]) b = 1;
        if (v[2] > v[b]) b = 2;
        if (v[b] < 0) return false;
        e.put(gmf::OP_EQ, reach - v[b]);
        e.put(b == 0 ? gmf::OP_X : (b == 1 ? gmf::OP_I : gmf::OP_D), 1);
        k = pk[b];
    }
    e.put(gmf::OP_EQ, H[0]);
    e.flush();
    return true;
}

__global__ void wfa_walk_kernel(WalkArgs A) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n_pairs) return;
    const int n = (int)(A.q_off[p + 1] - A.q_off[p]), m = (int)(A.t_off[p + 1] - A.t_off[p]);
    const int d = A.distance[p];
    const bool trivial = n == 0 || m == 0;
    const long long ho = trivial ? 0 : A.hist_off[p];
    if (d < 0 || ho < 0) {
        if (A.op_counts)
            for (int c = 0; c < 4; ++c) A.op_counts[4 * p + c] = 0;
        A.cigar_start[p] = 0;
        A.cigar_len[p] = -1;
        return;
    }
    Emit e;
    e.init(nullptr, 0);
    if (trivial) {
        e.put(gmf::OP_D, m);  // back to front: the D run follows the I run
        e.put(gmf::OP_I, n);
        e.flush();
    } else if (!wfa_walk(A.hist + ho, d, n - m, e)) {
        atomicOr(A.err, (int)GMF_SWF_INTERNAL);
        if (A.op_counts)
            for (int c = 0; c < 4; ++c) A.op_counts[4 * p + c] = 0;
        A.cigar_start[p] = 0;
        A.cigar_len[p] = -1;
        return;
    }
    const long long words = e.words;
    const unsigned long long at = atomicAdd(A.cigar_used, (unsigned long long)words);
    if (A.op_counts) {
        A.op_counts[4 * p + 0] = e.n_eq;
        A.op_counts[4 * p + 1] = e.n_x;
        A.op_counts[4 * p + 2] = e.n_i;
        A.op_counts[4 * p + 3] = e.n_d;
    }
    if ((long long)at + words > A.cigar_cap) {
        atomicOr(A.err, (int)GMF_SWF_CAPACITY);
        A.cigar_start[p] = 0;
        A.cigar_len[p] = -1;
        return;
    }
    e.init(A.cigar, (long long)at + words);
    if (trivial) {
        e.put(gmf::OP_D, m);
        e.put(gmf::OP_I, n);
        e.flush();
    } else {
        wfa_walk(A.hist + ho, d, n - m, e);
    }
    A.cigar_start[p] = (long long)at;
    A.cigar_len[p] = (int)words;
}

// ---- host side ----------------------------------------------------------------
constexpr size_t ALIGN = 256;
inline size_t up(size_t x) { return (x + ALIGN - 1) & ~(ALIGN - 1); }

// Persistent grid: up to 4 blocks per SM of a B200 (2 when the wavefronts
// may spill to global slots, which are sized per warp).  A fixed SM count
// keeps the workspace size independent of the device queried.
int grid_blocks(int n_pairs, int eff) {
    constexpr long long SMS = 148;
    const long long want = ((long long)n_pairs + WFA_WARPS - 1) / WFA_WARPS;
    const long long cap = SMS * (eff > WFA_SMEM_S ? 2 : WFA_MAX_BLOCKS_PER_SM);
    return (int)(want < cap ? (want > 0 ? want : 1) : cap);
}

// Workspace pieces: [counters | spill slots | history]
struct Ws {
    unsigned* work;
    unsigned long long* hist_used;
    long long* hist_off;
    int* spill;
    int* hist;
    long long hist_cap;
};

size_t fixed_bytes(int n_pairs, int eff, int blocks) {
    size_t b = up(64) + up(sizeof(long long) * (size_t)(n_pairs > 0 ? n_pairs : 1));
    if (eff > WFA_SMEM_S) b += up(sizeof(int) * 2 * (2 * (size_t)eff + 3) * (size_t)blocks * WFA_WARPS);
    return b;
}

int carve(void* ws, size_t bytes, int n_pairs, int eff, int blocks, Ws& w) {
    const size_t need = fixed_bytes(n_pairs, eff, blocks);
    if (!ws || bytes < need) return GMF_ERR_WORKSPACE;
    char* p = (char*)ws;
    w.work = (unsigned*)p;
    w.hist_used = (unsigned long long*)(p + 8);
    p += up(64);
    w.hist_off = (long long*)p;
    p += up(sizeof(long long) * (size_t)(n_pairs > 0 ? n_pairs : 1));
    w.spill = nullptr;
    if (eff > WFA_SMEM_S) {
        w.spill = (int*)p;
        p += up(sizeof(int) * 2 * (2 * (size_t)eff + 3) * (size_t)blocks * WFA_WARPS);
    }
    w.hist = (int*)p;
    w.hist_cap = (long long)((bytes - (size_t)(p - (char*)ws)) / sizeof(int));
    return GMF_OK;
}

int check_pairs(const gmf_wfa_pairs* pairs) {
    if (!pairs || pairs->n_pairs < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->n_pairs == 0) return GMF_OK;
    if (!pairs->query || !pairs->query_off || !pairs->target || !pairs->target_off) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->max_len < 0 || pairs->max_len > GMF_MAX_SEQ_LEN) return GMF_ERR_LIMIT;
    if (pairs->query_total < 0 || pairs->target_total < 0) return GMF_ERR_INVALID_ARGUMENT;
    return GMF_OK;
}

int effective(const gmf_wfa_pairs* pairs, int32_t max_distance) {
    return max_distance < pairs->max_len ? max_distance : pairs->max_len;
}

WfaArgs base_args(const gmf_wfa_pairs* pairs, int32_t max_distance, int eff, const Ws& w, long long q_total,
                  long long t_total) {
    WfaArgs a{};
    a.n_pairs = pairs->n_pairs;
    a.q = pairs->query;
    a.q_off = (const long long*)pairs->query_off;
    a.t = pairs->target;
    a.t_off = (const long long*)pairs->target_off;
    a.order = pairs->order;
    a.Q = make_seq(pairs->query, q_total);
    a.T = make_seq(pairs->target, t_total);
    a.max_distance = max_distance;
    a.eff = eff;
    a.spill = w.spill;
    a.work = w.work;
    a.hist_used = w.hist_used;
    a.hist_off = w.hist_off;
    a.long_len = WFA_LONG_LEN;
    a.long_d = WFA_LONG_D;
    return a;
}

}  // namespace

extern "C" size_t gmf_wfa_workspace_bytes(int32_t n_pairs, int32_t max_len, int32_t max_distance,
                                          int64_t history_entries) {
    if (n_pairs < 0 || max_len < 0 || max_distance < 0 || history_entries < 0) return 0;
    const int eff = max_distance < max_len ? max_distance : max_len;
    return fixed_bytes(n_pairs, eff, grid_blocks(n_pairs, eff)) + up(sizeof(int) * (size_t)history_entries);
}

extern "C" int64_t gmf_wfa_history_entries(int32_t n_pairs, const int32_t* query_len, const int32_t* target_len,
                                           const int32_t* distance) {
    if (n_pairs < 0 || (n_pairs > 0 && (!query_len || !target_len || !distance))) return -1;
    int64_t total = 0;
    for (int32_t p = 0; p < n_pairs; ++p) {
        if (distance[p] < 0 || query_len[p] == 0 || target_len[p] == 0) continue;
        total += (int64_t)(distance[p] + 1) * (distance[p] + 1);
    }
    return total;
}

extern "C" int gmf_wfa_distance(const gmf_wfa_pairs* pairs, int32_t max_distance, int32_t* distance,
                                void* workspace, size_t workspace_bytes, gmf_stream_t stream) {
    GMF_TRY(check_pairs(pairs));
    if (max_distance < 0 || max_distance > GMF_MAX_WFA_DISTANCE) return GMF_ERR_LIMIT;
    if (pairs->n_pairs == 0) return GMF_OK;
    if (!distance) return GMF_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    GMF_BIND_STREAM(st);
    const int eff = effective(pairs, max_distance);
    const int blocks = grid_blocks(pairs->n_pairs, eff);
    Ws w;
    GMF_TRY(carve(workspace, workspace_bytes, pairs->n_pairs, eff, blocks, w));
    WfaArgs a = base_args(pairs, max_distance, eff, w, pairs->query_total, pairs->target_total);
    a.distance = distance;
    GMF_CUDA_TRY(cudaMemsetAsync(w.work, 0, 64, st));
    wfa_forward_kernel<false><<<blocks, WFA_WARPS * 32, 0, st>>>(a);
    return gmf::cuda_status(cudaGetLastError());
}

extern "C" int gmf_wfa_align(const gmf_wfa_pairs* pairs, const int32_t* distance, int32_t max_distance,
                             const gmf_wfa_results* results, void* workspace, size_t workspace_bytes,
                             gmf_stream_t stream) {
    GMF_TRY(check_pairs(pairs));
    if (max_distance < 0 || max_distance > GMF_MAX_WFA_DISTANCE) return GMF_ERR_LIMIT;
    if (pairs->n_pairs == 0) return GMF_OK;
    if (!distance || !results || !results->cigar || !results->cigar_start || !results->cigar_len ||
        !results->cigar_used || !results->error_flags || results->cigar_capacity < 0)
        return GMF_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    GMF_BIND_STREAM(st);
    // the history pass replays each pair to its known distance (<= max_distance)
    const int eff = effective(pairs, max_distance);
    const int blocks = grid_blocks(pairs->n_pairs, eff);
    Ws w;
    GMF_TRY(carve(workspace, workspace_bytes, pairs->n_pairs, eff, blocks, w));
    WfaArgs a = base_args(pairs, max_distance, eff, w, pairs->query_total, pairs->target_total);
    a.distance = const_cast<int*>(distance);
    a.hist = w.hist;
    a.hist_cap = w.hist_cap;
    a.err = results->error_flags;
    GMF_CUDA_TRY(cudaMemsetAsync(w.work, 0, 64, st));
    GMF_CUDA_TRY(cudaMemsetAsync(results->error_flags, 0, sizeof(int32_t), st));
    GMF_CUDA_TRY(cudaMemsetAsync(results->cigar_used, 0, sizeof(unsigned long long), st));
    wfa_forward_kernel<true><<<blocks, WFA_WARPS * 32, 0, st>>>(a);
    GMF_CUDA_TRY(cudaGetLastError());
    WalkArgs b{};
    b.n_pairs = pairs->n_pairs;
    b.q_off = (const long long*)pairs->query_off;
    b.t_off = (const long long*)pairs->target_off;
    b.distance = distance;
    b.hist = w.hist;
    b.hist_off = w.hist_off;
    b.op_counts = results->op_counts;
    b.cigar = results->cigar;
    b.cigar_cap = results->cigar_capacity;
    b.cigar_start = (long long*)results->cigar_start;
    b.cigar_len = results->cigar_len;
    b.cigar_used = results->cigar_used;
    b.err = results->error_flags;
    wfa_walk_kernel<<<(pairs->n_pairs + 127) / 128, 128, 0, st>>>(b);
    return gmf::cuda_status(cudaGetLastError());
}
