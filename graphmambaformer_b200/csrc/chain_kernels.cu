// Anchor chaining for sm_100a: strand split + sort, float64 chaining DP,
// chain peeling and primary/secondary selection.
//
// Semantics (GraphMambaFormer):
//   sort      alignment/types.py L144-152   for_strand (+1 then -1) and
//             sorted_by_ref = stable lexsort by (ref_end, read_end)
//   DP        alignment/chaining.py L129-180 chain_dp_numpy: float64
//             ((f[j] + min(min(dq,dr), w_i)) - pen[|dr-dq|]) [+ bonus],
//             argmax = first maximum (lowest j), taken only if > w_i
//   peel      chaining.py L530-576 _backtrack: argsort(-f, stable), claimed
//             mask, partial score f[i] - f[stop]
//   select    chaining.py L579-617 select + _read_overlap
// The log2 penalty comes from a host table, so the device performs only IEEE
// float64 add / subtract / compare in the reference's order and the results
// are bit-identical.
//
// Layout: one CTA per read for sort and peel/select (shared-memory bitonic
// sort of 64-bit keys + 32-bit tie index; reads too large for shared memory
// sort in their own workspace range), one warp per (read, strand) segment for
// the DP: lanes own anchors and each finished score is broadcast to the
// window (up to 224 predecessors), or, for wider windows, the window sits in
// a shared-memory ring and a warp reduction picks each anchor's predecessor.

#include <float.h>

#include <algorithm>
#include <mutex>

#include "gmf_common.cuh"

namespace gmf {

// ---------------------------------------------------------------------------
// Block-wide bitonic sort of (key, idx) pairs, ascending, ties by idx.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool pair_less(unsigned long long ka, int ia, unsigned long long kb,
                                          int ib) {
    return ka < kb || (ka == kb && ia < ib);
}

__device__ __forceinline__ void bitonic_pair(unsigned long long* key, int* idx, int x, int j, int k) {
    const int y = x | j;  // x has bit j clear
    const bool up = (x & k) == 0;
    const unsigned long long kx = key[x], ky = key[y];
    const int ix = idx[x], iy = idx[y];
    const bool swap = up ? pair_less(ky, iy, kx, ix) : pair_less(kx, ix, ky, iy);
    if (swap) {
        key[x] = ky;
        key[y] = kx;
        idx[x] = iy;
        idx[y] = ix;
    }
}

// Threads take compare-exchange pairs (the p-th index with bit j clear and
// its partner), not elements, so no lane idles.  Stages whose pairs stay
// inside one warp's chunk of the array (j < chunk) need only __syncwarp; only
// the widest strides synchronise the block.  Ends with __syncthreads.
__device__ __forceinline__ void block_bitonic(unsigned long long* key, int* idx, int npow2) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int ch = npow2 / nw;
    if (ch < 64) ch = 64;
    if (ch > npow2) ch = npow2;
    const int n_chunks = npow2 / ch;
    bool block_synced = true;
    for (int k = 2; k <= npow2; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= ch) {
                if (!block_synced) __syncthreads();
                for (int p = threadIdx.x; p < (npow2 >> 1); p += blockDim.x)
                    bitonic_pair(key, idx, ((p & ~(j - 1)) << 1) | (p & (j - 1)), j, k);
                __syncthreads();
                block_synced = true;
            } else {
                for (int c = wid; c < n_chunks; c += nw) {
                    const int base = c * ch;
                    for (int p = lane; p < (ch >> 1); p += 32)
                        bitonic_pair(key, idx, base + (((p & ~(j - 1)) << 1) | (p & (j - 1))), j, k);
                }
                __syncwarp();
                block_synced = false;
            }
        }
    }
    __syncthreads();
}

__host__ __device__ inline int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Order-preserving map of a double onto uint64 (ascending), -0.0 == +0.0.
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    if (v == 0.0) v = 0.0;
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// ---------------------------------------------------------------------------
// Sort: per read, strand +1 anchors then strand -1 anchors, each by
// (ref_end, read_end, original index).
// ---------------------------------------------------------------------------
struct SortArgs {
    int32_t n_reads;
    const int64_t* read_off;
    const int32_t* read_pos;
    const int32_t* ref_pos;
    const int32_t* length;
    const int8_t* strand;
    int32_t* perm;
    int32_t* n_plus;
    int32_t* n_minus;
    int32_t* read_end_s;
    int32_t* ref_end_s;
    unsigned long long* gkey;  // workspace: 2 * n_anchors keys (large reads)
    int* gidx;                 // workspace: 2 * n_anchors indices
    int smem_elems;
    int64_t cap;               // anchors the sorted outputs can hold (-1: caller-sized)
    int64_t key_cap;           // anchors gkey / gidx cover (2 entries each)
    int* err;
};

__global__ void __launch_bounds__(256) chain_sort_kernel(SortArgs a) {
    extern __shared__ unsigned long long sm_keys[];
    const int r = blockIdx.x;
    if (r >= a.n_reads) return;
    const int64_t a0 = a.read_off[r];
    const int n = (int)(a.read_off[r + 1] - a0);
    __shared__ int cnt[2];
    if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
    if (n > GMF_MAX_READ_ANCHORS || (a.cap >= 0 && a.read_off[r + 1] > a.cap)) {
        // too many anchors for one read, or beyond what the workspace holds:
        // the read gets no sorted anchors (so no chains) and the error word says why
        if (threadIdx.x == 0) {
            a.n_plus[r] = 0;
            a.n_minus[r] = 0;
            if (a.err) atomicOr(a.err, n > GMF_MAX_READ_ANCHORS ? 1 : 4);
        }
        return;
    }
    const int np2 = next_pow2(n > 0 ? n : 1);
    unsigned long long* key;
    int* idx;
    if (np2 <= a.smem_elems) {
        key = sm_keys;
        idx = reinterpret_cast<int*>(sm_keys + a.smem_elems);
    } else if (a.gkey && a.gidx && 2 * a0 + np2 <= 2 * a.key_cap) {
        key = a.gkey + 2 * a0;
        idx = a.gidx + 2 * a0;
    } else {
        if (threadIdx.x == 0) {
            a.n_plus[r] = 0;
            a.n_minus[r] = 0;
            if (a.err) atomicOr(a.err, 2);
        }
        return;
    }
    __syncthreads();
    for (int x = threadIdx.x; x < np2; x += blockDim.x) {
        unsigned long long k = ~0ull;
        int ix = 0x7fffffff;
        if (x < n) {
            const int8_t s = a.strand[a0 + x];
            const unsigned long long grp = s == 1 ? 0ull : (s == -1 ? 1ull : 2ull);
            const unsigned re = (unsigned)(a.read_pos[a0 + x] + a.length[a0 + x]);
            const unsigned fe = (unsigned)(a.ref_pos[a0 + x] + a.length[a0 + x]);
            k = (grp << 62) | ((unsigned long long)(fe & 0x7fffffffu) << 31) |
                (unsigned long long)(re & 0x7fffffffu);
            ix = x;
            if (grp < 2) atomicAdd(&cnt[grp], 1);
        }
        key[x] = k;
        idx[x] = ix;
    }
    __syncthreads();
    // the shared-memory call is spelled out so the sort uses shared loads
    if (np2 <= a.smem_elems)
        block_bitonic(sm_keys, reinterpret_cast<int*>(sm_keys + a.smem_elems), np2);
    else
        block_bitonic(key, idx, np2);
    const int m = cnt[0] + cnt[1];
    for (int x = threadIdx.x; x < m; x += blockDim.x) {
        const unsigned long long k = key[x];
        a.perm[a0 + x] = idx[x];
        a.ref_end_s[a0 + x] = (int32_t)((k >> 31) & 0x7fffffffu);
        a.read_end_s[a0 + x] = (int32_t)(k & 0x7fffffffu);
    }
    if (threadIdx.x == 0) {
        a.n_plus[r] = cnt[0];
        a.n_minus[r] = cnt[1];
    }
}

// ---------------------------------------------------------------------------
// Chaining DP: one warp per segment of sorted anchors.
// ---------------------------------------------------------------------------
struct DpArgs {
    // segment source: either explicit rows (row_off) or sorted reads
    int32_t n_segments;
    const int64_t* row_off;   // rows mode
    const int64_t* read_off;  // reads mode
    const int32_t* n_plus;
    const int32_t* n_minus;
    const int32_t* read_end;
    const int32_t* ref_end;
    const double* weight;    // NULL: anchor length (reads mode), via length_s
    const int32_t* length;   // original lengths (reads mode, weight == NULL)
    const int32_t* perm;     // reads mode
    const double* bonus;
    int32_t lookback;
    int32_t max_gap;
    const double* lut;
    int32_t lut_len;
    double* f;
    int32_t* parent;
    int32_t ring;            // ring entries per warp (power of two > lookback)
    int64_t cap;             // reads mode: anchors f / parent hold (-1: caller-sized)
};

__device__ __forceinline__ void seg_range(const DpArgs& a, int s, int64_t& start, int& n) {
    if (a.row_off) {
        start = a.row_off[s];
        n = (int)(a.row_off[s + 1] - start);
    } else {
        const int r = s >> 1;
        const int64_t a0 = a.read_off[r];
        if ((s & 1) == 0) {
            start = a0;
            n = a.n_plus[r];
        } else {
            start = a0 + a.n_plus[r];
            n = a.n_minus[r];
        }
        if (a.cap >= 0 && start + n > a.cap) n = 0;  // beyond the workspace: skipped
    }
}

__global__ void __launch_bounds__(128) chain_dp_kernel(DpArgs a) {
    extern __shared__ double dp_smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int R = a.ring;
    const int mask = R - 1;
    double* rf = dp_smem + (size_t)wib * R * 2;  // f ring, then (read_end, ref_end) as int2
    int2* rc = reinterpret_cast<int2*>(rf + R);
    const int lb = a.lookback > 1 ? a.lookback : 1;
    for (int s = blockIdx.x * wpb + wib; s < a.n_segments; s += gridDim.x * wpb) {
        int64_t st;
        int n;
        seg_range(a, s, st, n);
        int64_t r0 = 0;
        if (!a.row_off) r0 = a.read_off[s >> 1];
        for (int i = 0; i < n; ++i) {
            const int64_t gi = st + i;
            const int qi = a.read_end[gi];
            const int ri = a.ref_end[gi];
            double wi;
            if (a.weight)
                wi = a.weight[gi];
            else
                wi = (double)a.length[r0 + a.perm[gi]];
            const int lo = i - lb > 0 ? i - lb : 0;
            double best = -DBL_MAX;
            int bj = -1;
            bool any = false;
            for (int j = lo + lane; j < i; j += 32) {
                const int2 c = rc[j & mask];
                const int dq = qi - c.x;
                const int dr = ri - c.y;
                double sc;
                if (dq > 0 && dr > 0 && dq <= a.max_gap && dr <= a.max_gap) {
                    any = true;
                    const double mn = (double)(dq < dr ? dq : dr);
                    const double adv = mn < wi ? mn : wi;
                    const int gap = dr > dq ? dr - dq : dq - dr;
                    sc = __dsub_rn(__dadd_rn(rf[j & mask], adv), __ldg(&a.lut[gap]));
                    if (a.bonus) sc = __dadd_rn(sc, __ldg(&a.bonus[gi * lb + (lb - (i - lo)) + (j - lo)]));
                } else {
                    sc = -1e30;
                }
                if (bj < 0 || sc > best) {
                    best = sc;
                    bj = j;
                }
            }
            any = __any_sync(FULL_MASK, any);
            double fi = wi;
            int pi = -1;
            if (any) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double ob = __shfl_xor_sync(FULL_MASK, best, o);
                    const int oj = __shfl_xor_sync(FULL_MASK, bj, o);
                    const bool take = (oj >= 0) && (bj < 0 || ob > best || (ob == best && oj < bj));
                    if (take) {
                        best = ob;
                        bj = oj;
                    }
                }
                if (best > wi) {
                    fi = best;
                    pi = bj;
                }
            }
            if (lane == 0) {
                rf[i & mask] = fi;
                rc[i & mask] = make_int2(qi, ri);
                a.f[gi] = fi;
                a.parent[gi] = pi;
            }
            __syncwarp();
        }
    }
}

// The same recurrence with the anchors owned by lanes: lane l holds anchor
// 32(b+k) + l of K consecutive blocks of 32 (K - 1 blocks cover the window).
// Step t finalises anchor t (its owner's running maximum against w_t),
// broadcasts (f_t, read_end_t, ref_end_t), and every anchor i with
// 1 <= i - t <= lb folds the candidate of predecessor t into its running
// maximum.  Candidates arrive in ascending j and replace the maximum only when
// strictly larger, so the first maximum (lowest j) wins as in the reference;
// each candidate is the same float64 add / subtract.  After 32 steps the
// finished block is stored (coalesced) and the next block is loaded.
template <bool WEIGHT>
__device__ __forceinline__ void dp_load_slot(const DpArgs& a, int64_t st, int64_t r0, int i, int n,
                                             int& q, int& r, double& w, int& wl) {
    if (i < n) {
        const int64_t gi = st + i;
        q = a.read_end[gi];
        r = a.ref_end[gi];
        if (WEIGHT) {
            w = a.weight[gi];
        } else {
            wl = a.length[r0 + a.perm[gi]];
            w = (double)wl;
        }
    } else {
        q = 0;
        r = 0;
        w = 0.0;
        wl = 0;
    }
}

// Every candidate of a step is computed without branches (the table index is
// clamped so that out-of-window pairs read in bounds) and folded in under one
// predicate.  The running maxima start at -inf: the first valid candidate
// (finite) always replaces it, as the reference's first maximum.
template <int K, bool WEIGHT, bool BONUS>
__global__ void __launch_bounds__(128) chain_dp_bcast_kernel(DpArgs a) {
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int lb = a.lookback > 1 ? a.lookback : 1;
    const unsigned mg = a.max_gap > 0 ? (unsigned)a.max_gap : 0u;
    const double* __restrict__ lut = a.lut;
    // reads mode: warps take every read's longer strand first, then the
    // shorter ones, so a block's warps have similar work and the short
    // segments fill the tail
    const int n_reads = a.n_segments >> 1;
    for (int g = blockIdx.x * wpb + wib; g < a.n_segments; g += gridDim.x * wpb) {
        int s = g;
        if (!a.row_off) {
            const int r = g < n_reads ? g : g - n_reads;
            const int minus_longer = a.n_minus[r] > a.n_plus[r] ? 1 : 0;
            s = 2 * r + (g < n_reads ? minus_longer : 1 - minus_longer);
        }
        int64_t st;
        int n;
        seg_range(a, s, st, n);
        if (n <= 0) continue;
        const int64_t r0 = a.row_off ? 0 : a.read_off[s >> 1];
        int q[K], rr[K], bj[K], wl[K];
        double w[K], best[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            dp_load_slot<WEIGHT>(a, st, r0, 32 * k + lane, n, q[k], rr[k], w[k], wl[k]);
            best[k] = -INFINITY;
            bj[k] = -1;
        }
        for (int base = 0; base < n; base += 32) {
            const int steps = n - base < 32 ? n - base : 32;
            bool live[K];
#pragma unroll
            for (int k = 0; k < K; ++k) live[k] = base + 32 * k + lane < n;
            for (int u = 0; u < steps; ++u) {
                const double fo = best[0] > w[0] ? best[0] : w[0];
                const double ft = __shfl_sync(FULL_MASK, fo, u);
                const int qt = __shfl_sync(FULL_MASK, q[0], u);
                const int rt = __shfl_sync(FULL_MASK, rr[0], u);
                const int t = base + u;
                const int lu = lane - u;
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    // a block none of whose anchors reaches back to t is skipped
                    if (32 * k - u > lb) continue;
                    const int d = 32 * k + lu;
                    const int dq = q[k] - qt;
                    const int dr = rr[k] - rt;
                    const bool ok = live[k] && (unsigned)(d - 1) < (unsigned)lb &&
                                    (unsigned)(dq - 1) < mg && (unsigned)(dr - 1) < mg;
                    const int mn = dq < dr ? dq : dr;
                    double adv;
                    if (WEIGHT) {
                        const double mnd = (double)mn;
                        adv = mnd < w[k] ? mnd : w[k];
                    } else {
                        adv = (double)(mn < wl[k] ? mn : wl[k]);
                    }
                    unsigned gap = (unsigned)(dr > dq ? dr - dq : dq - dr);
                    gap = gap < mg ? gap : mg;
                    double sc = __dsub_rn(__dadd_rn(ft, adv), __ldg(&lut[gap]));
                    if (BONUS) {
                        const int64_t bi = ok ? (st + base + 32 * k + lane) * lb + (lb - d) : 0;
                        sc = __dadd_rn(sc, __ldg(&a.bonus[bi]));
                    }
                    if (ok && sc > best[k]) {
                        best[k] = sc;
                        bj[k] = t;
                    }
                }
            }
            if (live[0]) {
                const bool take = best[0] > w[0];
                a.f[st + base + lane] = take ? best[0] : w[0];
                a.parent[st + base + lane] = take ? bj[0] : -1;
            }
#pragma unroll
            for (int k = 0; k + 1 < K; ++k) {
                q[k] = q[k + 1];
                rr[k] = rr[k + 1];
                w[k] = w[k + 1];
                wl[k] = wl[k + 1];
                best[k] = best[k + 1];
                bj[k] = bj[k + 1];
            }
            dp_load_slot<WEIGHT>(a, st, r0, base + 32 * K + lane, n, q[K - 1], rr[K - 1], w[K - 1], wl[K - 1]);
            best[K - 1] = -INFINITY;
            bj[K - 1] = -1;
        }
    }
}

// ---------------------------------------------------------------------------
// Chain peeling + select: one CTA per read.
// ---------------------------------------------------------------------------
struct PeelArgs {
    int32_t n_reads;
    const int64_t* read_off;
    const int32_t* n_plus;
    const int32_t* n_minus;
    const int32_t* perm;
    const int32_t* read_pos;  // original layout
    const int32_t* ref_pos;
    const int32_t* length;
    const double* f;
    const int32_t* parent;
    int32_t min_chain_anchors;
    int32_t max_chains;
    double min_chain_score;
    double secondary_overlap;
    double secondary_score_ratio;
    // workspace (per anchor, in the read's range)
    unsigned long long* gkey;  // 2 * n_anchors
    int* gidx;                 // 2 * n_anchors
    int32_t* mem_tmp;          // walk members (sorted-local indices), all walks
    double* c_score;           // candidate records; during a strand's walk, c_mem /
    int4* c_span;              // c_span hold every walk's (offset, count) / (start, stop)
    int2* c_mem;               // (member offset within read, count)
    int8_t* c_strand;
    int8_t* claimed;           // per anchor: skipped-start flags, then (strands
                               // beyond the shared buffer) claimed flags
    int smem_elems;
    int64_t cap;               // anchors the workspace arrays hold
    // results
    int32_t* n_chains;
    double* score;
    int32_t* strand;
    int32_t* span;
    int32_t* is_primary;
    int32_t* n_members;
    int32_t* members;
};

__global__ void __launch_bounds__(128) chain_peel_kernel(PeelArgs a) {
    extern __shared__ unsigned long long pk_smem[];
    const int r = blockIdx.x;
    if (r >= a.n_reads) return;
    const int64_t a0 = a.read_off[r];
    __shared__ int n_cand;
    __shared__ int n_memtot;
    if (threadIdx.x == 0) {
        n_cand = 0;
        n_memtot = 0;
    }
    const int np = a.n_plus[r], nm = a.n_minus[r];
    const int n_sorted = np + nm;
    if (a0 + n_sorted > a.cap) {  // beyond the workspace (the sort reported it): no chains
        if (threadIdx.x == 0) a.n_chains[r] = 0;
        return;
    }
    __shared__ int n_start;
    __shared__ int n_fill;
    __shared__ int n_walk;
    __shared__ int warp_cnt[4];
    for (int seg = 0; seg < 2; ++seg) {
        const int n = seg == 0 ? np : nm;
        const int s0 = seg == 0 ? 0 : np;  // offset of the segment inside the read
        __syncthreads();
        if (n < a.min_chain_anchors || n == 0) continue;
        const double* fs = a.f + a0 + s0;
        const int32_t* par = a.parent + a0 + s0;
        // Walk starts.  A node with a child of higher score is claimed before
        // its own turn (the child ranks first, and the claimed set is closed
        // under predecessors), so the walk skips it in the reference's order:
        // only the other nodes are ranked.  dom[] marks the skipped nodes.
        int8_t* dom = a.claimed + a0;
        for (int x = threadIdx.x; x < n; x += blockDim.x) dom[x] = 0;
        if (threadIdx.x == 0) {
            n_start = 0;
            n_fill = 0;
        }
        __syncthreads();
        for (int x = threadIdx.x; x < n; x += blockDim.x) {
            const int p = par[x];
            if (p >= 0 && fs[x] > fs[p]) dom[p] = 1;
        }
        __syncthreads();
        const int lane = threadIdx.x & 31;
        const unsigned lt = (1u << lane) - 1u;
        for (int x0 = threadIdx.x & ~31; x0 < n; x0 += blockDim.x) {
            const unsigned b = __ballot_sync(FULL_MASK, x0 + lane < n && !dom[x0 + lane]);
            if (lane == 0 && b) atomicAdd(&n_start, __popc(b));
        }
        __syncthreads();
        const int ns = n_start;
        const int np2 = next_pow2(ns);
        unsigned long long* key;
        int* idx;
        // shared buffer of 12 * smem_elems bytes: keys from the bottom, the
        // sorted indices at the top (they outlive the keys: the walk reads them)
        const bool sort_smem = np2 <= a.smem_elems;
        if (sort_smem) {
            key = pk_smem;
            idx = reinterpret_cast<int*>(reinterpret_cast<char*>(pk_smem) + 12 * a.smem_elems - 4 * np2);
        } else {
            key = a.gkey + 2 * a0;  // np2 <= 2n entries of this read's range
            idx = a.gidx + 2 * a0;
        }
        for (int x0 = threadIdx.x & ~31; x0 < n; x0 += blockDim.x) {
            const int x = x0 + lane;
            const bool st = x < n && !dom[x];
            const unsigned b = __ballot_sync(FULL_MASK, st);
            int base = 0;
            if (lane == 0 && b) base = atomicAdd(&n_fill, __popc(b));
            base = __shfl_sync(FULL_MASK, base, 0);
            if (st) {
                // argsort(-f, stable): ascending -f == descending f, ties by index
                const int slot = base + __popc(b & lt);
                key[slot] = ~ordered_bits(fs[x]);
                idx[slot] = x;
            }
        }
        for (int x = ns + threadIdx.x; x < np2; x += blockDim.x) {
            key[x] = ~0ull;
            idx[x] = 0x7fffffff;
        }
        __syncthreads();
        if (sort_smem)
            block_bitonic(pk_smem,
                          reinterpret_cast<int*>(reinterpret_cast<char*>(pk_smem) + 12 * a.smem_elems - 4 * np2),
                          np2);
        else
            block_bitonic(key, idx, np2);
        __syncthreads();
        const int c_first = n_cand;  // chains found in earlier segments
        // The walk is serial in rank order (the reference's loop): one thread
        // takes the starts in order (the next start's index loaded ahead) and
        // walks the unclaimed ones.  Every walk is recorded -- (member offset,
        // count) and (start, stop node) -- and scored afterwards by the whole
        // block.  The strand's walks claim all n nodes, so its members fill
        // mem_tmp[mem_base, mem_base + n).
        const int mem_base = n_memtot;
        if (6 * n + (sort_smem ? 4 * np2 : 0) <= 12 * a.smem_elems) {
            // shared memory, in the dead sort keys below the sorted starts:
            // pw[x] = predecessor + 1 with bit 31 set once claimed (one load
            // per step of a walk), and the member list (16-bit: n <= 4,096)
            int* pw = reinterpret_cast<int*>(pk_smem);
            unsigned short* ml = reinterpret_cast<unsigned short*>(pw + n);
            for (int x = threadIdx.x; x < n; x += blockDim.x) pw[x] = par[x] + 1;
            __syncthreads();
            if (threadIdx.x == 0) {
                int mo = 0, w = c_first;
                int i_next = idx[0];
                for (int k = 0; k < ns; ++k) {
                    const int i = i_next;
                    if (k + 1 < ns) i_next = idx[k + 1];
                    int v = pw[i];
                    if (v < 0) continue;
                    int m = 0;
                    int node = i;
                    do {
                        pw[node] = v | (int)0x80000000u;
                        ml[mo + m] = (unsigned short)node;
                        ++m;
                        node = v - 1;
                        if (node < 0) break;
                        v = pw[node];
                    } while (v >= 0);
                    a.c_mem[a0 + w] = make_int2(mem_base + mo, m);
                    a.c_span[a0 + w] = make_int4(i, node, 0, 0);
                    ++w;
                    mo += m;
                }
                n_walk = w;
            }
            __syncthreads();
            for (int x = threadIdx.x; x < n; x += blockDim.x) a.mem_tmp[a0 + mem_base + x] = (int)ml[x];
        } else {
            int8_t* claimed = a.claimed + a0;  // held the dom flags
            for (int x = threadIdx.x; x < n; x += blockDim.x) claimed[x] = 0;
            __syncthreads();
            if (threadIdx.x == 0) {
                int mo = 0, w = c_first;
                int i_next = idx[0];
                for (int k = 0; k < ns; ++k) {
                    const int i = i_next;
                    if (k + 1 < ns) i_next = idx[k + 1];
                    if (claimed[i]) continue;
                    int m = 0;
                    int node = i;
                    while (node >= 0) {
                        const int8_t cl = claimed[node];
                        const int nx = par[node];
                        if (cl) break;
                        claimed[node] = 1;
                        a.mem_tmp[a0 + mem_base + mo + m] = node;
                        ++m;
                        node = nx;
                    }
                    a.c_mem[a0 + w] = make_int2(mem_base + mo, m);
                    a.c_span[a0 + w] = make_int4(i, node, 0, 0);
                    ++w;
                    mo += m;
                }
                n_walk = w;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) n_memtot = mem_base + n;
        // candidates: the walks with enough members and a partial score
        // f[start] - f[stop] above the floor, kept in walk order (compacted in
        // place, 256 records at a time: a record moves only to a lower slot)
        {
            const int wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
            const int n_w = n_walk;
            for (int w0 = c_first; w0 < n_w; w0 += blockDim.x) {
                const int w = w0 + threadIdx.x;
                bool keep = false;
                double sc = 0.0;
                int2 cm = make_int2(0, 0);
                if (w < n_w) {
                    cm = a.c_mem[a0 + w];
                    const int4 se = a.c_span[a0 + w];
                    sc = fs[se.x] - (se.y >= 0 ? fs[se.y] : 0.0);
                    keep = cm.y >= a.min_chain_anchors && sc >= a.min_chain_score;
                }
                const unsigned kb = __ballot_sync(FULL_MASK, keep);
                if (lane == 0) warp_cnt[wid] = __popc(kb);
                __syncthreads();
                int slot = n_cand + __popc(kb & lt);
                int tot = 0;
                for (int q = 0; q < nwarp; ++q) {
                    if (q < wid) slot += warp_cnt[q];
                    tot += warp_cnt[q];
                }
                __syncthreads();
                if (keep) {
                    a.c_score[a0 + slot] = sc;
                    a.c_mem[a0 + slot] = cm;
                    a.c_strand[a0 + slot] = (int8_t)(seg == 0 ? 1 : -1);
                }
                if (threadIdx.x == 0) n_cand += tot;
                __syncthreads();
            }
        }
        __syncthreads();
    }
    __syncthreads();
    // ---- select ----
    // The reference sorts the candidates by score (stable) and scans them:
    // the first is kept, and once a chain is kept the scan stops at the
    // first score below cutoff = best * ratio.  Only the first maximum and
    // the candidates at or above the cutoff can be visited before that stop
    // (a scan that has kept nothing by then keeps nothing later either), so
    // only they are sorted and only their spans are computed.
    const int nc = n_cand;
    if (nc == 0) {
        if (threadIdx.x == 0) a.n_chains[r] = 0;
        return;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    __shared__ double red_s[4];  // one entry per warp (at most 128 threads)
    __shared__ int red_i[4];
    __shared__ int4 red_span[4];
    {
        double bs = -INFINITY;
        int bi = 0x7fffffff;
        for (int c = threadIdx.x; c < nc; c += blockDim.x) {
            const double sc = a.c_score[a0 + c];
            if (sc > bs || (sc == bs && c < bi)) {
                bs = sc;
                bi = c;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double os = __shfl_xor_sync(FULL_MASK, bs, o);
            const int oi = __shfl_xor_sync(FULL_MASK, bi, o);
            if (os > bs || (os == bs && oi < bi)) {
                bs = os;
                bi = oi;
            }
        }
        if (lane == 0) {
            red_s[wid] = bs;
            red_i[wid] = bi;
        }
        if (threadIdx.x == 0) {
            n_start = 0;
            n_fill = 0;
        }
    }
    __syncthreads();
    double best_sc = red_s[0];
    int best_c = red_i[0];
    for (int w = 1; w < nw; ++w) {
        if (red_s[w] > best_sc || (red_s[w] == best_sc && red_i[w] < best_c)) {
            best_sc = red_s[w];
            best_c = red_i[w];
        }
    }
    const double cutoff = best_sc * a.secondary_score_ratio;
    for (int x0 = threadIdx.x & ~31; x0 < nc; x0 += blockDim.x) {
        const int c = x0 + lane;
        const bool in = c < nc && (c == best_c || a.c_score[a0 + c] >= cutoff);
        const unsigned b = __ballot_sync(FULL_MASK, in);
        if (lane == 0 && b) atomicAdd(&n_start, __popc(b));
    }
    __syncthreads();
    const int ns = n_start;
    const int np2 = next_pow2(ns);
    const bool sel_smem = np2 <= a.smem_elems;
    unsigned long long* key;
    int* idx;
    if (sel_smem) {
        key = pk_smem;
        idx = reinterpret_cast<int*>(reinterpret_cast<char*>(pk_smem) + 12 * a.smem_elems - 4 * np2);
    } else {
        key = a.gkey + 2 * a0;
        idx = a.gidx + 2 * a0;
    }
    for (int x0 = threadIdx.x & ~31; x0 < nc; x0 += blockDim.x) {
        const int c = x0 + lane;
        const double sc = c < nc ? a.c_score[a0 + c] : 0.0;
        const bool in = c < nc && (c == best_c || sc >= cutoff);
        const unsigned b = __ballot_sync(FULL_MASK, in);
        int base = 0;
        if (lane == 0 && b) base = atomicAdd(&n_fill, __popc(b));
        base = __shfl_sync(FULL_MASK, base, 0);
        if (in) {
            const int slot = base + __popc(b & lt);
            key[slot] = ~ordered_bits(sc);  // sorted(key=-score), stable
            idx[slot] = c;
        }
    }
    for (int x = ns + threadIdx.x; x < np2; x += blockDim.x) {
        key[x] = ~0ull;
        idx[x] = 0x7fffffff;
    }
    __syncthreads();
    if (sel_smem)
        block_bitonic(pk_smem,
                      reinterpret_cast<int*>(reinterpret_cast<char*>(pk_smem) + 12 * a.smem_elems - 4 * np2),
                      np2);
    else
        block_bitonic(key, idx, np2);
    // spans of the sorted candidates over their members' original
    // coordinates, one candidate at a time across the block
    for (int k = 0; k < ns; ++k) {
        const int c = idx[k];
        const int2 cm = a.c_mem[a0 + c];
        const int s0 = a.c_strand[a0 + c] == 1 ? 0 : np;
        int rs = 0x7fffffff, re = -0x7fffffff - 1, fs = 0x7fffffff, fe = -0x7fffffff - 1;
#pragma unroll 4
        for (int x = threadIdx.x; x < cm.y; x += blockDim.x) {
            const int o = a.perm[a0 + s0 + a.mem_tmp[a0 + cm.x + x]];
            const int rp = a.read_pos[a0 + o], fp = a.ref_pos[a0 + o], ln = a.length[a0 + o];
            rs = min(rs, rp);
            re = max(re, rp + ln);
            fs = min(fs, fp);
            fe = max(fe, fp + ln);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rs = min(rs, __shfl_xor_sync(FULL_MASK, rs, o));
            re = max(re, __shfl_xor_sync(FULL_MASK, re, o));
            fs = min(fs, __shfl_xor_sync(FULL_MASK, fs, o));
            fe = max(fe, __shfl_xor_sync(FULL_MASK, fe, o));
        }
        if (lane == 0) red_span[wid] = make_int4(rs, re, fs, fe);
        __syncthreads();
        if (threadIdx.x == 0) {
            int4 sp = red_span[0];
            for (int w = 1; w < nw; ++w) {
                const int4 q = red_span[w];
                sp = make_int4(min(sp.x, q.x), max(sp.y, q.y), min(sp.z, q.z), max(sp.w, q.w));
            }
            a.c_span[a0 + c] = sp;
        }
        __syncthreads();
    }
    __shared__ int kept_c[64];
    __shared__ int n_kept;
    if (threadIdx.x == 0) {
        const int mc = a.max_chains < 64 ? a.max_chains : 64;
        int kept = 0;
        for (int k = 0; k < ns; ++k) {
            const int c = idx[k];
            const double sc = a.c_score[a0 + c];
            if (sc < cutoff && kept) break;
            double overlap = 0.0;
            if (kept) {  // only the first kept chain is primary
                const int4 x = a.c_span[a0 + c];
                const int4 y = a.c_span[a0 + kept_c[0]];
                const int lo = max(x.x, y.x), hi = min(x.y, y.y);
                if (hi > lo) {
                    const int den = max(min(x.y - x.x, y.y - y.x), 1);
                    overlap = (double)(hi - lo) / (double)den;
                }
            }
            if (overlap > a.secondary_overlap) continue;
            kept_c[kept++] = c;
            if (kept >= mc) break;
        }
        n_kept = kept;
        a.n_chains[r] = kept;
    }
    __syncthreads();
    // ---- output: records and members (original indices, read order) ----
    int wpos = 0;
    for (int k = 0; k < n_kept; ++k) {
        const int c = kept_c[k];
        const int2 cm = a.c_mem[a0 + c];
        const int s0 = a.c_strand[a0 + c] == 1 ? 0 : np;
        const size_t slot = (size_t)r * a.max_chains + k;
        if (threadIdx.x == 0) {
            a.score[slot] = a.c_score[a0 + c];
            a.strand[slot] = a.c_strand[a0 + c];
            const int4 sp = a.c_span[a0 + c];
            a.span[4 * slot + 0] = sp.x;
            a.span[4 * slot + 1] = sp.y;
            a.span[4 * slot + 2] = sp.z;
            a.span[4 * slot + 3] = sp.w;
            a.is_primary[slot] = k == 0;
            a.n_members[slot] = cm.y;
        }
        // the walk stored members from chain end to start: reverse to read order
        // four members per thread per round: their loads are issued together
        for (int x0 = threadIdx.x; x0 < cm.y; x0 += 4 * blockDim.x) {
            int loc[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int x = x0 + u * blockDim.x;
                loc[u] = x < cm.y ? a.mem_tmp[a0 + cm.x + (cm.y - 1 - x)] : 0;
            }
            int o[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) o[u] = x0 + u * blockDim.x < cm.y ? a.perm[a0 + s0 + loc[u]] : 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int x = x0 + u * blockDim.x;
                if (x < cm.y) a.members[a0 + wpos + x] = o[u];
            }
        }
        wpos += cm.y;
    }
    (void)n_sorted;
}

}  // namespace gmf

using namespace gmf;

namespace {

// Shared-memory sort buffers: 4096 keys (48 KB) for the per-read sort and
// 2048 (24 KB) for the per-strand peel, so 4 and 8 CTAs fit an SM (the peel's
// serial walk runs in 8 blocks of 4 warps per SM); larger reads / strands
// sort in their own workspace range instead.  The peel buffer also holds a
// strand's walk state (6 bytes per anchor) beside its sorted starts.
int sort_smem_elems() { return 4096; }
int peel_smem_elems() { return 2048; }

size_t sort_smem_bytes(int elems) { return (size_t)elems * (sizeof(unsigned long long) + sizeof(int)); }

int launch_sort(const gmf_anchor_batch* an, const gmf_sorted_anchors* so, unsigned long long* gkey,
                int* gidx, int64_t cap, int64_t key_cap, int* err, cudaStream_t stream) {
    SortArgs s;
    s.n_reads = an->n_reads;
    s.read_off = an->read_off;
    s.read_pos = an->read_pos;
    s.ref_pos = an->ref_pos;
    s.length = an->length;
    s.strand = an->strand;
    s.perm = so->perm;
    s.n_plus = so->n_plus;
    s.n_minus = so->n_minus;
    s.read_end_s = so->read_end;
    s.ref_end_s = so->ref_end;
    s.gkey = gkey;
    s.gidx = gidx;
    s.smem_elems = sort_smem_elems();
    s.cap = cap;
    s.key_cap = key_cap;
    s.err = err;
    const size_t smem = sort_smem_bytes(s.smem_elems);
    GMF_CUDA_TRY(cudaFuncSetAttribute(chain_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    chain_sort_kernel<<<an->n_reads, 256, smem, stream>>>(s);
    return cuda_status(cudaGetLastError());
}

template <int K>
int launch_dp_bcast(const DpArgs& d, int n_segments, cudaStream_t stream) {
    const int wpb = 4;
    const int blocks = (n_segments + wpb - 1) / wpb;
    if (blocks > 0) {
        if (d.weight && d.bonus)
            chain_dp_bcast_kernel<K, true, true><<<blocks, 32 * wpb, 0, stream>>>(d);
        else if (d.weight)
            chain_dp_bcast_kernel<K, true, false><<<blocks, 32 * wpb, 0, stream>>>(d);
        else if (d.bonus)
            chain_dp_bcast_kernel<K, false, true><<<blocks, 32 * wpb, 0, stream>>>(d);
        else
            chain_dp_bcast_kernel<K, false, false><<<blocks, 32 * wpb, 0, stream>>>(d);
    }
    return cuda_status(cudaGetLastError());
}

int launch_dp(DpArgs d, int n_segments, cudaStream_t stream) {
    d.n_segments = n_segments;
    int lb = d.lookback > 1 ? d.lookback : 1;
    // windows up to 224 predecessors: lanes own anchors, K = ceil(lb/32) + 1
    // blocks of 32 in registers
    switch ((lb + 31) / 32 + 1) {
        case 2: return launch_dp_bcast<2>(d, n_segments, stream);
        case 3: return launch_dp_bcast<3>(d, n_segments, stream);
        case 4: return launch_dp_bcast<4>(d, n_segments, stream);
        case 5: return launch_dp_bcast<5>(d, n_segments, stream);
        case 6: return launch_dp_bcast<6>(d, n_segments, stream);
        case 7: return launch_dp_bcast<7>(d, n_segments, stream);
        case 8: return launch_dp_bcast<8>(d, n_segments, stream);
        default: break;
    }
    d.ring = next_pow2(lb + 1);
    const int wpb = 4;
    const size_t smem = (size_t)wpb * d.ring * (sizeof(double) + sizeof(int2));
    GMF_CUDA_TRY(cudaFuncSetAttribute(chain_dp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    const int blocks = (n_segments + wpb - 1) / wpb;
    if (blocks > 0) chain_dp_kernel<<<blocks, 32 * wpb, smem, stream>>>(d);
    return cuda_status(cudaGetLastError());
}

bool valid_lut(const double* lut, int32_t lut_len, int32_t max_gap) {
    return lut != nullptr && lut_len >= max_gap + 1;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

extern "C" int gmf_chain_dp(int32_t n_rows, const int64_t* row_off, const int32_t* read_end,
                            const int32_t* ref_end, const double* weight, const double* bonus,
                            int32_t max_lookback, int32_t max_gap, const double* pen_lut,
                            int32_t lut_len, double* f, int32_t* parent, gmf_stream_t stream) {
    if (n_rows < 0 || max_gap < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (max_lookback > GMF_MAX_LOOKBACK) return GMF_ERR_LIMIT;
    if (n_rows == 0) return GMF_OK;
    if (!row_off || !read_end || !ref_end || !weight || !f || !parent) return GMF_ERR_INVALID_ARGUMENT;
    if (!valid_lut(pen_lut, lut_len, max_gap)) return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    DpArgs d{};
    d.row_off = row_off;
    d.read_end = read_end;
    d.ref_end = ref_end;
    d.weight = weight;
    d.bonus = bonus;
    d.lookback = max_lookback;
    d.max_gap = max_gap;
    d.lut = pen_lut;
    d.lut_len = lut_len;
    d.f = f;
    d.parent = parent;
    return launch_dp(d, n_rows, (cudaStream_t)stream);
}

extern "C" int gmf_chain_sort(const gmf_anchor_batch* an, const gmf_sorted_anchors* so,
                              void* workspace, size_t workspace_bytes, gmf_stream_t stream) {
    if (!an || !so || an->n_reads < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (an->n_reads == 0) return GMF_OK;
    if (!an->read_off || !an->read_pos || !an->ref_pos || !an->length || !an->strand ||
        !so->perm || !so->n_plus || !so->n_minus || !so->read_end || !so->ref_end)
        return GMF_ERR_INVALID_ARGUMENT;
    if (!workspace || workspace_bytes < 256) return GMF_ERR_WORKSPACE;
    GMF_BIND_STREAM(stream);
    // reads too large for shared memory sort in 12 * 2 bytes per anchor of
    // workspace (gmf_chain_workspace_bytes covers it)
    const size_t A = (workspace_bytes - 256) / 24;
    char* p = (char*)workspace;
    int* err = (int*)p;
    unsigned long long* gkey = (unsigned long long*)(p + 256);
    int* gidx = (int*)(p + 256 + align256(2 * A * 8));
    if (256 + align256(2 * A * 8) + 2 * A * 4 > workspace_bytes) {
        gidx = nullptr;
        gkey = nullptr;
    }
    GMF_CUDA_TRY(cudaMemsetAsync(err, 0, 4, (cudaStream_t)stream));
    return launch_sort(an, so, gkey, gidx, -1, (int64_t)A, err, (cudaStream_t)stream);
}

extern "C" size_t gmf_chain_workspace_bytes(int32_t n_reads, int64_t n_anchors) {
    const size_t A = (size_t)(n_anchors > 0 ? n_anchors : 0);
    const size_t R = (size_t)(n_reads > 0 ? n_reads : 0);
    size_t b = 256;                       // error word
    b += align256(2 * A * 8);             // gkey
    b += align256(2 * A * 4);             // gidx
    b += align256(A * 4) * 3;             // perm, read_end_s, ref_end_s
    b += align256(R * 4) * 2;             // n_plus, n_minus
    b += align256(A * 8);                 // f
    b += align256(A * 4);                 // parent
    b += align256(A * 4);                 // mem_tmp
    b += align256(A * 8);                 // c_score
    b += align256(A * 16);                // c_span
    b += align256(A * 8);                 // c_mem
    b += align256(2 * A);                 // c_strand + claimed flags
    return b;
}

extern "C" int gmf_chain_batch(const gmf_anchor_batch* an, const gmf_chain_params* cp,
                               const double* pen_lut, int32_t lut_len,
                               const gmf_sorted_anchors* sorted_in, const double* sorted_weight,
                               const double* sorted_bonus, const gmf_chain_results* res,
                               void* workspace, size_t workspace_bytes, gmf_stream_t stream_) {
    const cudaStream_t stream = (cudaStream_t)stream_;
    if (!an || !cp || !res || an->n_reads < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (cp->max_lookback > GMF_MAX_LOOKBACK) return GMF_ERR_LIMIT;
    if (cp->max_gap < 0 || cp->max_chains < 1 || cp->max_chains > 64) return GMF_ERR_INVALID_ARGUMENT;
    if (an->n_reads == 0) return GMF_OK;
    if (!an->read_off || !an->read_pos || !an->ref_pos || !an->length || !an->strand)
        return GMF_ERR_INVALID_ARGUMENT;
    if (!res->n_chains || !res->score || !res->strand || !res->span || !res->is_primary ||
        !res->n_members || !res->members)
        return GMF_ERR_INVALID_ARGUMENT;
    if (!valid_lut(pen_lut, lut_len, cp->max_gap)) return GMF_ERR_INVALID_ARGUMENT;
    if ((sorted_weight || sorted_bonus) && !sorted_in) return GMF_ERR_INVALID_ARGUMENT;
    if (!workspace) return GMF_ERR_WORKSPACE;
    GMF_BIND_STREAM(stream);

    // the host does not know n_anchors (device CSR); the caller sized the
    // workspace with gmf_chain_workspace_bytes, so derive A from its size.
    // Layout is computed for the largest A that fits.
    const size_t R = (size_t)an->n_reads;
    size_t lo = 0, hi = workspace_bytes;
    while (lo < hi) {  // largest A with bytes(R, A) <= workspace_bytes
        const size_t mid = (lo + hi + 1) / 2;
        if (gmf_chain_workspace_bytes((int32_t)R, (int64_t)mid) <= workspace_bytes)
            lo = mid;
        else
            hi = mid - 1;
    }
    const size_t A = lo;
    char* p = (char*)workspace;
    int* err = (int*)p;
    p += 256;
    auto take = [&](size_t bytes) {
        char* q = p;
        p += align256(bytes);
        return q;
    };
    unsigned long long* gkey = (unsigned long long*)take(2 * A * 8);
    int* gidx = (int*)take(2 * A * 4);
    gmf_sorted_anchors so;
    int32_t* perm_w = (int32_t*)take(A * 4);
    int32_t* re_w = (int32_t*)take(A * 4);
    int32_t* fe_w = (int32_t*)take(A * 4);
    int32_t* npl_w = (int32_t*)take(R * 4);
    int32_t* nmi_w = (int32_t*)take(R * 4);
    double* f = (double*)take(A * 8);
    int32_t* parent = (int32_t*)take(A * 4);
    int32_t* mem_tmp = (int32_t*)take(A * 4);
    double* c_score = (double*)take(A * 8);
    int4* c_span = (int4*)take(A * 16);
    int2* c_mem = (int2*)take(A * 8);
    int8_t* c_strand = (int8_t*)take(2 * A);
    if (sorted_in) {
        so = *sorted_in;
    } else {
        so.perm = perm_w;
        so.n_plus = npl_w;
        so.n_minus = nmi_w;
        so.read_end = re_w;
        so.ref_end = fe_w;
    }
    GMF_CUDA_TRY(cudaMemsetAsync(err, 0, 256, stream));
    int st;
    if (!sorted_in) {
        st = launch_sort(an, &so, gkey, gidx, (int64_t)A, (int64_t)A, err, stream);
        if (st) return st;
    }
    DpArgs d{};
    d.read_off = an->read_off;
    d.n_plus = so.n_plus;
    d.n_minus = so.n_minus;
    d.read_end = so.read_end;
    d.ref_end = so.ref_end;
    d.weight = sorted_weight;
    d.length = an->length;
    d.perm = so.perm;
    d.bonus = sorted_bonus;
    d.lookback = cp->max_lookback;
    d.max_gap = cp->max_gap;
    d.lut = pen_lut;
    d.lut_len = lut_len;
    d.f = f;
    d.parent = parent;
    d.cap = (int64_t)A;
    st = launch_dp(d, 2 * an->n_reads, stream);
    if (st) return st;

    PeelArgs k{};
    k.n_reads = an->n_reads;
    k.read_off = an->read_off;
    k.n_plus = so.n_plus;
    k.n_minus = so.n_minus;
    k.perm = so.perm;
    k.read_pos = an->read_pos;
    k.ref_pos = an->ref_pos;
    k.length = an->length;
    k.f = f;
    k.parent = parent;
    k.min_chain_anchors = cp->min_chain_anchors;
    k.max_chains = cp->max_chains;
    k.min_chain_score = cp->min_chain_score;
    k.secondary_overlap = cp->secondary_overlap;
    k.secondary_score_ratio = cp->secondary_score_ratio;
    k.gkey = gkey;
    k.gidx = gidx;
    k.mem_tmp = mem_tmp;
    k.c_score = c_score;
    k.c_span = c_span;
    k.c_mem = c_mem;
    k.c_strand = c_strand;
    k.claimed = c_strand + A;
    k.smem_elems = peel_smem_elems();
    k.cap = (int64_t)A;
    k.n_chains = res->n_chains;
    k.score = res->score;
    k.strand = res->strand;
    k.span = res->span;
    k.is_primary = res->is_primary;
    k.n_members = res->n_members;
    k.members = res->members;
    const size_t smem = sort_smem_bytes(k.smem_elems);
    GMF_CUDA_TRY(cudaFuncSetAttribute(chain_peel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    chain_peel_kernel<<<an->n_reads, 128, smem, stream>>>(k);
    return cuda_status(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Allocation-free chaining: the scratch is a fixed array of this library.
// ---------------------------------------------------------------------------

// Scratch of gmf_chain_batch_noalloc, one copy per GPU that loads the library.
// Host code must not pass `g_chain_scratch` itself to a kernel (on the host it
// names a stand-in, not device memory); it uses the address looked up below.
static __device__ __align__(256) unsigned char g_chain_scratch[GMF_CHAIN_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxScratchDevices] = {};

// Device address of g_chain_scratch on the current device, looked up once per
// device (the lookup may load this library's module on that device).
int chain_scratch_address(void** out) {
    int dev = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxScratchDevices) return GMF_ERR_LIMIT;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_chain_scratch);
        if (e != cudaSuccess || !p) return GMF_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return GMF_OK;
}

}  // namespace

extern "C" int gmf_chain_batch_noalloc(const gmf_anchor_batch* an, const gmf_chain_params* cp,
                                       const double* pen_lut, int32_t lut_len, int64_t n_anchors,
                                       const gmf_chain_results* res, gmf_stream_t stream) {
    if (!an || !cp || !res || an->n_reads < 0 || n_anchors < 0) return GMF_ERR_INVALID_ARGUMENT;
    const size_t need = gmf_chain_workspace_bytes(an->n_reads, n_anchors);
    if (need > GMF_CHAIN_NOALLOC_SCRATCH_BYTES) return GMF_ERR_LIMIT;
    if (an->n_reads == 0) return GMF_OK;
    GMF_BIND_STREAM(stream);
    void* scratch = nullptr;
    GMF_TRY(chain_scratch_address(&scratch));
    // gmf_chain_batch clears the error word itself; every other scratch array
    // is written before it is read (sort keys, DP values, claimed flags)
    return gmf_chain_batch(an, cp, pen_lut, lut_len, nullptr, nullptr, nullptr, res, scratch, need,
                           stream);
}

extern "C" int gmf_chain_noalloc_error_flags(int32_t* flags, gmf_stream_t stream) {
    if (!flags) return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    void* scratch = nullptr;
    GMF_TRY(chain_scratch_address(&scratch));
    // the error word is the first word of the scratch (gmf_chain_batch's layout)
    return cuda_status(cudaMemcpyAsync(flags, scratch, sizeof(int32_t), cudaMemcpyDefault, (cudaStream_t)stream));
}
