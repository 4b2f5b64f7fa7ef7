// (w, k) minimizer seeding against a device-resident reference index.
//
// Semantics (graphmambaformer/alignment/seeding.py): pack_kmers (L105-132:
// digits = code - 1, a window holding a digit > 3 is invalid and packs to 0,
// Horner packing in int64), hash64 (L83-103: minimap2's invertible 64-bit
// hash over every packed k-mer, invalid ones included), minimizer_mask
// (L172-199: a k-mer is selected when it equals the minimum hash of at least
// one window of w consecutive k-mers, ties all kept, w clipped to the number
// of k-mers), MinimizerIndex.query (L540-545: valid & selected k-mers, in
// read order) and KmerTable.join / lookup (L257-292: every reference position
// of the key, in the table's ascending order).  The index itself (sorted
// unique keys, CSR positions, max_occ applied) is built on the host with the
// same functions and kept on the device.
//
// Layout: one CTA per (read, orientation).  The read (or its reverse
// complement, built on the fly) is processed in tiles of TILE k-mer
// positions: codes of the tile plus halo go to shared memory, each thread
// packs and hashes its positions, the window minima and the selection are
// computed in shared memory, and selected k-mers are looked up by binary
// search in the key table.  Pass 1 counts anchors per (read, orientation);
// pass 2 writes them at the caller's offsets, in the reference's order, with
// a block-wide scan of the per-position counts of each tile.

#include <cub/block/block_scan.cuh>

#include "gmf_common.cuh"

namespace {

constexpr int SEED_THREADS = 256;
constexpr int SEED_TILE = 1024;   // k-mer positions per tile
constexpr int SEED_MAX_K = 31;
constexpr int SEED_MAX_W = 256;

__device__ __forceinline__ unsigned long long mm_hash64(unsigned long long x) {
    x = (~x) + (x << 21);
    x ^= x >> 24;
    x = x + (x << 3) + (x << 8);
    x ^= x >> 14;
    x = x + (x << 2) + (x << 4);
    x ^= x >> 28;
    x = x + (x << 31);
    return x;
}

__device__ __forceinline__ int8_t seq_code(const int8_t* read, int L, int rc, int x) {
    if (!rc) return read[x];
    const int8_t c = read[L - 1 - x];
    return (c >= 1 && c <= 4) ? (int8_t)(5 - c) : c;  // reverse_complement_codes
}

struct SeedArgs {
    int k, w;
    long long n_keys;
    const long long* keys;
    const long long* offsets;
    const int32_t* positions;
    int n_reads;
    const int8_t* codes;
    const long long* read_off;
    int both;
    long long* counts;         // pass 1: 2 per read
    const long long* aoff;     // pass 2: 2 * n_reads + 1
    int32_t* read_pos;
    int32_t* ref_pos;
    int32_t* length;
    int8_t* strand;
};

// First index with keys[i] >= x.
__device__ __forceinline__ long long lower_bound(const long long* keys, long long n, long long x) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

template <bool FILL>
__global__ void __launch_bounds__(SEED_THREADS) seed_kernel(SeedArgs a) {
    using Scan = cub::BlockScan<long long, SEED_THREADS>;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ int8_t s_code[SEED_TILE + 2 * SEED_MAX_W + SEED_MAX_K];
    __shared__ unsigned long long s_hash[SEED_TILE + 2 * SEED_MAX_W];
    __shared__ long long s_pack[SEED_TILE];
    __shared__ unsigned char s_valid[SEED_TILE];
    __shared__ unsigned long long s_wmin[SEED_TILE + SEED_MAX_W];
    __shared__ long long s_total;
    constexpr int PER = SEED_TILE / SEED_THREADS;

    const int k = a.k;
    for (int seg = blockIdx.x; seg < 2 * a.n_reads; seg += gridDim.x) {
        const int r = seg >> 1, rc = seg & 1;
        if (rc && !a.both) {
            if (!FILL && threadIdx.x == 0) a.counts[seg] = 0;
            continue;
        }
        const long long r0 = a.read_off[r];
        const int L = (int)(a.read_off[r + 1] - r0);
        const int8_t* read = a.codes + r0;
        const int m = L - k + 1;  // k-mer positions
        if (threadIdx.x == 0) s_total = 0;
        __syncthreads();
        if (m > 0) {
            const int ww = a.w < 1 ? 1 : (a.w < m ? a.w : m);
            const int n_win = m - ww + 1;
            long long out_base = FILL ? a.aoff[seg] : 0;
            for (int t0 = 0; t0 < m; t0 += SEED_TILE) {
                // hashed positions [h0, h1): windows starting in [t0 - ww + 1, t0 + TILE) and their k-mers
                const int h0 = t0 - ww + 1 > 0 ? t0 - ww + 1 : 0;
                const int h1 = t0 + SEED_TILE + ww - 1 < m ? t0 + SEED_TILE + ww - 1 : m;
                const int c1 = h1 + k - 1;  // codes [h0, c1)
                for (int x = threadIdx.x; x < c1 - h0; x += SEED_THREADS) s_code[x] = seq_code(read, L, rc, h0 + x);
                __syncthreads();
                for (int x = threadIdx.x; x < h1 - h0; x += SEED_THREADS) {
                    long long packed = 0;
                    bool bad = false;
                    for (int o = 0; o < k; ++o) {
                        const long long dg = (long long)s_code[x + o] - 1;
                        bad |= dg > 3;
                        packed = packed * 4 + dg;
                    }
                    if (bad) packed = 0;
                    s_hash[x] = mm_hash64((unsigned long long)packed);
                    const int p = h0 + x;
                    if (p >= t0 && p < t0 + SEED_TILE) {
                        s_pack[p - t0] = packed;
                        s_valid[p - t0] = bad ? 0 : 1;
                    }
                }
                __syncthreads();
                // window minima for windows j in [jw0, jw1)
                const int jw0 = h0, jw1 = (t0 + SEED_TILE < n_win) ? t0 + SEED_TILE : n_win;
                for (int j = jw0 + threadIdx.x; j < jw1; j += SEED_THREADS) {
                    unsigned long long mn = s_hash[j - h0];
                    for (int o = 1; o < ww; ++o) {
                        const unsigned long long v = s_hash[j - h0 + o];
                        mn = v < mn ? v : mn;
                    }
                    s_wmin[j - jw0] = mn;
                }
                __syncthreads();
                // per position: selected & valid -> key lookup -> anchor count
                long long cnt[PER];
                long long kfirst[PER];
#pragma unroll
                for (int e = 0; e < PER; ++e) {
                    const int i = t0 + threadIdx.x * PER + e;
                    cnt[e] = 0;
                    kfirst[e] = 0;
                    if (i < m && s_valid[i - t0]) {
                        const unsigned long long h = s_hash[i - h0];
                        const int jlo = i - ww + 1 > 0 ? i - ww + 1 : 0;
                        const int jhi = i < n_win - 1 ? i : n_win - 1;
                        bool sel = false;
                        for (int j = jlo; j <= jhi && !sel; ++j) sel = s_wmin[j - jw0] == h;
                        if (sel) {
                            const long long key = s_pack[i - t0];
                            const long long at = lower_bound(a.keys, a.n_keys, key);
                            if (at < a.n_keys && __ldg(a.keys + at) == key) {
                                kfirst[e] = __ldg(a.offsets + at);
                                cnt[e] = __ldg(a.offsets + at + 1) - kfirst[e];
                            }
                        }
                    }
                }
                long long excl[PER];
                long long tile_total = 0;
                Scan(scan_tmp).ExclusiveSum(cnt, excl, tile_total);
                if (FILL) {
                    const int8_t sgn = rc ? (int8_t)-1 : (int8_t)1;
#pragma unroll
                    for (int e = 0; e < PER; ++e) {
                        const int i = t0 + threadIdx.x * PER + e;
                        for (long long c = 0; c < cnt[e]; ++c) {
                            const long long o = out_base + excl[e] + c;
                            a.read_pos[o] = i;
                            a.ref_pos[o] = __ldg(a.positions + kfirst[e] + c);
                            a.length[o] = k;
                            a.strand[o] = sgn;
                        }
                    }
                    out_base += tile_total;
                } else if (threadIdx.x == 0) {
                    s_total += tile_total;
                }
                __syncthreads();
            }
        }
        if (!FILL && threadIdx.x == 0) a.counts[seg] = s_total;
        __syncthreads();
    }
}

int check_index(const gmf_minimizer_index* idx) {
    if (!idx || idx->k < 1 || idx->k > SEED_MAX_K || idx->w < 1 || idx->w > SEED_MAX_W || idx->n_keys < 0)
        return GMF_ERR_INVALID_ARGUMENT;
    if (idx->n_keys > 0 && (!idx->keys || !idx->offsets || !idx->positions)) return GMF_ERR_INVALID_ARGUMENT;
    return GMF_OK;
}

SeedArgs seed_args(const gmf_minimizer_index* idx, int32_t n_reads, const int8_t* codes, const int64_t* read_off,
                   int32_t both) {
    SeedArgs a{};
    a.k = idx->k;
    a.w = idx->w;
    a.n_keys = idx->n_keys;
    a.keys = (const long long*)idx->keys;
    a.offsets = (const long long*)idx->offsets;
    a.positions = idx->positions;
    a.n_reads = n_reads;
    a.codes = codes;
    a.read_off = (const long long*)read_off;
    a.both = both ? 1 : 0;
    return a;
}

int seed_grid(int n_reads) {
    const int segs = 2 * n_reads;
    return segs < 148 * 8 ? segs : 148 * 8;
}

}  // namespace

extern "C" int gmf_seed_count(const gmf_minimizer_index* idx, int32_t n_reads, const int8_t* codes,
                              const int64_t* read_off, int32_t both_strands, int64_t* counts, gmf_stream_t stream) {
    GMF_TRY(check_index(idx));
    if (n_reads < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (n_reads == 0) return GMF_OK;
    if (!codes || !read_off || !counts) return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    SeedArgs a = seed_args(idx, n_reads, codes, read_off, both_strands);
    a.counts = (long long*)counts;
    seed_kernel<false><<<seed_grid(n_reads), SEED_THREADS, 0, (cudaStream_t)stream>>>(a);
    return gmf::cuda_status(cudaGetLastError());
}

extern "C" int gmf_seed_fill(const gmf_minimizer_index* idx, int32_t n_reads, const int8_t* codes,
                             const int64_t* read_off, int32_t both_strands, const int64_t* anchor_off,
                             int32_t* read_pos, int32_t* ref_pos, int32_t* length, int8_t* strand,
                             gmf_stream_t stream) {
    GMF_TRY(check_index(idx));
    if (n_reads < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (n_reads == 0) return GMF_OK;
    if (!codes || !read_off || !anchor_off || !read_pos || !ref_pos || !length || !strand)
        return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    SeedArgs a = seed_args(idx, n_reads, codes, read_off, both_strands);
    a.aoff = (const long long*)anchor_off;
    a.read_pos = read_pos;
    a.ref_pos = ref_pos;
    a.length = length;
    a.strand = strand;
    seed_kernel<true><<<seed_grid(n_reads), SEED_THREADS, 0, (cudaStream_t)stream>>>(a);
    return gmf::cuda_status(cudaGetLastError());
}
