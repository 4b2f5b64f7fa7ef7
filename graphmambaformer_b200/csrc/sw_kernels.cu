// Banded affine-gap Smith-Waterman with traceback for sm_100a.
//
// Semantics: graphmambaformer/alignment/extension.py L78-302
// (banded_affine_sw_batch + traceback_banded), applied per pair:
//   band slot d of query row i is target column j = i + off - hb + d;
//   F(i,d) = max(H(i-1,d+1) - open, F(i-1,d+1) - ext)          (vertical)
//   M(i,d) = max(H(i-1,d) + sub, F(i,d), 0)                      (no horizontal gap)
//   E(i,d) = max(M(i,d-1) - open, E(i,d-1) - ext)               (the reference's
//            exclusive cummax of M + d*ext, in recurrence form: identical values)
//   H(i,d) = max(M, E); out-of-band cells: H = 0, M = E = F = -inf;
//   row max with the first slot winning, best updated on a strictly larger
//   row max (earliest row wins), x-drop on (max row max so far) - row max.
// Integer arithmetic is exact, so every decision the reference makes on its
// float32 matrices is reproduced bit for bit.
//
// Parallel layout ("lane-per-row pipeline"): one warp aligns one pair.  Lane
// k owns query rows k+1, k+33, ...; it sweeps the W band slots of its row one
// per step, two steps behind lane k-1, so the vertical (d+1) and diagonal (d)
// predecessors from the row above arrive by warp shuffle exactly one and two
// steps after they were produced.  The last row of a 32-row strip reaches
// lane 0 of the next strip through a one-row shared-memory buffer, so a strip
// takes max(64, W) steps and the pipeline never stalls for W >= 64.
//
// Traceback: each cell stores 4 bits (the decision traceback_banded would
// take in that cell): H-state move {stop, diagonal, to F, to E}, F keeps
// extending, E keeps extending.  Words of 8 cells are written coalesced per
// (strip, 8-slot block, lane) into the workspace, then lane 0 walks them back
// from the best cell and the run-length CIGAR is copied out densely.

#include <algorithm>
#include <vector>

#include "gmf_common.cuh"

namespace gmf {

struct SwArgs {
    const int8_t* q;
    const int64_t* q_off;
    const int8_t* t;
    const int64_t* t_off;
    const int32_t* hb;
    const int32_t* boff;
    const int32_t* order;
    int32_t n_pairs;
    int32_t match, mismatch, gap_open, gap_extend, x_drop;
    int32_t w_max;
    unsigned long long* counters;  // [0] workspace words handed out (bump allocator)
    uint32_t* pool;                // traceback words and CIGAR-run scratch
    unsigned long long pool_cap;   // words
    int32_t* score;
    int32_t* q_end;
    int32_t* t_end;
    int32_t* q_start;
    int32_t* t_start;
    int32_t* op_counts;
    uint32_t* cigar;
    long long cigar_cap;
    int64_t* cigar_start;
    int32_t* cigar_len;
    unsigned long long* cigar_used;
    int32_t* err;
};

__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// Bits word address of cell (row i (1-based), slot d) inside a pair's block.
__device__ __forceinline__ long long tb_index(int i, int d, int nblk) {
    return ((long long)((i - 1) >> 5) * nblk + (d >> 3)) * 32 + ((i - 1) & 31);
}

template <bool TB, bool XD>
__device__ void sw_pair(const SwArgs& a, int p, int lane, int2* rowbuf, int* xs) {
    const int64_t q0 = a.q_off[p], t0 = a.t_off[p];
    const int qlen = (int)(a.q_off[p + 1] - q0);
    const int tlen = (int)(a.t_off[p + 1] - t0);
    const int8_t* __restrict__ q = a.q + q0;
    const int8_t* __restrict__ t = a.t + t0;
    const int hb = a.hb[p];
    const int off = a.boff[p];
    const int W = 2 * hb + 1;

    if (qlen <= 0 || tlen <= 0 || hb < 0 || hb > a.w_max) {
        if (lane == 0) {
            a.score[p] = 0;
            a.q_end[p] = 0;
            a.t_end[p] = 0;
            if (a.q_start) a.q_start[p] = 0;
            if (a.t_start) a.t_start[p] = 0;
            if (a.op_counts)
                for (int k = 0; k < 4; ++k) a.op_counts[4 * p + k] = 0;
            if (TB) {
                a.cigar_start[p] = 0;
                a.cigar_len[p] = (hb < 0 || hb > a.w_max) ? -1 : 0;
            }
            if (hb < 0 || hb > a.w_max) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
        }
        return;
    }

    const int P = imax(64, W);
    const int nstrips = (qlen + 31) >> 5;
    const int nblk = (W + 7) >> 3;

    uint32_t* bits = nullptr;
    bool tb_ok = TB;
    if (TB) {
        const unsigned long long need = (unsigned long long)nstrips * nblk * 32ull;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&a.counters[0], need);
        base = __shfl_sync(FULL_MASK, base, 0);
        if (base + need > a.pool_cap) {
            tb_ok = false;
            if (lane == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
        } else {
            bits = a.pool + base;
        }
    }

    // Row 0 of the reference: H = 0, F = -inf (slot W is the guard column).
    for (int x = lane; x <= W; x += 32) rowbuf[x] = make_int2(0, NEG);
    if (XD) {
        xs[lane] = 0;
        xs[32 + lane] = 0;
    }
    __syncwarp();

    int row = lane + 1;  // current query row (1-based)
    int d = -2 * lane;   // slot of the current row; negative before the lane starts
    int hin_d = 0, hin_v = 0, fin_v = NEG;  // H(i-1,d), H(i-1,d+1), F(i-1,d+1)
    int qx = 256, j0 = 0, dlo = 0, dhi = -1;
    int m_left = NEG, e_left = NEG, h_left = 0;
    int row_best = -1, row_bd = 0;
    int lane_best = 0, lane_bi = 0, lane_bd = 0;
    uint32_t acc = 0;
    const long long last_step = (long long)(nstrips - 1) * P + 2 * ((qlen - 1) & 31) + W - 1;

    for (long long g = 0; g <= last_step; ++g) {
        const bool live = (row <= qlen);
        const bool active = live && d >= 0 && d < W;
        if (d == 0 && live) {
            const int8_t qc = q[row - 1];
            // a query code only matches an equal target code when >= 0 and != N
            qx = (qc >= 0 && qc != 5) ? (int)(uint8_t)qc : 256;
            j0 = row + off - hb;
            dlo = imax(0, 1 - j0);
            dhi = imin(W - 1, tlen - j0);
            m_left = NEG;
            e_left = NEG;
            h_left = 0;
            row_best = -1;
            row_bd = 0;
        }
        int H = 0, F = NEG;
        int stop_now = 0;
        if (active) {
            int M = NEG, E = NEG;
            uint32_t nib = 0;
            if (d >= dlo && d <= dhi) {
                const int tc = (int)(uint8_t)t[j0 + d - 1];
                const int sub = (qx == tc) ? a.match : -a.mismatch;
                const int diag = hin_d + sub;
                F = imax(hin_v - a.gap_open, fin_v - a.gap_extend);
                M = imax(imax(diag, F), 0);
                E = imax(m_left - a.gap_open, e_left - a.gap_extend);
                H = imax(M, E);
                if (TB) {
                    const uint32_t code = (H <= 0) ? 0u : (H == diag ? 1u : (H == F ? 2u : 3u));
                    const uint32_t fc = (d < W - 1) && (F != hin_v - a.gap_open) &&
                                        (F == fin_v - a.gap_extend);
                    const uint32_t ec = (d > 0) && (E != h_left - a.gap_open) &&
                                        (E == e_left - a.gap_extend);
                    nib = code | (fc << 2) | (ec << 3);
                }
            }
            if (H > row_best) {
                row_best = H;
                row_bd = d;
            }
            m_left = M;
            e_left = E;
            h_left = H;
            if (TB) {
                acc |= nib << ((d & 7) * 4);
                if ((d & 7) == 7 || d == W - 1) {
                    if (tb_ok) bits[tb_index(row, d, nblk)] = acc;
                    acc = 0;
                }
            }
            if (d == W - 1) {  // row end: merge the row max (x-drop rule per pair)
                if (XD) {
                    const int pk = (lane + 31) & 31;
                    const int prev_seen = xs[pk];
                    const int prev_stop = xs[32 + pk];
                    int seen = prev_seen, stop = 1;
                    if (!prev_stop) {
                        if (row_best > lane_best) {
                            lane_best = row_best;
                            lane_bi = row;
                            lane_bd = row_bd;
                        }
                        seen = imax(prev_seen, row_best);
                        stop = (seen - row_best > a.x_drop) ? 1 : 0;
                        stop_now = stop;
                    }
                    xs[lane] = seen;
                    xs[32 + lane] = stop;
                } else if (row_best > lane_best) {
                    lane_best = row_best;
                    lane_bi = row;
                    lane_bd = row_bd;
                }
            }
        }
        // hand the cell to the lane below (lane 31 -> next strip via rowbuf)
        if (lane == 31 && active) rowbuf[d] = make_int2(H, F);
        const int nh = __shfl_up_sync(FULL_MASK, active ? H : 0, 1);
        const int nf = __shfl_up_sync(FULL_MASK, active ? F : NEG, 1);
        int dn = d + 1;
        if (dn == P) {
            dn = 0;
            row += 32;
        }
        __syncwarp();
        if (XD && __any_sync(FULL_MASK, stop_now)) break;
        if (lane == 0) {
            if (dn < W) {
                const int2 a0 = rowbuf[dn];
                const int2 a1 = rowbuf[dn + 1];
                hin_d = a0.x;
                hin_v = a1.x;
                fin_v = a1.y;
            }
        } else {
            hin_d = hin_v;
            hin_v = nh;
            fin_v = nf;
        }
        d = dn;
    }

    // best cell: max score, then earliest row, then lowest slot
    int bh = lane_best, bi = lane_bi, bd = lane_bd;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int oh = __shfl_xor_sync(FULL_MASK, bh, o);
        const int oi = __shfl_xor_sync(FULL_MASK, bi, o);
        const int od = __shfl_xor_sync(FULL_MASK, bd, o);
        if (oh > bh || (oh == bh && (oi < bi || (oi == bi && od < bd)))) {
            bh = oh;
            bi = oi;
            bd = od;
        }
    }
    const int qe = bh > 0 ? bi : 0;
    const int te = bh > 0 ? bi + off - hb + bd : 0;
    if (lane == 0) {
        a.score[p] = bh;
        a.q_end[p] = qe;
        a.t_end[p] = te;
    }
    if (!TB) return;

    // ---- traceback (lane 0 walks, the warp copies the CIGAR out) ----
    int nruns = 0, qs = 0, ts = 0;
    int cnt[4] = {0, 0, 0, 0};
    uint32_t* runs = nullptr;
    bool runs_ok = tb_ok;
    if (tb_ok && bh > 0) {
        const unsigned long long need = (unsigned long long)qlen + tlen + 1;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&a.counters[0], need);
        base = __shfl_sync(FULL_MASK, base, 0);
        if (base + need > a.pool_cap) {
            runs_ok = false;
            if (lane == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
        } else {
            runs = a.pool + base;
        }
    }
    __syncwarp();  // traceback words written by every lane are visible to lane 0
    if (lane == 0 && runs_ok && bh > 0) {
        int i = qe, j = te, state = 0;
        int cur_op = -1, cur_len = 0;
        while (i > 0 && j > 0) {
            const int dd = j - i - off + hb;
            uint32_t nib = 0;
            if (dd >= 0 && dd < W) nib = (bits[tb_index(i, dd, nblk)] >> ((dd & 7) * 4)) & 15u;
            int op;
            if (state == 0) {
                const uint32_t code = nib & 3u;
                if (code == 0) break;
                if (code != 1) {
                    state = (code == 2) ? 1 : 2;
                    continue;
                }
                const int8_t qc = q[i - 1], tc = t[j - 1];
                op = (qc == tc && qc >= 0 && qc != 5) ? (int)OP_EQ : (int)OP_X;
                --i;
                --j;
            } else if (state == 1) {
                op = OP_I;
                --i;
                state = ((nib >> 2) & 1u) ? 1 : 0;
            } else {
                op = OP_D;
                --j;
                state = ((nib >> 3) & 1u) ? 2 : 0;
            }
            ++cnt[op];
            if (op == cur_op) {
                ++cur_len;
            } else {
                if (cur_len) runs[nruns++] = ((uint32_t)cur_len << 4) | (uint32_t)cur_op;
                cur_op = op;
                cur_len = 1;
            }
        }
        if (cur_len) runs[nruns++] = ((uint32_t)cur_len << 4) | (uint32_t)cur_op;
        qs = i;
        ts = j;
    }
    nruns = __shfl_sync(FULL_MASK, nruns, 0);
    unsigned long long cbase = 0;
    bool fits = runs_ok;
    if (runs_ok && nruns > 0) {
        if (lane == 0) cbase = atomicAdd(a.cigar_used, (unsigned long long)nruns);
        cbase = __shfl_sync(FULL_MASK, cbase, 0);
        if (cbase + nruns > (unsigned long long)a.cigar_cap) {
            fits = false;
            if (lane == 0) atomicOr(a.err, (int)GMF_SWF_CAPACITY);
        }
    }
    __syncwarp();
    if (fits)
        for (int x = lane; x < nruns; x += 32) a.cigar[cbase + x] = runs[nruns - 1 - x];
    if (lane == 0) {
        if (a.q_start) a.q_start[p] = qs;
        if (a.t_start) a.t_start[p] = ts;
        if (a.op_counts)
            for (int k = 0; k < 4; ++k) a.op_counts[4 * p + k] = cnt[k];
        a.cigar_start[p] = (int64_t)cbase;
        a.cigar_len[p] = fits ? nruns : -1;
    }
}

template <bool TB, bool XD>
__global__ void __launch_bounds__(128) sw_warp_kernel(SwArgs a) {
    extern __shared__ int smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    int2* rowbuf = reinterpret_cast<int2*>(smem) + (size_t)wib * (2 * a.w_max + 2);
    int* xs = smem + (size_t)wpb * (2 * a.w_max + 2) * 2 + wib * 64;
    for (int w = blockIdx.x * wpb + wib; w < a.n_pairs; w += gridDim.x * wpb) {
        const int p = a.order ? a.order[w] : w;
        sw_pair<TB, XD>(a, p, lane, rowbuf, xs);
    }
}

static size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

}  // namespace gmf

using namespace gmf;

extern "C" size_t gmf_banded_sw_workspace_bytes(int32_t n_pairs, const int32_t* qlen,
                                                const int32_t* tlen, const int32_t* half_band,
                                                int32_t with_traceback) {
    size_t bits = 0, runs = 0;
    if (with_traceback && n_pairs > 0 && qlen && tlen && half_band) {
        for (int32_t p = 0; p < n_pairs; ++p) {
            const size_t W = 2 * (size_t)std::max(half_band[p], 0) + 1;
            const size_t strips = ((size_t)std::max(qlen[p], 0) + 31) / 32;
            bits += strips * ((W + 7) / 8) * 32;
            runs += (size_t)std::max(qlen[p], 0) + (size_t)std::max(tlen[p], 0) + 1;
        }
    }
    return 256 + round_up((bits + runs) * 4, 256);
}

extern "C" int gmf_banded_sw(const gmf_pairs* pairs, const gmf_sw_params* params,
                             const gmf_sw_results* res, void* workspace, size_t workspace_bytes,
                             gmf_stream_t stream_) {
    if (!pairs || !params || !res) return GMF_ERR_INVALID_ARGUMENT;
    const cudaStream_t stream = (cudaStream_t)stream_;
    if (pairs->n_pairs < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->max_half_band < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->max_half_band > GMF_MAX_HALF_BAND) return GMF_ERR_LIMIT;
    const int lim = 1 << 20;
    if (params->match_score <= 0 || params->match_score > lim || params->mismatch_penalty < 0 ||
        params->mismatch_penalty > lim || params->gap_open < 0 || params->gap_open > lim ||
        params->gap_extend < 0 || params->gap_extend > lim)
        return GMF_ERR_INVALID_ARGUMENT;
    const bool tb = res->cigar != nullptr;
    if (!res->score || !res->query_end || !res->target_end || !res->cigar_used || !res->error_flags)
        return GMF_ERR_INVALID_ARGUMENT;
    if (tb && (!res->cigar_start || !res->cigar_len || res->cigar_capacity < 0))
        return GMF_ERR_INVALID_ARGUMENT;
    if (pairs->n_pairs > 0 && (!pairs->query || !pairs->query_off || !pairs->target ||
                               !pairs->target_off || !pairs->half_band || !pairs->band_offset))
        return GMF_ERR_INVALID_ARGUMENT;
    if (!workspace || workspace_bytes < 256) return GMF_ERR_WORKSPACE;
    GMF_TRY(bind_stream_device(stream));

    GMF_CUDA_TRY(cudaMemsetAsync(workspace, 0, 256, stream));
    GMF_CUDA_TRY(cudaMemsetAsync(res->cigar_used, 0, sizeof(unsigned long long), stream));
    GMF_CUDA_TRY(cudaMemsetAsync(res->error_flags, 0, sizeof(int32_t), stream));
    if (pairs->n_pairs == 0) return GMF_OK;

    SwArgs a;
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
    a.w_max = pairs->max_half_band;  // rowbuf holds W+1 <= 2*max_half_band+2 entries
    a.counters = (unsigned long long*)workspace;
    a.pool = (uint32_t*)((char*)workspace + 256);
    a.pool_cap = tb ? (workspace_bytes - 256) / 4 : 0;
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

    const size_t per_warp = (size_t)(2 * a.w_max + 2) * sizeof(int2) + 64 * sizeof(int);
    int dev = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    int smem_optin = 0;
    GMF_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    int wpb = 4;
    while (wpb > 1 && per_warp * wpb > (size_t)smem_optin) --wpb;
    if (per_warp > (size_t)smem_optin) return GMF_ERR_LIMIT;
    const size_t smem = per_warp * wpb;
    const int blocks = (pairs->n_pairs + wpb - 1) / wpb;
    const bool xd = params->x_drop > 0;
    void (*kern)(SwArgs) = tb ? (xd ? sw_warp_kernel<true, true> : sw_warp_kernel<true, false>)
                              : (xd ? sw_warp_kernel<false, true> : sw_warp_kernel<false, false>);
    if (smem > 48 * 1024)
        GMF_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<blocks, 32 * wpb, smem, stream>>>(a);
    return cuda_status(cudaGetLastError());
}
