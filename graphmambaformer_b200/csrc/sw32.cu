// Banded affine-gap Smith-Waterman with traceback, int32 form (sm_100a).
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
// Layout ("lane-per-row pipeline"): one warp aligns one pair.  Lane k owns
// query rows k+1, k+33, ...; it sweeps the band slots of its row one per
// step, two steps behind lane k-1, so the vertical (d+1) and diagonal (d)
// predecessors from the row above arrive by warp shuffle one and two steps
// after they were produced.  A strip of 32 rows takes P = max(64, W+1)
// steps (slot W is an idle guard step whose outputs are H = 0, F = -inf, the
// reference's guard column); lane 0 of the next strip reads lane 31's outputs
// through a shared-memory delay line of P-64 steps.  The step body has no
// divergent branches.
//
// Traceback bits (4 per cell): H state {stop, diagonal, enter F, enter E},
// "F extends", "E extends".  A gap state extends iff the extend operand of
// its max is strictly larger than the open operand (open > ext; with
// open == ext E never extends, with open < ext ties extend), which is exactly
// traceback_banded's test.  Each lane packs 8 steps per word; the warp stores
// 32 words (128 bytes) every 8 steps.
//
// This form handles any score range; the int16x2 form (sw16.cu) takes the
// pairs whose scores fit 16 bits.  It is also the "plain" per-batch form:
// one warp per pair in input order, one launch per batch.

#include <algorithm>

#include "sw_common.cuh"

namespace gmf {

// Words of traceback bits of one pair (one 32-bit word per lane per 8 steps).
__host__ __device__ inline unsigned long long sw32_tb_words(int qlen, int W) {
    const long long P = W + 1 > 64 ? W + 1 : 64;
    const long long nstrips = (qlen + 31) / 32;
    const long long last = (nstrips - 1) * P + 2 * ((qlen - 1) & 31) + W - 1;
    return (unsigned long long)((last >> 3) + 1) * 32ull;
}

template <bool TB, bool XD, int EM>
__device__ void sw32_pair(const SwArgs& a, int p, const Grp<32>& grp, int2* ring) {
    PairGeo G = load_geo(a, p);
    const int lane = grp.k;
    const int qlen = G.qlen, tlen = G.tlen, W = G.W;
    if (G.hb < 0 || G.hb > a.max_hb) {
        if (lane == 0) write_empty<TB>(a, p, true);
        return;
    }
    if (qlen <= 0 || tlen <= 0) {
        if (lane == 0) write_empty<TB>(a, p, false);
        return;
    }
    const int P = imax(64, W + 1);
    G.P = P;
    const int D = P - 64;
    const int rmask = a.ring - 1;
    const int nstrips = (qlen + 31) >> 5;
    const int last_step = (nstrips - 1) * P + 2 * ((qlen - 1) & 31) + W - 1;

    const unsigned long long tbw = TB ? sw32_tb_words(qlen, W) : 0ull;
    uint32_t* ws = ws_alloc<32>(a, grp, tbw + (XD ? 2ull * qlen : 0ull), TB || XD);
    if ((TB || XD) && !ws) {
        if (lane == 0) write_empty<TB>(a, p, true);
        return;
    }
    uint32_t* bits = ws;
    int2* rowmax = XD ? reinterpret_cast<int2*>(ws + tbw) : nullptr;

    for (int x = lane; x < a.ring; x += 32) ring[x] = make_int2(0, NEG);
    __syncwarp();

    const int match = a.match, mism = a.mismatch, go = a.gap_open, ge = a.gap_extend;
    const int8_t* __restrict__ q = G.q;
    const int8_t* __restrict__ t = G.t;
    int d = -2 * lane;
    int row = lane + 1;
    int j = row + G.off - G.hb + d;
    int qx = 256;
    int hin_d = 0, hin_v = 0, fin_v = NEG;
    int m_l = NEG, e_l = NEG;
    int rb = -1, rbd = 0;
    int lb = 0, lbi = 0, lbd = 0;
    uint32_t acc = 0;

    for (int g = 0; g <= last_step; ++g) {
        const bool live = row <= qlen;
        if (d == 0) {
            const int8_t qc = q[imin(row, qlen) - 1];
            qx = (qc >= 0 && qc != 5) ? (int)(uint8_t)qc : 256;
        }
        const bool inb = live && (unsigned)d < (unsigned)W && (unsigned)(j - 1) < (unsigned)tlen;
        const int tc = inb ? (int)(uint8_t)__ldg(t + (j - 1)) : 0;
        const int sub = (qx == tc) ? match : -mism;
        const int diag = hin_d + sub;
        const int fa = hin_v - go, fb = fin_v - ge;
        int F = imax(fa, fb);
        int M = imax(imax(diag, F), 0);
        const int ea = m_l - go, eb = e_l - ge;
        int E = imax(ea, eb);
        int H = imax(M, E);
        if (TB) {
            const uint32_t code = H > 0 ? (H == diag ? 1u : (H == F ? 2u : 3u)) : 0u;
            const uint32_t fc = fb > fa ? 4u : 0u;
            const uint32_t ec = (EM == 0 ? eb > ea : (EM == 2 && eb >= ea)) ? 8u : 0u;
            const uint32_t nib = inb ? (code | fc | ec) : 0u;
            acc = __funnelshift_r(acc, nib, 4);  // (acc >> 4) | (nib << 28)
            if ((g & 7) == 7) bits[(g >> 3) * 32 + lane] = acc;
        }
        if (!inb) {
            H = 0;
            F = NEG;
            M = NEG;
            E = NEG;
        }
        if (XD) {
            if (d == 0) rb = -1;
            if (H > rb) {
                rb = H;
                rbd = d;
            }
            if (d == W - 1 && live) rowmax[row - 1] = make_int2(rb, rbd);
        } else if (H > lb) {
            lb = H;
            lbi = row;
            lbd = d;
        }
        m_l = M;
        e_l = E;
        if (lane == 31) ring[g & rmask] = make_int2(H, F);
        int nh = __shfl_up_sync(FULL_MASK, H, 1);
        int nf = __shfl_up_sync(FULL_MASK, F, 1);
        __syncwarp();
        if (lane == 0) {
            const int2 r = ring[(g - D) & rmask];
            nh = r.x;
            nf = r.y;
        }
        hin_d = hin_v;
        hin_v = nh;
        fin_v = nf;
        ++d;
        ++j;
        if (d == P) {
            d = 0;
            row += 32;
            j += 32 - P;
        }
    }
    if (TB && (last_step & 7) != 7) bits[(last_step >> 3) * 32 + lane] = acc >> (4 * (7 - (last_step & 7)));
    __syncwarp();

    int bh, bi, bd;
    if (XD) {
        if (lane == 0) record_rowmax(a, p, rowmax);
        xdrop_best<32>(grp, rowmax, qlen, a.x_drop, true, bh, bi, bd);
    } else {
        bh = lb;
        bi = lbi;
        bd = lbd;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int oh = grp.xr(bh, o);
            const int oi = grp.xr(bi, o);
            const int od = grp.xr(bd, o);
            if (oh > bh || (oh == bh && (oi < bi || (oi == bi && od < bd)))) {
                bh = oh;
                bi = oi;
                bd = od;
            }
        }
    }
    const int qe = bh > 0 ? bi : 0;
    const int te = bh > 0 ? bi + G.off - G.hb + bd : 0;
    if (lane == 0) {
        a.score[p] = bh;
        a.q_end[p] = qe;
        a.t_end[p] = te;
    }
    if (!TB) return;
    if (a.defer_walk) {  // the traceback walk runs later, in sw_walk_kernel
        if (lane == 0) record_walk(a, p, bits, 0);
        return;
    }

    RunWriter rw;
    uint32_t* runs = ws_alloc<32>(a, grp, (unsigned long long)qe + te + 1, bh > 0);
    const bool runs_ok = bh == 0 || runs != nullptr;
    if (!runs_ok && lane == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
    rw.init(runs);
    Layout32 lay{bits, P, W, qlen};
    int qs = 0, ts = 0;
    walk<32>(grp, lay, G, a, qe, te, bh, runs_ok && bh > 0, rw, qs, ts);
    finish_cigar<32>(a, grp, p, true, rw, runs_ok, qs, ts);
}

// Plain form: warp w aligns pair order[w] (or w).  Queued form: warps pull
// pairs of class CLS_I32 from the device work queue.
template <bool TB, bool XD, int EM, bool QUEUED>
__global__ void __launch_bounds__(128) sw32_kernel(SwArgs a) {
    extern __shared__ int2 sw32_ring[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    int2* ring = sw32_ring + (size_t)wib * a.ring;
    Grp<32> grp(lane);
    if (QUEUED) {
        const int count = a.queue[N_CLASSES + CLS_I32];
        const int32_t* list = a.lists + (size_t)CLS_I32 * a.n_pairs;
        for (;;) {
            int idx = 0;
            if (lane == 0) idx = atomicAdd(&a.queue[CLS_I32], 1);
            idx = __shfl_sync(FULL_MASK, idx, 0);
            if (idx >= count) break;
            sw32_pair<TB, XD, EM>(a, list[idx], grp, ring);
        }
    } else {
        for (int w = blockIdx.x * wpb + wib; w < a.n_pairs; w += gridDim.x * wpb) {
            const int p = a.order ? a.order[w] : w;
            sw32_pair<TB, XD, EM>(a, p, grp, ring);
        }
    }
}

int sw32_smem_per_warp(int ring) { return ring * (int)sizeof(int2); }

template <bool TB, bool XD, int EM>
static int launch_q(const SwArgs& a, bool queued, int grid, int wpb, cudaStream_t stream) {
    const size_t smem = (size_t)sw32_smem_per_warp(a.ring) * wpb;
    void (*k)(SwArgs) = queued ? sw32_kernel<TB, XD, EM, true> : sw32_kernel<TB, XD, EM, false>;
    if (smem > 48 * 1024)
        GMF_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (queued) {  // persistent grid: every resident block of every SM
        int dev = 0, sms = 0, per_sm = 0;
        GMF_CUDA_TRY(cudaGetDevice(&dev));
        GMF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        GMF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * wpb, smem));
        grid = sms * (per_sm > 0 ? per_sm : 1);
    }
    k<<<grid, 32 * wpb, smem, stream>>>(a);
    return cuda_status(cudaGetLastError());
}

template <bool TB, bool XD>
static int launch_e(const SwArgs& a, int e_mode, bool queued, int grid, int wpb, cudaStream_t s) {
    if (e_mode == 0) return launch_q<TB, XD, 0>(a, queued, grid, wpb, s);
    if (e_mode == 1) return launch_q<TB, XD, 1>(a, queued, grid, wpb, s);
    return launch_q<TB, XD, 2>(a, queued, grid, wpb, s);
}

int launch_sw32(const SwArgs& a, bool tb, bool xd, int e_mode, bool queued, int grid, int wpb,
                cudaStream_t stream) {
    if (tb) return xd ? launch_e<true, true>(a, e_mode, queued, grid, wpb, stream)
                      : launch_e<true, false>(a, e_mode, queued, grid, wpb, stream);
    return xd ? launch_e<false, true>(a, e_mode, queued, grid, wpb, stream)
              : launch_e<false, false>(a, e_mode, queued, grid, wpb, stream);
}

}  // namespace gmf
