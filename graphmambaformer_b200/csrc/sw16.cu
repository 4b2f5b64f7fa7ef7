// Banded affine-gap Smith-Waterman with traceback, int16x2 form (sm_100a).
//
// Same recurrences and traceback decisions as the int32 form (sw32.cu, which
// restates graphmambaformer/alignment/extension.py L78-302); the cells are
// 16-bit and two of them share every 32-bit SIMD instruction.  Only
// instructions that run at full integer rate on sm_100a are used: __vadd2,
// __vsub2, __vmaxs2, the DPX forms __vimax_s16x2_relu / __vimin_s16x2_relu,
// byte permutes, funnel shifts and 32-bit logic.  The 16x2 compares
// (__vcmpeq2 ...) cost about eight instructions each on this part, so every
// comparison is arithmetic instead:
//   match             min(q ^ t, 1) == 0           (codes are small and >= 0)
//   a != b, a >= b    clamp(a - b, 0, 1)           (differences never wrap)
//   strictly larger   (max(a, b) ^ a) != 0
//
// Exactness: "-inf" is -(2*pmax + 2) with pmax = max(mismatch, open, extend),
// every value stays in [-(4*pmax + 2), smax] with smax = match * (min(qlen,
// tlen) + 1), and the classifier only sends pairs with smax + 6*pmax + 64 <=
// 32767 here, so no 16-bit sum or difference ever wraps.
//
// Layout: a pair is aligned by a group of L lanes (L = 8, 16 or 32, so one
// warp aligns 4, 2 or 1 pairs).  Lane k carries two "virtual lanes", 2k in
// the low halves and 2k+1 in the high halves; virtual lane v owns query rows
// v+1, v+1+2L, ... and runs two steps behind virtual lane v-1, exactly like a
// lane of the int32 pipeline.  The low half's inputs from the row above come
// from the high half of lane k-1 (one shuffle + byte permute), the high half's
// from the low half of the same lane.  A strip of 2L rows takes
// P = max(4L, W + 2) steps; virtual lane 0 of the next strip reads the last
// virtual lane's outputs through a shared-memory delay line of P - 4L steps.
//
// Traceback bits: 4 per cell as in the int32 form; each step yields one byte
// (low nibble: low half, high nibble: high half) and every 4 steps the group
// stores one coalesced word per lane.

#include <algorithm>

#include "sw_common.cuh"

namespace gmf {

template <int L>
__host__ __device__ inline unsigned long long sw16_tb_words(int qlen, int W) {
    const long long V = 2 * L;
    const long long P = (W + 2 > 4 * L) ? W + 2 : 4 * L;
    const long long nstrips = (qlen + V - 1) / V;
    const long long last = (nstrips - 1) * P + 2 * ((qlen - 1) % V) + W - 1;
    return (unsigned long long)((last >> 2) + 1) * L;
}

template <int L>
struct Layout16 {
    const uint32_t* bits;
    int P, W, qlen;
    __device__ uint32_t nib(int i, int d) const {
        if (d < 0 || d >= W || i < 1 || i > qlen) return 0u;
        constexpr int V = 2 * L;
        const int v = (i - 1) & (V - 1), s = (i - 1) / V;
        const long long g = (long long)s * P + 2 * v + d;
        const int k = v >> 1, h = v & 1;
        return (bits[(g >> 2) * L + k] >> ((int)(g & 3) * 8 + 4 * h)) & 15u;
    }
};

__device__ __forceinline__ int lo16(unsigned x) { return (int)(short)(x & 0xFFFFu); }
__device__ __forceinline__ int hi16(unsigned x) { return (int)(short)(x >> 16); }
__device__ __forceinline__ unsigned pack16(int lo, int hi) {
    return ((unsigned)lo & 0xFFFFu) | ((unsigned)hi << 16);
}

constexpr unsigned ONE2 = 0x00010001u;

template <int L, bool TB, bool XD, int EM>
__device__ void sw16_group(const SwArgs& a, int p, const Grp<L>& grp, uint32_t* ring) {
    constexpr int V = 2 * L;
    PairGeo G = load_geo(a, p);
    const int k = grp.k;
    const bool has = p >= 0;
    const bool bad = has && (G.hb < 0 || G.hb > a.max_hb);
    bool active = has && !bad && G.qlen > 0 && G.tlen > 0;
    if (has && !active && k == 0) write_empty<TB>(a, p, bad);
    const int qlen = G.qlen, tlen = G.tlen, W = G.W;
    const int P = imax(4 * L, W + 2);
    G.P = P;
    const int D = P - 4 * L;
    const int rmask = a.ring - 1;

    const unsigned long long tbw = (TB && active) ? sw16_tb_words<L>(qlen, W) : 0ull;
    uint32_t* ws = ws_alloc<L>(a, grp, tbw + (XD && active ? 2ull * qlen : 0ull), active && (TB || XD));
    if (active && (TB || XD) && !ws) {
        if (k == 0) write_empty<TB>(a, p, true);
        active = false;
    }
    uint32_t* bits = ws;
    int2* rowmax = (XD && active) ? reinterpret_cast<int2*>(ws + tbw) : nullptr;
    const int nstrips = (qlen + V - 1) / V;
    const int my_last = active ? (nstrips - 1) * P + 2 * ((qlen - 1) % V) + W - 1 : -1;
    const int loop_last = __reduce_max_sync(FULL_MASK, my_last);

    const int neg = a.neg16;
    const unsigned NEG2 = pack16(neg, neg);
    for (int x = k; x < a.ring; x += L) ring[x] = pack16(0, neg);  // H = 0, F = -inf
    __syncwarp();

    const unsigned GO2 = (unsigned)a.gap_open * ONE2;
    const unsigned GE2 = (unsigned)a.gap_extend * ONE2;
    const unsigned GO2P = (unsigned)(a.gap_open + 1) * ONE2;
    const unsigned MATCH2 = (unsigned)a.match * ONE2;
    const unsigned MX = (unsigned)(a.match + a.mismatch);
    const int8_t* __restrict__ q = G.q;
    const int8_t* __restrict__ t = G.t;
    const int c0 = G.off - G.hb;  // j = row + c0 + d
    int d = -4 * k;           // slot of the low half (virtual lane 2k)
    int row = 2 * k + 1;      // row of the low half; the high half is row + 1 at slot d - 2
    int j = row + c0 + d;     // target column of the low half
    unsigned band_lo = ONE2, band_hi = 0u;  // per-half in-band slot interval (in low-half d); empty
    unsigned dp = pack16(d, d);
    unsigned hv = 0u, fv = NEG2, hd = 0u, ml = NEG2, el = NEG2;
    unsigned qp = 0x01000100u;
    unsigned tprev = 0u, acc = 0u;
    unsigned lb2 = 0u;
    int lpos0 = 0, lpos1 = 0;
    unsigned rm2 = 0xFFFFFFFFu;
    int rp0 = 0, rp1 = 0;

    // steps run in chunks of 4 (one traceback word per lane per chunk); the
    // steps past a group's last cell only see out-of-band cells
    const int last_word = my_last >> 2;
    for (int g0 = 0; g0 <= loop_last; g0 += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int g = g0 + u;
        if (d == 0) {
            // both halves start new rows (the high half two steps later, idle until then)
            const int j0 = row + c0;
            const int cq0 = row <= qlen ? (int)q[row - 1] : -1;
            const int cq1 = row + 1 <= qlen ? (int)q[row] : -1;
            qp = pack16((cq0 >= 0 && cq0 != 5) ? cq0 : 0x100, (cq1 >= 0 && cq1 != 5) ? cq1 : 0x100);
            // interval bounds clamped into int16: an empty interval stays empty
            const int lo0 = imin(imax(0, 1 - j0), 32000);
            const int hi0 = row <= qlen ? imax(imin(W - 1, tlen - j0), -1) : -1;
            const int lo1 = imin(imax(2, 2 - j0), 32000);
            const int hi1 = row + 1 <= qlen ? imax(imin(W + 1, tlen - j0 + 1), -1) : -1;
            band_lo = pack16(lo0, lo1);
            band_hi = pack16(hi0, hi1);
            if (XD) rm2 = pack16(-1, hi16(rm2));
        }
        if (XD && d == 2) rm2 = pack16(lo16(rm2), -1);
        // in-band mask: lo <= d <= hi per half (differences are small: no wrap)
        const unsigned outb = (__vsub2(dp, band_lo) | __vsub2(band_hi, dp)) & 0x80008000u;
        const unsigned mask = ((outb ^ 0x80008000u) >> 15) * 0xFFFFu;  // 0xFFFF per in-band half
        const unsigned tc = (unsigned)(j - 1) < (unsigned)tlen ? (unsigned)(uint8_t)__ldg(t + (j - 1)) : 0u;
        const unsigned tp = tc | (tprev << 16);
        tprev = tc;
        const unsigned mis = __vimin_s16x2_relu(qp ^ tp, ONE2);  // 0: match, 1: mismatch
        const unsigned sub = __vsub2(MATCH2, mis * MX);
        const unsigned diag = __vadd2(hd, sub);
        const unsigned fa = __vsub2(hv, GO2), fb = __vsub2(fv, GE2);
        unsigned F = __vmaxs2(fa, fb);
        unsigned M = __vimax_s16x2_relu(diag, F);
        const unsigned ea = __vsub2(ml, GO2), eb = __vsub2(el, GE2);
        unsigned E = __vmaxs2(ea, eb);
        unsigned H = __vmaxs2(M, E);
        if (TB) {
            const unsigned nz = __vimin_s16x2_relu(H, ONE2);                 // H > 0
            const unsigned n1 = __vimin_s16x2_relu(__vsub2(H, diag), ONE2);  // H != diag
            const unsigned n2 = __vimin_s16x2_relu(__vsub2(H, F), ONE2);     // H != F
            const unsigned fc = __vimin_s16x2_relu(__vsub2(fb, fa), ONE2);   // F extends
            unsigned ec = 0u;                                                // E extends
            if (EM == 0) ec = __vimin_s16x2_relu(__vsub2(eb, ea), ONE2);
            if (EM == 2) ec = __vimin_s16x2_relu(__vsub2(el, __vsub2(ml, __vsub2(GO2P, GE2))), ONE2);
            const unsigned b0 = nz & ((n1 ^ ONE2) | n2);   // diagonal or E, when H > 0
            const unsigned b1 = nz & n1;                    // F or E
            unsigned x = b0 + 2u * b1 + 4u * fc + 8u * ec;
            x &= mask;
            const unsigned y = x | (x >> 12);  // low nibble: low half, high nibble: high half
            acc = __funnelshift_r(acc, y, 8);
            if (u == 3 && (g0 >> 2) <= last_word) bits[(g0 >> 2) * L + k] = acc;
        }
        H &= mask;
        F = (F & mask) | (NEG2 & ~mask);
        M = (M & mask) | (NEG2 & ~mask);
        E = (E & mask) | (NEG2 & ~mask);
        if (XD) {
            const unsigned nr = __vmaxs2(rm2, H);
            const unsigned inc = nr ^ rm2;
            rm2 = nr;
            if (inc & 0xFFFFu) rp0 = d;
            if (inc >> 16) rp1 = d - 2;
            if (d == W - 1 && row <= qlen) rowmax[row - 1] = make_int2(lo16(rm2), rp0);
            if (d == W + 1 && row + 1 <= qlen) rowmax[row] = make_int2(hi16(rm2), rp1);
        } else {
            const unsigned nb = __vmaxs2(lb2, H);
            const unsigned inc = nb ^ lb2;
            lb2 = nb;
            if (inc & 0xFFFFu) lpos0 = g;
            if (inc >> 16) lpos1 = g;
        }
        ml = M;
        el = E;
        if (k == L - 1) ring[g & rmask] = __byte_perm(H, F, 0x7632);  // (H.hi, F.hi)
        unsigned sh = grp.up(H, 1), sf = grp.up(F, 1);
        __syncwarp();
        if (k == 0) {
            const unsigned r = ring[(g - D) & rmask];
            sh = r << 16;
            sf = r & 0xFFFF0000u;
        }
        hd = hv;
        hv = __byte_perm(sh, H, 0x5432);  // low: row above (lane k-1 high), high: own low
        fv = __byte_perm(sf, F, 0x5432);
        ++d;
        ++j;
        dp = __vadd2(dp, ONE2);
        if (d == P) {
            d = 0;
            row += V;
            j += V - P;
            dp = 0u;
        }
    }
    }
    __syncwarp();

    int bh, bi, bd;
    if (XD) {
        xdrop_best<L>(grp, rowmax, qlen, a.x_drop, active, bh, bi, bd);
    } else {
        // first cell of each virtual lane's maximum, then the group's best
        const int v0 = lo16(lb2), v1 = hi16(lb2);
        int r0 = 0, s0 = 0, r1 = 0, s1 = 0;
        if (v0 > 0) {
            const int tt = lpos0 - 2 * (2 * k);
            const int s = tt / P;
            r0 = s * V + 2 * k + 1;
            s0 = tt - s * P;
        }
        if (v1 > 0) {
            const int tt = lpos1 - 2 * (2 * k + 1);
            const int s = tt / P;
            r1 = s * V + 2 * k + 2;
            s1 = tt - s * P;
        }
        bh = v0;
        bi = r0;
        bd = s0;
        if (v1 > bh || (v1 == bh && v1 > 0 && (r1 < bi || (r1 == bi && s1 < bd)))) {
            bh = v1;
            bi = r1;
            bd = s1;
        }
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) {
            const int oh = grp.xr(bh, o);
            const int oi = grp.xr(bi, o);
            const int od = grp.xr(bd, o);
            if (oh > bh || (oh == bh && (oi < bi || (oi == bi && od < bd)))) {
                bh = oh;
                bi = oi;
                bd = od;
            }
        }
        if (!active) bh = 0;
    }
    const int qe = bh > 0 ? bi : 0;
    const int te = bh > 0 ? bi + G.off - G.hb + bd : 0;
    if (active && k == 0) {
        a.score[p] = bh;
        a.q_end[p] = qe;
        a.t_end[p] = te;
    }
    if (!TB) return;

    RunWriter rw;
    uint32_t* runs = ws_alloc<L>(a, grp, (unsigned long long)qe + te + 1, active && bh > 0);
    const bool runs_ok = !(active && bh > 0) || runs != nullptr;
    if (!runs_ok && k == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
    rw.init(runs);
    Layout16<L> lay{bits, P, W, qlen};
    int qs = 0, ts = 0;
    walk<L>(grp, lay, G, qe, te, active && runs_ok && bh > 0, rw, qs, ts);
    finish_cigar<L>(a, grp, p, active, rw, runs_ok, qs, ts);
}

template <int L, bool TB, bool XD, int EM>
__global__ void __launch_bounds__(128) sw16_kernel(SwArgs a) {
    extern __shared__ uint32_t sw16_ring[];
    constexpr int GPW = 32 / L;  // pairs per warp
    constexpr int CLS = L == 8 ? CLS_I16_L8 : (L == 16 ? CLS_I16_L16 : CLS_I16_L32);
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gi = lane / L;
    uint32_t* ring = sw16_ring + ((size_t)wib * GPW + gi) * a.ring;
    Grp<L> grp(lane);
    const int count = a.queue[N_CLASSES + CLS];
    const int32_t* list = a.lists + (size_t)CLS * a.n_pairs;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&a.queue[CLS], GPW);
        base = __shfl_sync(FULL_MASK, base, 0);
        if (base >= count) break;
        const int idx = base + gi;
        const int p = idx < count ? list[idx] : -1;
        sw16_group<L, TB, XD, EM>(a, p, grp, ring);
    }
}

int sw16_smem_per_warp(int cls, int ring) {
    const int L = cls == CLS_I16_L8 ? 8 : (cls == CLS_I16_L16 ? 16 : 32);
    return (32 / L) * ring * (int)sizeof(uint32_t);
}

template <int L, bool TB, bool XD, int EM>
static int launch_l(const SwArgs& a, int grid, int wpb, cudaStream_t stream) {
    const int cls = L == 8 ? CLS_I16_L8 : (L == 16 ? CLS_I16_L16 : CLS_I16_L32);
    const size_t smem = (size_t)sw16_smem_per_warp(cls, a.ring) * wpb;
    void (*k)(SwArgs) = sw16_kernel<L, TB, XD, EM>;
    if (smem > 48 * 1024)
        GMF_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {  // persistent grid: every resident block of every SM
        int dev = 0, sms = 0, per_sm = 0;
        GMF_CUDA_TRY(cudaGetDevice(&dev));
        GMF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        GMF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * wpb, smem));
        grid = sms * (per_sm > 0 ? per_sm : 1);
    }
    k<<<grid, 32 * wpb, smem, stream>>>(a);
    return cuda_status(cudaGetLastError());
}

template <int L, bool TB, bool XD>
static int launch_le(const SwArgs& a, int e_mode, int grid, int wpb, cudaStream_t s) {
    if (e_mode == 0) return launch_l<L, TB, XD, 0>(a, grid, wpb, s);
    if (e_mode == 1) return launch_l<L, TB, XD, 1>(a, grid, wpb, s);
    return launch_l<L, TB, XD, 2>(a, grid, wpb, s);
}

template <int L>
static int launch_lx(const SwArgs& a, bool tb, bool xd, int e_mode, int grid, int wpb, cudaStream_t s) {
    if (tb) return xd ? launch_le<L, true, true>(a, e_mode, grid, wpb, s) : launch_le<L, true, false>(a, e_mode, grid, wpb, s);
    return xd ? launch_le<L, false, true>(a, e_mode, grid, wpb, s) : launch_le<L, false, false>(a, e_mode, grid, wpb, s);
}

int launch_sw16(const SwArgs& a, int cls, bool tb, bool xd, int e_mode, int grid, int wpb,
                cudaStream_t stream) {
    if (cls == CLS_I16_L8) return launch_lx<8>(a, tb, xd, e_mode, grid, wpb, stream);
    if (cls == CLS_I16_L16) return launch_lx<16>(a, tb, xd, e_mode, grid, wpb, stream);
    return launch_lx<32>(a, tb, xd, e_mode, grid, wpb, stream);
}

}  // namespace gmf
