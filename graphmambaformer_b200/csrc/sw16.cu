// Banded affine-gap Smith-Waterman with traceback, biased unsigned 16x2 form
// (sm_100a).
//
// Same recurrences and traceback decisions as the int32 form (sw32.cu, which
// restates graphmambaformer/alignment/extension.py L78-302); the cells are
// 16-bit and two of them share every 32-bit SIMD instruction.
//
// Biased cells.  Every value is stored as v + Z with Z = 4*pmax + 2 (pmax =
// the largest penalty), so the biased "-inf" N = Z - (2*pmax + 2) = 2*pmax is
// still >= 0 and every value the recurrences form stays in [pmax, smax + Z]
// with smax = match * (min(qlen, tlen) + 1).  The classifier sends a pair here
// only when smax + Z + 2*pmax + 64 <= 65535, so all cells are exact unsigned
// 16-bit integers and the local-alignment floor is a three-way max with Z.
// Only full-rate instructions are used: __vadd2 / __vsub2, the DPX
// __viaddmax_u16x2 / __viaddmin_u16x2 / __vimax3_u16x2, byte permutes, funnel
// shifts and 32-bit integer ops.  Comparisons are differences of values known
// to be ordered (H >= M >= diag, H >= F, F >= fa, E >= ea, E >= eb), turned
// into 0/1 flags with min(x, 1).
//
// Layout: a pair is aligned by a group of L lanes (L = 8, 16 or 32, so one
// warp aligns 4, 2 or 1 pairs).  Lane k carries two "virtual lanes", 2k in the
// low halves and 2k+1 in the high halves; virtual lane v owns query rows v+1,
// v+1+2L, ... and runs two steps behind virtual lane v-1.  The low half's
// inputs from the row above come from the high half of lane k-1 through ONE
// shuffle of the packed word (H.hi, F.hi); the high half's come from the low
// half of the same lane.  A strip of 2L rows takes P = sw16_period(W, L)
// steps, a multiple of 4; the first lane of the next strip reads the last
// lane's outputs through a shared-memory delay line of D = P - 4L steps
// (a rotation of the same shuffle when D = 0).
//
// Steps run in chunks of 4, and rows always start on a chunk boundary, so
// once per chunk a lane: reads one word of target codes (a sliding window,
// prefetched two chunks ahead), exchanges 4 delay-line entries with one
// 16-byte shared-memory access, stores one 32-bit traceback word (4 bits per
// cell: low half's 4 steps in bits 15..0, high half's in bits 31..16, the
// chunk's first step in the top nibble), and checks the chunk's maxima for
// the best cell (the first maximum in row-then-slot order is recovered from
// the chunk's 4 kept H values when the maximum grows).

#include <algorithm>

#include "sw_common.cuh"

namespace gmf {

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
        return (bits[(g >> 2) * L + k] >> (16 * h + 4 * (3 - (int)(g & 3)))) & 15u;
    }
};

__device__ __forceinline__ int lo16(unsigned x) { return (int)(x & 0xFFFFu); }
__device__ __forceinline__ int hi16(unsigned x) { return (int)(x >> 16); }
__device__ __forceinline__ unsigned pack16(int lo, int hi) {
    return ((unsigned)lo & 0xFFFFu) | ((unsigned)hi << 16);
}

constexpr unsigned ONE2 = 0x00010001u;

// Unsigned 16x2 max / min(x, 1) through the DPX add-max / add-min forms,
// which issue at the full integer rate (the plain __vmaxu2 / __vminu2 do not).
__device__ __forceinline__ unsigned umax2(unsigned a, unsigned b) { return __viaddmax_u16x2(a, 0u, b); }
__device__ __forceinline__ unsigned flag2(unsigned x) { return __viaddmin_u16x2(x, 0u, ONE2); }

// Selectors building the packed target codes of one step from the chunk's
// window (bytes 0..3) and the previous chunk's last code (byte 6): low half =
// this step's code, high half = the previous step's code, zero-extended.
__device__ __forceinline__ unsigned tsel(int u) {
    return u == 0 ? 0x4640u : (u == 1 ? 0x4041u : (u == 2 ? 0x4142u : 0x4243u));
}

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
    const int P = sw16_period(W, L);
    G.P = P;
    const int D = P - 4 * L;  // delay-line steps, a multiple of 4
    const bool use_ring = D > 0;
    const int rmask = a.ring - 1;

    const unsigned long long tbw = (TB && active) ? sw16_tb_words_l(qlen, W, L) : 0ull;
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
    const int last_chunk = my_last >> 2;  // -1 when inactive

    const unsigned Z = (unsigned)a.zero16, NEGV = (unsigned)a.neg16;
    const unsigned Z2 = Z * ONE2, NEG2 = NEGV * ONE2;
    const unsigned GO2 = (unsigned)a.gap_open * ONE2;
    const unsigned GE2 = (unsigned)a.gap_extend * ONE2;
    const unsigned MATCH2 = (unsigned)a.match * ONE2;
    const unsigned NGE2 = ((0x10000u - (unsigned)a.gap_extend) & 0xFFFFu) * ONE2;  // -ext mod 2^16
    const unsigned NZ2 = ((0x10000u - Z) & 0xFFFFu) * ONE2;                        // -zero mod 2^16
    const unsigned MX = (unsigned)(a.match + a.mismatch);
    for (int x = k; x < a.ring; x += L) ring[x] = Z | (NEGV << 16);  // row 0: H = 0, F = -inf
    __syncwarp();

    // target codes: 32-bit words of the whole target buffer, indexed from its
    // first aligned word; the window of a chunk is a funnel shift of two words
    const long long tbase = (long long)(uintptr_t)a.t & ~3ll;
    const long long t_total = active ? a.t_off[a.n_pairs] : 1;  // codes in the buffer
    const long long tend = (long long)(uintptr_t)a.t + t_total;  // one past the last code
    const long long nw64 = ((tend - 1 - tbase) >> 2) + 1;
    const int nwords = nw64 > 0x7fffffffll ? 0x7fffffff : (int)nw64;
    const uint32_t* tw32 = reinterpret_cast<const uint32_t*>((uintptr_t)tbase);
    const long long pair_t = (long long)(uintptr_t)G.t - tbase;  // byte offset of the pair's codes

    const int8_t* __restrict__ q = G.q;
    const int c0 = G.off - G.hb;  // j = row + c0 + d
    int d = -4 * k;               // slot of the low half at the chunk start
    int row = 2 * k + 1 - V;      // row of the low half (advanced by V at each row start)
    unsigned ma = pack16(-30000, -30000), mb = 0u;  // slot - band_lo, band_hi - slot (per half)
    unsigned qp = 0x01000100u;
    unsigned hv = Z2, fv = NEG2, hd = Z2, ml = NEG2, el = NEG2;
    unsigned w0 = 0u, w1 = 0u, w2 = 0u, tpv = 0u;
    int wi = 0, tsh = 0;
    unsigned acc = 0u;
    unsigned lb = Z2;  // best H so far per half (non-x-drop) / row max (x-drop)
    int pos0 = 0, pos1 = 0;
    unsigned rv0 = 0u, rv1 = 0u, rv2 = 0u, rv3 = 0u;  // delay-line entries of the chunk
    const int src = (k + L - 1) & (L - 1);
    const int dW0 = (W - 1) & ~3, dW1 = (W + 1) & ~3;  // chunks that end a row (x-drop)

    for (int g0 = 0; g0 <= loop_last; g0 += 4) {
        if (d == 0) {  // both halves start new rows (the high half two steps later)
            row += V;
            const int j0 = row + c0;
            const int cq0 = row <= qlen ? (int)q[row - 1] : -1;
            const int cq1 = row + 1 <= qlen ? (int)q[row] : -1;
            qp = pack16((cq0 >= 0 && cq0 != 5) ? cq0 : 0x100, (cq1 >= 0 && cq1 != 5) ? cq1 : 0x100);
            // interval bounds clamped into int16: an empty interval stays empty
            const int lo0 = imin(imax(0, 1 - j0), 32000);
            const int hi0 = row <= qlen ? imax(imin(W - 1, tlen - j0), -1) : -1;
            const int lo1 = imin(imax(2, 2 - j0), 32000);
            const int hi1 = row + 1 <= qlen ? imax(imin(W + 1, tlen - j0 + 1), -1) : -1;
            ma = pack16(-1 - lo0, -1 - lo1);
            mb = pack16(hi0 + 1, hi1 + 1);
            // target window at code index j0 - 1 of the pair (words outside the
            // buffer are clamped: they only feed out-of-band cells)
            const long long off = pair_t + (long long)(j0 - 1);
            tsh = (int)(off & 3) * 8;
            wi = (int)(off >> 2);
            if (active) {
                w0 = __ldg(tw32 + imin(imax(wi, 0), nwords - 1));
                w1 = __ldg(tw32 + imin(imax(wi + 1, 0), nwords - 1));
                w2 = __ldg(tw32 + imin(imax(wi + 2, 0), nwords - 1));
            }
            tpv = 0u;
            if (XD) {
                lb = Z2;
                pos0 = 0;
                pos1 = 0;
            }
        }
        if (use_ring && k == 0) {
            const uint4 r = *reinterpret_cast<const uint4*>(ring + ((g0 - D) & rmask));
            rv0 = r.x;
            rv1 = r.y;
            rv2 = r.z;
            rv3 = r.w;
        }
        const unsigned tw = __funnelshift_r(w0, w1, tsh);
        unsigned hk0, hk1, hk2, hk3, pk0, pk1, pk2, pk3;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const unsigned tp = prmt(tw, tpv, tsel(u));
            const unsigned mis = flag2(qp ^ tp);  // 0: match, 1: mismatch
            const unsigned diag = __vadd2(hd, __vsub2(MATCH2, mis * MX));
            const unsigned fa = __vsub2(hv, GO2);
            unsigned F = __viaddmax_u16x2(fv, NGE2, fa);  // max(F above - ext, H above - open)
            unsigned M = __vimax3_u16x2(diag, F, Z2);
            const unsigned ea = __vsub2(ml, GO2);
            unsigned E = __viaddmax_u16x2(el, NGE2, ea);
            unsigned H = umax2(M, E);
            if (TB) {
                const unsigned nz = __viaddmin_u16x2(H, NZ2, ONE2);  // H > 0
                const unsigned n1 = flag2(__vsub2(H, diag));         // H != diag
                const unsigned n2 = flag2(__vsub2(H, F));            // H != F
                const unsigned fc = flag2(__vsub2(F, fa));           // F extends
                unsigned ec = 0u;                                    // E extends
                if (EM == 0) ec = flag2(__vsub2(E, ea));
                if (EM == 2) ec = flag2(__vsub2(E, __vsub2(el, GE2))) ^ ONE2;
                const unsigned b0 = nz & (~n1 | n2);  // diagonal or E, when H > 0
                const unsigned b1 = nz & n1;          // F or E
                const unsigned x = b0 + 2u * b1 + 4u * fc + 8u * ec;
                acc = u == 0 ? x : acc * 16u + x;
            }
            // in-band mask: slot - lo >= 0 and hi - slot >= 0 per half
            ma = __vadd2(ma, ONE2);
            mb = __vsub2(mb, ONE2);
            const unsigned m = prmt(ma | mb, 0u, 0xBB99u);  // 0xFFFF per out-of-band half
            H = (H & ~m) | (Z2 & m);
            F = (F & ~m) | (NEG2 & m);
            M = (M & ~m) | (NEG2 & m);
            E = (E & ~m) | (NEG2 & m);
            const unsigned pk = prmt(H, F, 0x7632u);  // (H.hi, F.hi)
            unsigned sh = grp.shfl(pk, src);
            if (use_ring && k == 0) sh = u == 0 ? rv0 : (u == 1 ? rv1 : (u == 2 ? rv2 : rv3));
            hd = hv;
            hv = prmt(sh, H, 0x5410u);  // low: row above (lane k-1 high), high: own low
            fv = prmt(sh, F, 0x5432u);
            ml = M;
            el = E;
            if (u == 0) { hk0 = H; pk0 = pk; }
            if (u == 1) { hk1 = H; pk1 = pk; }
            if (u == 2) { hk2 = H; pk2 = pk; }
            if (u == 3) { hk3 = H; pk3 = pk; }
        }
        // ---- once per chunk ----
        tpv = prmt(tw, tpv, 0x4344u);  // this chunk's last code, for the next chunk's high half
        w0 = w1;
        w1 = w2;
        ++wi;
        if (active) w2 = __ldg(tw32 + imin(imax(wi + 2, 0), nwords - 1));
        if (TB && (g0 >> 2) <= last_chunk) bits[(g0 >> 2) * L + k] = acc;
        if (use_ring && k == L - 1)
            *reinterpret_cast<uint4*>(ring + (g0 & rmask)) = make_uint4(pk0, pk1, pk2, pk3);
        {
            const unsigned cm = umax2(umax2(hk0, hk1), umax2(hk2, hk3));
            const unsigned nb = umax2(lb, cm);
            if (nb != lb) {  // the maximum grew in this chunk: first step reaching it
                const unsigned inc = nb ^ lb;
                if (inc & 0xFFFFu) {
                    const int t = lo16(nb);
                    const int u = lo16(hk0) == t ? 0 : (lo16(hk1) == t ? 1 : (lo16(hk2) == t ? 2 : 3));
                    pos0 = XD ? d + u : g0 + u;
                }
                if (inc >> 16) {
                    const int t = hi16(nb);
                    const int u = hi16(hk0) == t ? 0 : (hi16(hk1) == t ? 1 : (hi16(hk2) == t ? 2 : 3));
                    pos1 = XD ? d + u - 2 : g0 + u;
                }
                lb = nb;
            }
            if (XD) {
                if (d == dW0 && row <= qlen && row >= 1) rowmax[row - 1] = make_int2(lo16(lb) - (int)Z, pos0);
                if (d == dW1 && row + 1 <= qlen && row >= 1) rowmax[row] = make_int2(hi16(lb) - (int)Z, pos1);
            }
        }
        __syncwarp();
        d += 4;
        if (d == P) d = 0;
    }
    __syncwarp();

    int bh, bi, bd;
    if (XD) {
        xdrop_best<L>(grp, rowmax, qlen, a.x_drop, active, bh, bi, bd);
    } else {
        // first cell of each virtual lane's maximum, then the group's best
        const int v0 = lo16(lb) - (int)Z, v1 = hi16(lb) - (int)Z;
        int r0 = 0, s0 = 0, r1 = 0, s1 = 0;
        if (v0 > 0) {
            const int tt = pos0 - 2 * (2 * k);
            const int s = tt / P;
            r0 = s * V + 2 * k + 1;
            s0 = tt - s * P;
        }
        if (v1 > 0) {
            const int tt = pos1 - 2 * (2 * k + 1);
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
    extern __shared__ uint4 sw16_ring4[];
    uint32_t* sw16_ring = reinterpret_cast<uint32_t*>(sw16_ring4);
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
