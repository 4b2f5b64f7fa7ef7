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
// The step uses the DPX __viaddmax_u16x2 / __viaddmin_u16x2 / __vimax3_u16x2,
// byte permutes and logic on the ALU pipe, and puts its adds on the FMA pipe
// (16x2 adds of constants, multiply-adds): the ALU pipe issues at half rate
// and bounds the step.  Packed adds and subtracts never carry or borrow
// across halves.  Comparisons are differences of values known to be ordered
// (H >= M >= diag, H >= F, F >= fa, E >= ea, E >= eb), read as bit 15 of
// (difference + 0x7fff) per half.
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
//
// Long pairs with wide bands run in the cooperative form below: the warps of
// one CTA share a pair strip by strip.

#include <algorithm>

#include "sw_common.cuh"

namespace gmf {

// Traceback word of one lane and chunk, byte-planar: bit u (step u of the
// chunk) of byte h holds "H != diag" of half h, bit 4+u of byte h "F
// extends"; bit u of byte 2+h holds "H != F", bit 4+u of byte 2+h "E
// extends".  nib() turns a cell's bits into the walk's 4-bit code (H source
// 1 diagonal / 2 F / 3 E, F extends, E extends); this form stores no stop
// bit, the walk stops on the H value it tracks.
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
        const uint32_t w = bits[(g >> 2) * L + k] >> (8 * h + (int)(g & 3));
        const uint32_t n1 = w & 1u, fc = (w >> 4) & 1u, n2 = (w >> 16) & 1u, ec = (w >> 20) & 1u;
        return (n1 ? (n2 ? 3u : 2u) : 1u) | (fc << 2) | (ec << 3);
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

// ---------------------------------------------------------------------------
// Pieces shared by the one-warp and the cooperative (several warps per pair)
// kernels.
// ---------------------------------------------------------------------------

// Per-lane DP state carried from step to step.
struct Cells16 {
    unsigned hv, fv, hd, ml, el;  // H / F of the row above (this and the previous slot), M / E on the left
    unsigned ma, mb;              // 32768 + slot - band_lo, 32768 + band_hi - slot per half (bit 15 set: in)
    unsigned qp;                  // query codes of the two rows (0x100 = never matches)
    unsigned acc;                 // traceback nibbles of the chunk
};

__device__ __forceinline__ void cells_init(Cells16& c, const K16& K) {
    c.hv = K.Z2;
    c.fv = K.NEG2;
    c.hd = K.Z2;
    c.ml = K.NEG2;
    c.el = K.NEG2;
    c.ma = pack16(2768, 2768);  // out of band until the lane's first row starts
    c.mb = pack16(20000, 20000);
    c.qp = 0x01000100u;
    c.acc = 0u;
}

// Target codes as 32-bit words of the whole target buffer, indexed from its
// first aligned word; a chunk's 4 codes are a funnel shift of two words, and
// the window slides one word per chunk with a load two chunks ahead.  Words
// outside the buffer are clamped: they only ever feed out-of-band cells.
struct TWin {
    const uint32_t* w32;
    int nwords;
    long long pair_t;  // byte offset of the pair's codes from w32
    unsigned w0, w1, w2;
    int wi, tsh;
    __device__ void setup(const SwArgs& a, const PairGeo& G, bool active) {
        const long long tbase = (long long)(uintptr_t)a.t & ~3ll;
        const long long t_total = active ? a.t_off[a.n_pairs] : 1;
        const long long nw64 = (((long long)(uintptr_t)a.t + t_total - 1 - tbase) >> 2) + 1;
        nwords = nw64 > 0x7fffffffll ? 0x7fffffff : (int)nw64;
        w32 = reinterpret_cast<const uint32_t*>((uintptr_t)tbase);
        pair_t = (long long)(uintptr_t)G.t - tbase;
        w0 = w1 = w2 = 0u;
        wi = 0;
        tsh = 0;
    }
    // a negative index wraps to a large unsigned one and reads the last word
    __device__ unsigned ld(int i) const { return __ldg(w32 + min((unsigned)i, (unsigned)(nwords - 1))); }
    __device__ void start(int code_index, bool active) {  // window at code index `code_index` of the pair
        const long long off = pair_t + (long long)code_index;
        tsh = (int)(off & 3) * 8;
        wi = (int)(off >> 2);
        if (active) {
            w0 = ld(wi);
            w1 = ld(wi + 1);
            w2 = ld(wi + 2);
        }
    }
    __device__ unsigned window() const { return __funnelshift_r(w0, w1, tsh); }
    __device__ void advance(bool active) {
        w0 = w1;
        w1 = w2;
        ++wi;
        if (active) w2 = ld(wi + 2);
    }
};

// New rows for both halves of a lane: query codes and band intervals (the
// high half's interval is expressed in the low half's slot, two steps later).
__device__ __forceinline__ void row_start16(Cells16& c, int row, int j0, int qlen, int tlen, int W,
                                            const int8_t* q) {
    const int cq0 = row <= qlen ? (int)q[row - 1] : -1;
    const int cq1 = row + 1 <= qlen ? (int)q[row] : -1;
    c.qp = pack16((cq0 >= 0 && cq0 != 5) ? cq0 : 0x100, (cq1 >= 0 && cq1 != 5) ? cq1 : 0x100);
    // interval bounds clamped into int16: an empty interval stays empty
    const int lo0 = imin(imax(0, 1 - j0), 32000);
    const int hi0 = row <= qlen ? imax(imin(W - 1, tlen - j0), -1) : -1;
    const int lo1 = imin(imax(2, 2 - j0), 32000);
    const int hi1 = row + 1 <= qlen ? imax(imin(W + 1, tlen - j0 + 1), -1) : -1;
    c.ma = pack16(32768 - 1 - lo0, 32768 - 1 - lo1);
    c.mb = pack16(32768 + hi0 + 1, 32768 + hi1 + 1);
}

// Four pipeline steps of one lane.  The first lane of the group takes its
// row-above inputs from rv[] when `from_rv` (delay line or previous warp),
// every other lane from lane k-1 by one shuffle of the packed (H.hi, F.hi).
// MASKED: reset out-of-band cells (H = 0, M = E = F = -inf) at every step;
// the caller drops it for chunks in which every lane of the warp stays
// inside its band on all four steps (there the reset changes nothing) and
// advances the band counters itself.
template <int L, bool TB, int EM, bool MASKED>
__device__ __forceinline__ void chunk16(Cells16& c, const K16& K, const Grp<L>& grp, int src, unsigned tw,
                                        unsigned tpv, bool from_rv, const unsigned (&rv)[4],
                                        unsigned (&hk)[4], unsigned (&pko)[4]) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        // Every operand half is a biased value >= pmax and every difference
        // is taken between values known to be ordered, so the adds and
        // subtracts below never carry or borrow across halves.  They are
        // written to issue on the FMA pipe: 16x2 adds of a constant, and
        // multiply-adds by the run-time constants ONE / NEG1.  The DPX
        // maxima, permutes and logic of the step all take the ALU pipe,
        // which runs at half rate and bounds the step.
        const unsigned tp = prmt(tw, tpv, tsel(u));
        const unsigned mis = flag2(c.qp ^ tp);  // 0: match, 1: mismatch
        const unsigned diag = __vadd2(c.hd, K.MATCH2) - mis * K.MX;  // one multiply-add, no borrow
        const unsigned fa = __vsub2(c.hv, K.GO2);
        unsigned F = __viaddmax_u16x2(c.fv, K.NGE2, fa);  // max(F above - ext, H above - open)
        unsigned M = __vimax3_u16x2(diag, F, K.Z2);
        const unsigned ea = __vsub2(c.ml, K.GO2);
        unsigned E = __viaddmax_u16x2(c.el, K.NGE2, ea);
        unsigned H = umax2(M, E);
        if (TB) {
            // Each flag is bit 15 of a half of (ordered difference + 0x7fff):
            // set when the difference is at least 1.  The classifier keeps
            // every difference within 15 bits, so the sums neither carry nor
            // borrow across halves (the 32-bit x + 0x7fff7fff may carry, and
            // the subtraction that follows takes the carry back).
            const unsigned hb = H * K.ONE + 0x7FFF7FFFu;
            const unsigned n1 = diag * K.NEG1 + hb;                        // H != diag
            const unsigned n2 = F * K.NEG1 + hb;                           // H != F
            const unsigned fc = fa * K.NEG1 + (F * K.ONE + 0x7FFF7FFFu);   // F extends (F above - ext > H above - open)
            unsigned ec = 0u;                                              // E extends
            if (EM == 0) ec = ea * K.NEG1 + (E * K.ONE + 0x7FFF7FFFu);     //   open > ext: E_left - ext > M_left - open
            if (EM == 2) ec = c.el - E + K.EB2;          //   open < ext: E == E_left - ext (ties extend)
            // sign-replicated high bytes: [n1.lo n1.hi n2.lo n2.hi], [fc.lo fc.hi ec.lo ec.hi]
            const unsigned w1 = prmt(n1, n2, 0xFDB9u);
            const unsigned w2 = prmt(fc, ec, 0xFDB9u);
            const unsigned b = (w1 & (0x01010101u << u)) | (w2 & (0x10101010u << u));
            c.acc = u == 0 ? b : (c.acc | b);
        }
        if (MASKED) {
            // in-band mask: slot - lo >= 0 and hi - slot >= 0 per half, kept as
            // counters biased by 32768 (they never leave [0, 65535], so plain
            // adds suffice); bit 15 of both set = in band
            c.ma = __vadd2(c.ma, ONE2);
            c.mb = __vsub2(c.mb, ONE2);
            const unsigned m = prmt(c.ma & c.mb, 0u, 0xBB99u);  // 0xFFFF per in-band half
            H = (H & m) | (K.Z2 & ~m);
            F = (F & m) | (K.NEG2 & ~m);
            M = (M & m) | (K.NEG2 & ~m);
            E = (E & m) | (K.NEG2 & ~m);
        }
        const unsigned pk = prmt(H, F, 0x7632u);  // (H.hi, F.hi)
        unsigned sh = grp.shfl(pk, src);
        if (from_rv) sh = rv[u];
        c.hd = c.hv;
        c.hv = prmt(sh, H, 0x5410u);  // low: row above (lane k-1 high), high: own low
        c.fv = prmt(sh, F, 0x5432u);
        c.ml = M;
        c.el = E;
        hk[u] = H;
        pko[u] = pk;
    }
}

// True when every cell of the lane's next chunk (4 steps, both halves) is in
// band: the first step's lower-bound counters and the last step's upper-
// bound counters both have bit 15 set.
__device__ __forceinline__ bool chunk_in_band(const Cells16& c) {
    return ((c.ma + ONE2) & (c.mb - 4u * ONE2) & 0x80008000u) == 0x80008000u;
}

// A chunk with or without the band reset: the unmasked form when the whole
// warp stays in band (warp-uniform decision).
template <int L, bool TB, int EM>
__device__ __forceinline__ void chunk16_any(Cells16& c, const K16& K, const Grp<L>& grp, int src, unsigned tw,
                                            unsigned tpv, bool from_rv, const unsigned (&rv)[4],
                                            unsigned (&hk)[4], unsigned (&pko)[4]) {
    if (__all_sync(FULL_MASK, chunk_in_band(c))) {
        chunk16<L, TB, EM, false>(c, K, grp, src, tw, tpv, from_rv, rv, hk, pko);
        c.ma = __vadd2(c.ma, 4u * ONE2);
        c.mb = __vsub2(c.mb, 4u * ONE2);
    } else {
        chunk16<L, TB, EM, true>(c, K, grp, src, tw, tpv, from_rv, rv, hk, pko);
    }
}

// Best-cell bookkeeping of a chunk: `lb` is the running maximum per half (the
// row maximum under x-drop); when it grows, the first of the chunk's 4 steps
// that reaches it gives the position (global step, or slot under x-drop).
template <bool XD>
__device__ __forceinline__ void best16(unsigned& lb, int& pos0, int& pos1, const unsigned (&hk)[4], int gstep,
                                       int d) {
    const unsigned nb = __vimax3_u16x2(lb, __vimax3_u16x2(hk[0], hk[1], hk[2]), hk[3]);
    if (nb != lb) {
        // per half, the steps before the first that reaches nb, counted for
        // both halves at once: nb >= hk[u] in each half, so the plain
        // subtractions do not borrow across halves, and flag2 is 1 while
        // hk[u] < nb
        const unsigned e0 = flag2(nb - hk[0]);
        const unsigned e01 = e0 & flag2(nb - hk[1]);
        const unsigned e012 = e01 & flag2(nb - hk[2]);
        const unsigned u = e0 + e01 + e012;  // 0..3 in each half
        const unsigned inc = nb ^ lb;
        if (inc & 0xFFFFu) pos0 = (XD ? d : gstep) + (int)(u & 0xFFFFu);
        if (inc >> 16) pos1 = (XD ? d - 2 : gstep) + (int)(u >> 16);
        lb = nb;
    }
}

// Best-cell bookkeeping without x-drop, branch-free: when a half's running
// maximum grows, that half's 4 H values of the chunk and the chunk's first
// global step are kept (a per-half select); the first step that reaches the
// final maximum is found once, after the DP, from the kept values.  The
// maximum only grows on a strictly larger value, so the kept chunk is the
// one in which the final maximum first appears.
struct BestTrack16 {
    unsigned sv[4];
    int g_lo, g_hi;
    __device__ __forceinline__ void init(unsigned z2) {
        sv[0] = sv[1] = sv[2] = sv[3] = z2;
        g_lo = g_hi = 0;
    }
    // Run by the whole warp (every caller's chunk loop is warp-uniform): the
    // selects are skipped in the chunks where no lane's maximum grows.
    __device__ __forceinline__ void update(unsigned& lb, const unsigned (&hk)[4], int g0) {
        const unsigned nb = __vimax3_u16x2(lb, __vimax3_u16x2(hk[0], hk[1], hk[2]), hk[3]);
        if (__any_sync(FULL_MASK, nb != lb)) {
            // nb >= lb in each half and the difference stays within 15 bits:
            // bit 15 of difference + 0x7fff is "grew", spread over the half
            const unsigned up = prmt(nb - lb + 0x7FFF7FFFu, 0u, 0xBB99u);
#pragma unroll
            for (int u = 0; u < 4; ++u) sv[u] = (hk[u] & up) | (sv[u] & ~up);
            g_lo = (up & 1u) ? g0 : g_lo;
            g_hi = (up >> 31) ? g0 : g_hi;
            lb = nb;
        }
    }
    // Global steps of the first cell of each half that holds its maximum.
    __device__ __forceinline__ void positions(unsigned lb, int& pos0, int& pos1) const {
        int u0 = 3, u1 = 3;
#pragma unroll
        for (int u = 2; u >= 0; --u) {
            if (lo16(sv[u]) == lo16(lb)) u0 = u;
            if (hi16(sv[u]) == hi16(lb)) u1 = u;
        }
        pos0 = g_lo + u0;
        pos1 = g_hi + u1;
    }
};

// Best cell of a lane (non-x-drop): the first maximum of each half, from its
// global step, as (score, row, slot).
template <int L>
__device__ __forceinline__ void lane_best16(unsigned lb, int pos0, int pos1, unsigned Z, int g, int k, int P,
                                            int& bh, int& bi, int& bd) {
    constexpr int V = 2 * L;
    const int v0 = (lo16(lb) - (int)Z) * g, v1 = (hi16(lb) - (int)Z) * g;  // true scores
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
}

// (score, row, slot) ordering of the best cell: higher score, then earlier
// row, then earlier slot.
__device__ __forceinline__ bool better_cell(int oh, int oi, int od, int bh, int bi, int bd) {
    return oh > bh || (oh == bh && (oi < bi || (oi == bi && od < bd)));
}

// ---------------------------------------------------------------------------
// One group of L lanes per pair.
// ---------------------------------------------------------------------------
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

    const K16& K = a.k16;
    for (int x = k; x < a.ring; x += L) ring[x] = K.init_pk();
    __syncwarp();
    TWin tw;
    tw.setup(a, G, active);

    const int8_t* __restrict__ q = G.q;
    const int c0 = G.off - G.hb;  // j = row + c0 + d
    int d = -4 * k;               // slot of the low half at the chunk start (x-drop bookkeeping)
    int until = k;                // chunks until the lane's next row start (every P / 4 chunks)
    int tbi = k;                  // word of the chunk's traceback bits: (g0 / 4) * L + k
    const int tb_end = last_chunk * L + k;
    int row = 2 * k + 1 - V;      // row of the low half (advanced by V at each row start)
    Cells16 c;
    cells_init(c, K);
    unsigned tpv = 0u;
    unsigned lb = K.Z2;  // best H so far per half (non-x-drop) / row max (x-drop)
    int pos0 = 0, pos1 = 0;
    BestTrack16 bt;
    bt.init(K.Z2);
    unsigned rv[4] = {0u, 0u, 0u, 0u};  // delay-line entries of the chunk
    const int src = (k + L - 1) & (L - 1);
    const bool from_rv = use_ring && k == 0;
    const int dW0 = (W - 1) & ~3, dW1 = (W + 1) & ~3;  // chunks that end a row (x-drop)

    // The lane's next row (query codes, band counters, target window) is
    // prepared by the whole group in the chunk where the group's lane 0
    // starts its row (until == k there), and taken up k chunks later: the
    // loads and bounds run once per period for all lanes instead of one lane
    // at a time.
    unsigned nqp = 0u, nma = 0u, nmb = 0u, nw0 = 0u, nw1 = 0u, nw2 = 0u;
    int nwi = 0, ntsh = 0;

    for (int g0 = 0; g0 <= loop_last; g0 += 4) {
        if (until == k) {
            Cells16 nx;
            row_start16(nx, row + V, row + V + c0, qlen, tlen, W, q);
            TWin tn = tw;
            tn.start(row + V + c0 - 1, active);
            nqp = nx.qp;
            nma = nx.ma;
            nmb = nx.mb;
            nw0 = tn.w0;
            nw1 = tn.w1;
            nw2 = tn.w2;
            nwi = tn.wi;
            ntsh = tn.tsh;
        }
        if (until == 0) {  // both halves start new rows (the high half two steps later)
            until = P >> 2;
            row += V;
            c.qp = nqp;
            c.ma = nma;
            c.mb = nmb;
            tw.w0 = nw0;
            tw.w1 = nw1;
            tw.w2 = nw2;
            tw.wi = nwi;
            tw.tsh = ntsh;
            tpv = 0u;
            if (XD) {
                lb = K.Z2;
                pos0 = 0;
                pos1 = 0;
            }
        }
        if (from_rv) {
            const uint4 r = *reinterpret_cast<const uint4*>(ring + ((g0 - D) & rmask));
            rv[0] = r.x;
            rv[1] = r.y;
            rv[2] = r.z;
            rv[3] = r.w;
        }
        const unsigned twin = tw.window();
        unsigned hk[4], pk[4];
        chunk16_any<L, TB, EM>(c, K, grp, src, twin, tpv, from_rv, rv, hk, pk);
        // ---- once per chunk ----
        tpv = prmt(twin, tpv, 0x4344u);  // this chunk's last code, for the next chunk's high half
        tw.advance(active);
        if (TB && tbi <= tb_end) bits[tbi] = c.acc;
        tbi += L;
        if (use_ring && k == L - 1)
            *reinterpret_cast<uint4*>(ring + (g0 & rmask)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        if (XD)
            best16<XD>(lb, pos0, pos1, hk, g0, d);
        else
            bt.update(lb, hk, g0);
        if (XD) {
            if (d == dW0 && row <= qlen && row >= 1) rowmax[row - 1] = make_int2((lo16(lb) - (int)K.Z) * K.G, pos0);
            if (d == dW1 && row + 1 <= qlen && row >= 1) rowmax[row] = make_int2((hi16(lb) - (int)K.Z) * K.G, pos1);
        }
        __syncwarp();
        --until;
        if (XD) {
            d += 4;
            if (d == P) d = 0;
        }
    }
    __syncwarp();

    int bh, bi, bd;
    if (XD) {
        if (active && k == 0) record_rowmax(a, p, rowmax);
        xdrop_best<L>(grp, rowmax, qlen, a.x_drop, active, bh, bi, bd);
    } else {
        bt.positions(lb, pos0, pos1);
        lane_best16<L>(lb, pos0, pos1, K.Z, K.G, k, P, bh, bi, bd);
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) {
            const int oh = grp.xr(bh, o);
            const int oi = grp.xr(bi, o);
            const int od = grp.xr(bd, o);
            if (better_cell(oh, oi, od, bh, bi, bd)) {
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
    if (a.defer_walk) {  // the traceback walk runs later, in sw_walk_kernel
        if (active && k == 0) record_walk(a, p, bits, L);
        return;
    }

    RunWriter rw;
    uint32_t* runs = ws_alloc<L>(a, grp, (unsigned long long)qe + te + 1, active && bh > 0);
    const bool runs_ok = !(active && bh > 0) || runs != nullptr;
    if (!runs_ok && k == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
    rw.init(runs);
    Layout16<L> lay{bits, P, W, qlen};
    int qs = 0, ts = 0;
    walk<L>(grp, lay, G, a, qe, te, bh, active && runs_ok && bh > 0, rw, qs, ts);
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

// ---------------------------------------------------------------------------
// Cooperative form: the NW warps of one CTA align one long pair.
//
// Warp w runs strips w, w+NW, w+2NW, ... of the pair with the one-warp
// pipeline; the first lane of each strip reads the row above (the last lane's
// (H.hi, F.hi) of the strip before) from the previous warp's shared-memory
// ring instead of its own delay line.  Entry e of warp w's ring is its last
// lane's output at warp-local step e; warp w reads entry t + 4L of warp w-1
// at its local step t (t + 4L - P from warp NW-1 for warp 0), so each warp
// runs at least 4L + 4 steps behind its predecessor, and the cycle of NW
// warps keeps moving only when P >= NW * (4L + 4) -- the classifier sends a
// pair here only then.  Under that bound no writer is ever more than P
// entries ahead of its reader, so the 2- and 4-warp classes use rings of
// R >= P + 8 entries and no back-pressure.  The 8-warp class (periods up to
// COOP_PMAX) adds back-pressure instead and keeps 1,024-entry rings: its
// writers also wait for their readers (see sw16_coop_pair).  Each writer
// publishes its progress after every chunk (ring store, then a release store
// of the flag); each reader polls the flag with acquire loads and an
// iteration limit, after which it records GMF_SWF_TIMEOUT and goes on.
// Traceback words land at the same (global step, lane) positions as in the
// one-warp layout, so the walk (warp 0, after a block barrier) is unchanged.
// ---------------------------------------------------------------------------

// Progress flags between the warps of a CTA: the writer publishes with a
// release store after its ring store, the reader polls with acquire loads;
// neither waits for the thread's outstanding global loads or stores (a block
// fence would).
__device__ __forceinline__ int ld_acquire_cta(const int* p) {
    int v;
    asm volatile("ld.acquire.cta.shared.b32 %0, [%1];" : "=r"(v)
                 : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_cta(int* p, int v) {
    asm volatile("st.release.cta.shared.b32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v)
                 : "memory");
}

template <int NW, bool TB, bool XD, int EM>
__device__ void sw16_coop_pair(const SwArgs& a, int p, uint32_t* rings, int* prog, int* cons, int (*sbest)[3],
                               uint32_t** sws) {
    constexpr int L = 32, V = 64;
    // The 8-warp class (wide bands) bounds each warp's lead over the warp that
    // reads it as well: lane 31 waits until its reader has taken the entries
    // it is about to overwrite, so a ring of a.ring entries (1024) serves
    // periods up to COOP_PMAX instead of needing P + 8.  A warp's lag behind
    // its predecessor then stays within [132, a.ring + 128] steps; the lags
    // of the NW links sum to P, so with NW * 132 <= P <= NW * (a.ring + 128)
    // the warps cannot all be waiting at once.
    constexpr bool BP = NW == 8;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    Grp<32> grp(lane);
    PairGeo G = load_geo(a, p);
    const bool bad = G.hb < 0 || G.hb > a.max_hb;
    if (bad || G.qlen <= 0 || G.tlen <= 0) {  // uniform over the CTA
        if (threadIdx.x == 0) write_empty<TB>(a, p, bad);
        return;
    }
    const int qlen = G.qlen, tlen = G.tlen, W = G.W;
    const int P = sw16_period(W, L);
    G.P = P;
    const int nstrips = (qlen + V - 1) / V;
    const int my_last = (nstrips - 1) * P + 2 * ((qlen - 1) % V) + W - 1;  // global step of the last cell
    const int last_chunk = my_last >> 2;

    const unsigned long long tbw = TB ? sw16_tb_words_l(qlen, W, L) : 0ull;
    if (w == 0) {
        uint32_t* ws0 = ws_alloc<32>(a, grp, tbw + (XD ? 2ull * qlen : 0ull), TB || XD);
        if (lane == 0) *sws = ws0;
    }
    if (threadIdx.x < NW) {
        prog[threadIdx.x] = 0;
        cons[threadIdx.x] = (int)threadIdx.x < nstrips ? 0 : 0x7fffffff;  // a warp without strips reads nothing
    }
    __syncthreads();
    uint32_t* ws = *sws;
    if ((TB || XD) && !ws) {
        if (threadIdx.x == 0) write_empty<TB>(a, p, true);
        return;
    }
    uint32_t* bits = ws;
    int2* rowmax = XD ? reinterpret_cast<int2*>(ws + tbw) : nullptr;

    const K16& K = a.k16;
    TWin tw;
    tw.setup(a, G, true);
    const int8_t* __restrict__ q = G.q;
    const int c0 = G.off - G.hb;
    const int kk_last = w < nstrips ? (nstrips - 1 - w) / NW : -1;  // this warp's last strip (local index)
    const int loop_end = (kk_last + 1) * P + 4 * L + 4;             // drains what the next warp may read
    uint32_t* ring_out = rings + (size_t)w * a.ring;
    const int wprev = (w + NW - 1) % NW;
    const uint32_t* ring_in = rings + (size_t)wprev * a.ring;
    const int rmask = a.ring - 1;
    const unsigned INIT = K.init_pk();

    int d = -4 * lane;  // slot of the low half at the chunk start (x-drop bookkeeping)
    int until = lane;   // chunks until the lane's next row start (every P / 4 chunks)
    int tbi = 0x3fffffff;  // word of the chunk's traceback bits ((t + gofs) / 4 * L + lane), none before a row
    const int tb_end = last_chunk * L + lane;
    int kk = -1;        // local index of the lane's current strip
    int row = 0, gofs = 0;
    Cells16 c;
    cells_init(c, K);
    unsigned tpv = 0u, lb = K.Z2;
    int pos0 = 0, pos1 = 0;
    BestTrack16 bt;
    bt.init(K.Z2);
    unsigned rv[4] = {INIT, INIT, INIT, INIT};
    const int src = (lane + 31) & 31;
    const int dW0 = (W - 1) & ~3, dW1 = (W + 1) & ~3;

    // the lane's next row, prepared by the whole warp when lane 0 starts its
    // strip (until == lane there) and taken up lane chunks later
    unsigned nqp = 0u, nma = 0u, nmb = 0u, nw0 = 0u, nw1 = 0u, nw2 = 0u;
    int nwi = 0, ntsh = 0;

    if (kk_last >= 0) {
        for (int t = 0; t < loop_end; t += 4) {
            if (until == lane) {
                const int nrow = (w + NW * (kk + 1)) * V + 2 * lane + 1;
                Cells16 nx;
                row_start16(nx, nrow, nrow + c0, qlen, tlen, W, q);
                TWin tn = tw;
                tn.start(nrow + c0 - 1, true);
                nqp = nx.qp;
                nma = nx.ma;
                nmb = nx.mb;
                nw0 = tn.w0;
                nw1 = tn.w1;
                nw2 = tn.w2;
                nwi = tn.wi;
                ntsh = tn.tsh;
            }
            if (until == 0) {
                until = P >> 2;
                ++kk;
                const int s = w + NW * kk;
                row = s * V + 2 * lane + 1;
                gofs = (s - kk) * P;  // local step -> step of the one-warp schedule
                tbi = ((t + gofs) >> 2) * L + lane;
                c.qp = nqp;
                c.ma = nma;
                c.mb = nmb;
                tw.w0 = nw0;
                tw.w1 = nw1;
                tw.w2 = nw2;
                tw.wi = nwi;
                tw.tsh = ntsh;
                tpv = 0u;
                if (XD) {
                    lb = K.Z2;
                    pos0 = 0;
                    pos1 = 0;
                }
            }
            if (lane == 0) {
                const int s0 = w + NW * kk;  // lane 0 starts its strips at t = kk * P
                if (s0 >= 1 && s0 < nstrips) {
                    const int e = t + 4 * L - (w == 0 ? P : 0);
                    int spins = 0;
                    while (ld_acquire_cta(prog + wprev) < e + 4) {
                        // bounded: after the limit, or once any wait in the grid gave up
                        // (every later wait then ends within ~1k spins), record and go on
                        if (++spins > a.coop_spin_limit ||
                            ((spins & 1023) == 0 && (*(volatile int*)a.err & (int)GMF_SWF_TIMEOUT))) {
                            atomicOr(a.err, (int)GMF_SWF_TIMEOUT);
                            break;
                        }
                        __nanosleep(20);
                    }
                    const uint4 r = *reinterpret_cast<const uint4*>(ring_in + (e & rmask));
                    rv[0] = r.x;
                    rv[1] = r.y;
                    rv[2] = r.z;
                    rv[3] = r.w;
                } else {
                    rv[0] = rv[1] = rv[2] = rv[3] = INIT;  // row 0, or a strip past the query
                }
                // the previous warp's entries before t + 4 * L (+ 4), in its step
                // numbering, are no longer needed (also when this strip reads none)
                if (BP) st_release_cta(cons + w, t + 4 * L + 4 - (w == 0 ? P : 0));
            }
            const unsigned twin = tw.window();
            unsigned hk[4], pk[4];
            chunk16_any<32, TB, EM>(c, K, grp, src, twin, tpv, lane == 0, rv, hk, pk);
            tpv = prmt(twin, tpv, 0x4344u);
            tw.advance(true);
            if (lane == 31) {  // publish before the global store, so the release does not wait on it
                if (BP) {
                    // the slots of steps t .. t+3 held steps t - ring .. t - ring + 3
                    const int need = t + 4 - a.ring;
                    int spins = 0;
                    while (ld_acquire_cta(cons + (w + 1) % NW) < need) {
                        if (++spins > a.coop_spin_limit ||
                            ((spins & 1023) == 0 && (*(volatile int*)a.err & (int)GMF_SWF_TIMEOUT))) {
                            atomicOr(a.err, (int)GMF_SWF_TIMEOUT);
                            break;
                        }
                        __nanosleep(20);
                    }
                }
                *reinterpret_cast<uint4*>(ring_out + (t & rmask)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                if (!a.coop_stall) st_release_cta(prog + w, t + 4);
            }
            const int g0 = t + gofs;
            if (TB && tbi <= tb_end) bits[tbi] = c.acc;
            tbi += L;
            if (XD)
                best16<XD>(lb, pos0, pos1, hk, g0, d);
            else
                bt.update(lb, hk, g0);
            if (XD && kk >= 0) {
                if (d == dW0 && row <= qlen) rowmax[row - 1] = make_int2((lo16(lb) - (int)K.Z) * K.G, pos0);
                if (d == dW1 && row + 1 <= qlen) rowmax[row] = make_int2((hi16(lb) - (int)K.Z) * K.G, pos1);
            }
            __syncwarp();
            --until;
            if (XD) {
                d += 4;
                if (d == P) d = 0;
            }
        }
    }
    if (BP && lane == 0 && kk_last >= 0) st_release_cta(cons + w, 0x7fffffff);  // reads nothing more
    __syncthreads();  // every traceback word and row maximum is written

    int bh = 0, bi = 0, bd = 0;
    if (!XD) {
        bt.positions(lb, pos0, pos1);
        lane_best16<L>(lb, pos0, pos1, K.Z, K.G, lane, P, bh, bi, bd);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int oh = grp.xr(bh, o);
            const int oi = grp.xr(bi, o);
            const int od = grp.xr(bd, o);
            if (better_cell(oh, oi, od, bh, bi, bd)) {
                bh = oh;
                bi = oi;
                bd = od;
            }
        }
        if (lane == 0) {
            sbest[w][0] = bh;
            sbest[w][1] = bi;
            sbest[w][2] = bd;
        }
        __syncthreads();
    }
    if (w != 0) return;
    if (XD) {
        if (lane == 0) record_rowmax(a, p, rowmax);
        xdrop_best<L>(grp, rowmax, qlen, a.x_drop, true, bh, bi, bd);
    } else {
        bh = sbest[0][0];
        bi = sbest[0][1];
        bd = sbest[0][2];
        for (int x = 1; x < NW; ++x)
            if (better_cell(sbest[x][0], sbest[x][1], sbest[x][2], bh, bi, bd)) {
                bh = sbest[x][0];
                bi = sbest[x][1];
                bd = sbest[x][2];
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
        if (lane == 0) record_walk(a, p, bits, L);
        return;
    }
    RunWriter rw;
    uint32_t* runs = ws_alloc<32>(a, grp, (unsigned long long)qe + te + 1, bh > 0);
    const bool runs_ok = bh == 0 || runs != nullptr;
    if (!runs_ok && lane == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
    rw.init(runs);
    Layout16<L> lay{bits, P, W, qlen};
    int qs = 0, ts = 0;
    walk<L>(grp, lay, G, a, qe, te, bh, runs_ok && bh > 0, rw, qs, ts);
    finish_cigar<L>(a, grp, p, true, rw, runs_ok, qs, ts);
}

template <int NW, bool TB, bool XD, int EM>
__global__ void __launch_bounds__(32 * NW) sw16_coop_kernel(SwArgs a) {
    extern __shared__ uint4 coop_ring4[];
    uint32_t* rings = reinterpret_cast<uint32_t*>(coop_ring4);
    __shared__ int prog[NW];
    __shared__ int cons[NW];
    __shared__ int sbest[NW][3];
    __shared__ uint32_t* sws;
    __shared__ int spair;
    constexpr int CLS = NW == 2 ? CLS_I16_C2 : (NW == 4 ? CLS_I16_C4 : CLS_I16_C8);
    const int count = a.queue[N_CLASSES + CLS];
    const int32_t* list = a.lists + (size_t)CLS * a.n_pairs;
    for (;;) {
        if (threadIdx.x == 0) spair = atomicAdd(&a.queue[CLS], 1);
        __syncthreads();
        const int idx = spair;
        if (idx >= count) break;
        sw16_coop_pair<NW, TB, XD, EM>(a, list[idx], rings, prog, cons, sbest, &sws);
        __syncthreads();
    }
}

int sw16_coop_warps(int cls) { return cls == CLS_I16_C2 ? 2 : (cls == CLS_I16_C4 ? 4 : 8); }

template <int NW, bool TB, bool XD, int EM>
static int launch_coop(const SwArgs& a, cudaStream_t stream) {
    const size_t smem = (size_t)NW * a.ring * sizeof(uint32_t);
    void (*k)(SwArgs) = sw16_coop_kernel<NW, TB, XD, EM>;
    if (smem > 48 * 1024)
        GMF_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    GMF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    GMF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 32 * NW, smem));
    if (per_sm <= 0) return GMF_ERR_LIMIT;
    k<<<sms * per_sm, 32 * NW, smem, stream>>>(a);
    return cuda_status(cudaGetLastError());
}

template <int NW, bool TB, bool XD>
static int launch_coop_e(const SwArgs& a, int e_mode, cudaStream_t s) {
    if (e_mode == 0) return launch_coop<NW, TB, XD, 0>(a, s);
    if (e_mode == 1) return launch_coop<NW, TB, XD, 1>(a, s);
    return launch_coop<NW, TB, XD, 2>(a, s);
}

template <int NW>
static int launch_coop_x(const SwArgs& a, bool tb, bool xd, int e_mode, cudaStream_t s) {
    if (tb) return xd ? launch_coop_e<NW, true, true>(a, e_mode, s) : launch_coop_e<NW, true, false>(a, e_mode, s);
    return xd ? launch_coop_e<NW, false, true>(a, e_mode, s) : launch_coop_e<NW, false, false>(a, e_mode, s);
}

int launch_sw16_coop(const SwArgs& a, int cls, bool tb, bool xd, int e_mode, cudaStream_t stream) {
    if (cls == CLS_I16_C2) return launch_coop_x<2>(a, tb, xd, e_mode, stream);
    if (cls == CLS_I16_C4) return launch_coop_x<4>(a, tb, xd, e_mode, stream);
    return launch_coop_x<8>(a, tb, xd, e_mode, stream);
}

// ---------------------------------------------------------------------------
// Deferred traceback walk of the batched form: one warp per pair, longest
// pairs first, after every DP kernel has stored its bits.  Running the walks
// as one wide kernel hides their scattered loads behind many warps and keeps
// the warps of the cooperative classes from idling while one warp walks.
// ---------------------------------------------------------------------------
template <class Lay>
__device__ void walk_pair(const SwArgs& a, const Grp<32>& grp, int p, const PairGeo& G, const Lay& lay) {
    const int bh = a.score[p], qe = a.q_end[p], te = a.t_end[p];
    RunWriter rw;
    uint32_t* runs = ws_alloc<32>(a, grp, (unsigned long long)qe + te + 1, bh > 0);
    const bool runs_ok = bh == 0 || runs != nullptr;
    if (!runs_ok && grp.k == 0) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
    rw.init(runs);
    int qs = 0, ts = 0;
    walk<32>(grp, lay, G, a, qe, te, bh, runs_ok && bh > 0, rw, qs, ts);
    finish_cigar<32>(a, grp, p, true, rw, runs_ok, qs, ts);
}

__global__ void __launch_bounds__(128) sw_walk_kernel(SwArgs a) {
    const int lane = threadIdx.x & 31;
    Grp<32> grp(lane);
    for (;;) {
        unsigned long long idx = 0;
        if (lane == 0) idx = atomicAdd(&a.counters[1], 1ull);
        idx = __shfl_sync(FULL_MASK, idx, 0);
        if (idx >= (unsigned long long)a.n_pairs) break;
        const int p = a.order ? a.order[idx] : (int)idx;
        const int tag = a.tb_tag[p];
        if (tag < 0) continue;  // no traceback: empty pair, bad band or workspace exhausted
        const PairGeo G = load_geo(a, p);
        const uint32_t* bits = a.pool + a.tb_base[p];
        if (tag == 0) {
            walk_pair(a, grp, p, G, Layout32{bits, imax(64, G.W + 1), G.W, G.qlen});
        } else if (tag == 8) {
            walk_pair(a, grp, p, G, Layout16<8>{bits, sw16_period(G.W, 8), G.W, G.qlen});
        } else if (tag == 16) {
            walk_pair(a, grp, p, G, Layout16<16>{bits, sw16_period(G.W, 16), G.W, G.qlen});
        } else {
            walk_pair(a, grp, p, G, Layout16<32>{bits, sw16_period(G.W, 32), G.W, G.qlen});
        }
    }
}

int launch_sw_walk(const SwArgs& a, cudaStream_t stream) {
    int dev = 0, sms = 0, per_sm = 0;
    GMF_CUDA_TRY(cudaGetDevice(&dev));
    GMF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    GMF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sw_walk_kernel, 128, 0));
    sw_walk_kernel<<<sms * (per_sm > 0 ? per_sm : 1), 128, 0, stream>>>(a);
    return cuda_status(cudaGetLastError());
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
