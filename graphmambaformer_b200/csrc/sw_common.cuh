// Shared machinery of the banded SW kernels (int32 and int16x2 forms):
// argument block, lane-group helpers, per-pair workspace allocation, the
// x-drop / best-cell post-pass and the warp-cooperative traceback walk.
//
// Reference semantics (graphmambaformer/alignment/extension.py L78-302) are
// restated at the top of sw32.cu; both kernel forms compute identical cell
// values and traceback decisions.
#pragma once

#include "gmf_common.cuh"

namespace gmf {

// Pair classes of the batched form (device-side classifier).
enum SwClass : int {
    CLS_I16_L8 = 0,   // 16x2, 8 lanes per pair (W <= 61)
    CLS_I16_L16 = 1,  // 16x2, 16 lanes per pair (W <= 125)
    CLS_I16_L32 = 2,  // 16x2, 32 lanes per pair
    CLS_I32 = 3,      // int32, 32 lanes per pair (scores beyond the 16-bit range)
    CLS_I16_C2 = 4,   // 16x2, 2 warps of one CTA per pair (264 <= P < 528)
    CLS_I16_C4 = 5,   // 16x2, 4 warps of one CTA per pair (528 <= P < 1056)
    CLS_I16_C8 = 6,   // 16x2, 8 warps of one CTA per pair (1056 <= P <= COOP_PMAX)
    N_CLASSES = 7
};

// Packed constants of the 16x2 form (each value in both 16-bit halves), on
// the gcd-scaled scoring; filled on the host so that kernels read them from
// the parameter bank instead of holding them in registers.
struct K16 {
    unsigned Z, NEGV, Z2, NEG2;  // biased zero and "-inf" (plain, packed)
    unsigned GO2, GE2, MATCH2;   // open, extend, match (packed)
    unsigned NGE2;               // -extend mod 2^16 (packed)
    unsigned MX;                 // match + mismatch (a mismatch flag times this is subtracted)
    unsigned EB2;                // 0x8000 - extend (packed): bit 15 of E_left - E + EB2 is E == E_left - extend
    int G;                       // gcd of the scoring: true score = scaled score * G
    // 1 and 2^32 - 1, read at run time: x * ONE + c and y * NEG1 + x are adds
    // and subtracts the compiler must issue as multiply-adds (FMA pipe)
    unsigned ONE, NEG1;
    __host__ __device__ unsigned init_pk() const { return Z | (NEGV << 16); }  // row 0: H = 0, F = -inf
};

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
    int32_t max_hb;
    int32_t zero16;                // biased zero of the 16x2 form: 4 * max penalty + 2
    int32_t neg16;                 // biased "-inf" of the 16x2 form: zero16 - (2 * max penalty + 2)
    // The 16x2 form runs on the scoring divided by g = gcd(match, mismatch,
    // open, extend): every cell value is a multiple of g, every decision is
    // a comparison of two cell values, so the scaled DP makes the same
    // decisions and its scores are the true scores / g.
    int32_t g16, m16, x16, o16, e16;  // g, and match / mismatch / open / extend divided by g
    K16 k16;                          // the 16x2 form's packed constants
    int32_t ring;                  // delay-line entries per lane group (power of two)
    unsigned long long* counters;  // [0] workspace words handed out (bump allocator)
    int32_t* queue;                // [N_CLASSES] heads, [N_CLASSES] counts
    int32_t* lists;                // N_CLASSES lists of n_pairs pair ids
    uint32_t* pool;                // traceback words, row maxima, CIGAR-run scratch
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
    int32_t defer_walk;              // batched form: DP kernels leave the walk to sw_walk_kernel
    int32_t l8w, l16w;               // classifier: widest bands of the 8- and 16-lane classes
    int32_t cmin[3];                 // classifier: fewest strips of the 2-, 4-, 8-warp classes (0: off)
    unsigned long long* tb_base;     // per pair: first traceback word (pool offset)
    int32_t* tb_tag;                 // per pair: traceback layout (0 int32, L for 16x2), -1 none
    const int32_t* xg_off;           // x-drop groups (n_xg+1 offsets), or null
    int32_t n_xg;
    unsigned long long* rm_base;     // per pair: row maxima (pool offset), ~0 none; null without groups
    int32_t* rm_seen;                // per pair: running row max carried between row chunks
    int32_t coop_spin_limit;         // polls before a wait between cooperating warps gives up
    int32_t coop_stall;              // test hook: writers never publish, so every wait runs out
};

// Polls (each followed by a ~20 ns sleep) before a wait between the warps of
// a cooperative class gives up and records GMF_SWF_TIMEOUT.
constexpr int COOP_WAIT_LIMIT = 1 << 22;

// Traceback-bit layout of the int32 form: one 32-bit word per lane per 8
// steps, 4 bits per step; virtual lane v of strip s handles slot d at step
// s*P + 2v + d.
struct Layout32 {
    const uint32_t* bits;
    int P, W, qlen;
    __device__ uint32_t nib(int i, int d) const {
        if (d < 0 || d >= W || i < 1 || i > qlen) return 0u;
        const int v = (i - 1) & 31, s = (i - 1) >> 5;
        const long long g = (long long)s * P + 2 * v + d;
        return (bits[(g >> 3) * 32 + v] >> ((int)(g & 7) * 4)) & 15u;
    }
};

// Where the deferred walk of pair p finds its traceback bits.
__device__ __forceinline__ void record_walk(const SwArgs& a, int p, const uint32_t* bits, int tag) {
    a.tb_base[p] = (unsigned long long)(bits - a.pool);
    a.tb_tag[p] = tag;
}

// Where the group x-drop pass finds the row maxima of pair p.
__device__ __forceinline__ void record_rowmax(const SwArgs& a, int p, const int2* rowmax) {
    if (a.rm_base) a.rm_base[p] = (unsigned long long)(reinterpret_cast<const uint32_t*>(rowmax) - a.pool);
}

// Pipeline period of the 16x2 form: steps per strip of 2L rows, a multiple of
// 4 so that rows start on 4-step chunk boundaries.
__host__ __device__ inline int sw16_period(int W, int L) {
    const int p = (W + 2 > 4 * L) ? W + 2 : 4 * L;
    return (p + 3) & ~3;
}

// Traceback words of one pair in the 16x2 form (one word per lane per chunk).
__host__ __device__ inline unsigned long long sw16_tb_words_l(int qlen, int W, int L) {
    const long long V = 2 * L;
    const long long P = sw16_period(W, L);
    const long long nstrips = (qlen + V - 1) / V;
    const long long last = (nstrips - 1) * P + 2 * ((qlen - 1) % V) + W - 1;
    return (unsigned long long)((last >> 2) + 1) * L;
}

// PTX byte permute in the generic mode: selector nibbles with bit 3 set
// replicate the sign of the selected byte.
__device__ __forceinline__ unsigned prmt(unsigned a, unsigned b, unsigned sel) {
    unsigned d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

__device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

__device__ __forceinline__ bool codes_match(int8_t qc, int8_t tc) {
    return qc == tc && qc >= 0 && qc != 5;
}

// A group of G consecutive lanes of a warp (G = 8, 16 or 32).  Every helper is
// called by all 32 lanes in lockstep.
template <int G>
struct Grp {
    int k;      // lane within the group
    int base;   // first warp lane of the group
    __device__ explicit Grp(int lane) : k(lane & (G - 1)), base(lane & ~(G - 1)) {}
    __device__ unsigned ballot(bool pred) const {
        const unsigned b = __ballot_sync(FULL_MASK, pred);
        return G == 32 ? b : (b >> base) & ((1u << G) - 1u);
    }
    template <class T>
    __device__ T shfl(T v, int src) const {
        return __shfl_sync(FULL_MASK, v, src, G);
    }
    template <class T>
    __device__ T up(T v, int d) const {
        return __shfl_up_sync(FULL_MASK, v, d, G);
    }
    template <class T>
    __device__ T xr(T v, int m) const {
        return __shfl_xor_sync(FULL_MASK, v, m, G);
    }
};

// Number of leading set bits of a G-bit ballot (G when all are set).
template <int G>
__device__ __forceinline__ int lead_ones(unsigned b) {
    const unsigned inv = ~b;
    const int f = __ffs(inv);
    return (f == 0 || f - 1 > G) ? G : f - 1;
}

// Run-length writer of the reversed CIGAR: group-uniform state, lane 0 stores.
struct RunWriter {
    uint32_t* buf;
    int n;
    int cur_op, cur_len;
    int c_eq, c_x, c_i, c_d;
    __device__ void init(uint32_t* b) {
        buf = b;
        n = 0;
        cur_op = -1;
        cur_len = 0;
        c_eq = c_x = c_i = c_d = 0;
    }
    __device__ void add(int op, int len, bool leader) {
        if (len <= 0) return;
        if (op == OP_EQ)
            c_eq += len;
        else if (op == OP_X)
            c_x += len;
        else if (op == OP_I)
            c_i += len;
        else
            c_d += len;
        if (op == cur_op) {
            cur_len += len;
            return;
        }
        if (cur_len > 0) {
            if (leader) buf[n] = ((uint32_t)cur_len << 4) | (uint32_t)cur_op;
            ++n;
        }
        cur_op = op;
        cur_len = len;
    }
    __device__ void flush(bool leader) {
        if (cur_len > 0) {
            if (leader) buf[n] = ((uint32_t)cur_len << 4) | (uint32_t)cur_op;
            ++n;
        }
        cur_len = 0;
    }
};

// Geometry of one pair.
struct PairGeo {
    int p;       // pair id (-1: none)
    int qlen, tlen, hb, off, W, P;
    const int8_t* q;
    const int8_t* t;
};

__device__ __forceinline__ PairGeo load_geo(const SwArgs& a, int p) {
    PairGeo G;
    G.p = p;
    if (p < 0) {
        G.qlen = G.tlen = 0;
        G.hb = G.off = 0;
        G.W = 1;
        G.P = 64;
        G.q = G.t = nullptr;
        return G;
    }
    const int64_t q0 = a.q_off[p], t0 = a.t_off[p];
    G.qlen = (int)(a.q_off[p + 1] - q0);
    G.tlen = (int)(a.t_off[p + 1] - t0);
    G.q = a.q + q0;
    G.t = a.t + t0;
    G.hb = a.hb[p];
    G.off = a.boff[p];
    G.W = 2 * G.hb + 1;
    G.P = 64;
    return G;
}

// Writes the all-zero result of a pair with no alignment (bad = invalid band
// or exhausted workspace, reported through the error word).
template <bool TB>
__device__ void write_empty(const SwArgs& a, int p, bool bad) {
    a.score[p] = 0;
    a.q_end[p] = 0;
    a.t_end[p] = 0;
    if (a.q_start) a.q_start[p] = 0;
    if (a.t_start) a.t_start[p] = 0;
    if (a.op_counts)
        for (int k = 0; k < 4; ++k) a.op_counts[4 * p + k] = 0;
    if (TB) {
        a.cigar_start[p] = 0;
        a.cigar_len[p] = bad ? -1 : 0;
    }
    if (bad) atomicOr(a.err, (int)GMF_SWF_WORKSPACE);
}

// Bump-allocates `words` (rounded to 16 bytes) of workspace for the group;
// returns nullptr for every lane when it does not fit.
template <int G>
__device__ uint32_t* ws_alloc(const SwArgs& a, const Grp<G>& grp, unsigned long long words, bool want) {
    unsigned long long base = 0;
    words = (words + 3) & ~3ull;
    if (grp.k == 0 && want && words) base = atomicAdd(&a.counters[0], words);
    base = grp.shfl(base, 0);
    if (!want || !words || base + words > a.pool_cap) return nullptr;
    return a.pool + base;
}

// Best cell from per-row maxima (row r at rowmax[r] = {row max, first slot}),
// applying the x-drop rule exactly as the reference's row loop: rows are taken
// in order, the best is updated on a strictly larger row max, and the row on
// which (max row max so far) - row max > x_drop is the last one considered.
// `active` groups run the scan; all lanes of the warp take part.
template <int G>
__device__ void xdrop_best(const Grp<G>& grp, const int2* rowmax, int qlen, int x_drop, bool active,
                           int& bh, int& bi, int& bd) {
    bh = 0;
    bi = 0;
    bd = 0;
    int seen = 0;
    bool done = !active;
    const int k = grp.k;
    for (int r0 = 0; __any_sync(FULL_MASK, !done); r0 += G) {
        if (!done && r0 >= qlen) done = true;
        const int r = r0 + k;
        const int2 v = (!done && r < qlen) ? rowmax[r] : make_int2(-1, 0);
        int pm = v.x;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            const int u = grp.up(pm, o);
            if (k >= o) pm = imax(pm, u);
        }
        pm = imax(pm, seen);
        const bool trig = !done && r < qlen && (pm - v.x > x_drop);
        const unsigned tm = grp.ballot(trig);
        const int last = tm ? __ffs(tm) - 1 : G - 1;
        int cv = (!done && k <= last && r < qlen) ? v.x : -1;
        int cl = k;
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            const int ov = grp.xr(cv, o);
            const int ol = grp.xr(cl, o);
            if (ov > cv || (ov == cv && ol < cl)) {
                cv = ov;
                cl = ol;
            }
        }
        const int cd = grp.shfl(v.y, cl);
        if (!done && cv > bh) {
            bh = cv;
            bi = r0 + cl + 1;
            bd = cd;
        }
        seen = grp.shfl(pm, G - 1);
        if (tm) done = true;
    }
}

// Warp-cooperative traceback from (qe, te) with the reference's decision
// order.  `Lay::nib(i, d)` returns the 4-bit cell code (0 outside the band):
// H source (0 stop, 1 diagonal, 2 F, 3 E), "F extends", "E extends".
// Each iteration the group fetches G cells of its current run -- diagonal
// (state H), vertical (state F) or horizontal (state E) -- and ballots give
// the run length and the =/X pattern.  Every lane of the warp executes the
// same collectives each iteration (groups of one warp may be in different
// states or already done); only group-uniform scalars depend on the state.
//
// The walk also carries the exact score of its current cell, starting from
// the best score: a diagonal step back subtracts the substitution score, a
// gap step adds the extension (or, where the gap opens, extension and open)
// penalty.  The reference stops in state H on a cell whose H is 0; the
// carried value gives that test, so layouts without a stop code (the 16x2
// form) stop exactly where the reference does.
template <int G, class Lay>
__device__ void walk(const Grp<G>& grp, const Lay& lay, const PairGeo& P, const SwArgs& a, int qe, int te,
                     int score, bool active, RunWriter& rw, int& i_out, int& j_out) {
    int i = qe, jj = te, state = 0;
    int v = score;  // H (state 0), F (state 1) or E (state 2) of the current cell
    bool walking = active && i > 0 && jj > 0;
    const int k = grp.k;
    const bool leader = k == 0;
    while (__any_sync(FULL_MASK, walking)) {
        const int d0 = jj - i - P.off + P.hb;
        const int ci = state == 2 ? i : i - k;
        const int cj = state == 1 ? jj : jj - k;
        const int dd = state == 0 ? d0 : (state == 1 ? d0 + k : d0 - k);
        const bool valid = walking && ci > 0 && cj > 0;
        const uint32_t nib = valid ? lay.nib(ci, dd) : 0u;
        // state H: the substitution score of each lane's cell, and the H value
        // there (the carried value minus the lanes before it)
        const bool is_eq = state == 0 && valid && codes_match(P.q[ci - 1], P.t[cj - 1]);
        const int sub = state == 0 && valid ? (is_eq ? a.match : -a.mismatch) : 0;
        int incl = sub;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) {
            const int t = grp.up(incl, o);
            if (k >= o) incl += t;
        }
        const int hval = v - (incl - sub);
        const uint32_t cbit = state == 0 ? (((nib & 3u) == 1u && hval > 0) ? 1u : 0u)
                                         : (state == 1 ? (nib & 4u) : (nib & 8u));
        const unsigned cont = grp.ballot(valid && cbit);
        const unsigned vm = grp.ballot(valid);
        const int c = lead_ones<G>(cont);
        const unsigned mm = grp.ballot(is_eq && k < c);
        const int at = c < G ? c : 0;
        const uint32_t nb = grp.shfl(nib, at);
        const int hv_at = grp.shfl(hval, at);
        const int total = grp.shfl(incl, G - 1);
        if (walking) {
            if (state == 0) {
                int pos = 0;
                while (pos < c) {  // the =/X runs of the c diagonal cells, in walk order
                    const unsigned rest = mm >> pos;
                    const bool eq = rest & 1u;
                    int len = eq ? lead_ones<32>(rest) : (rest ? __ffs(rest) - 1 : 32);
                    len = imin(len, c - pos);
                    rw.add(eq ? (int)OP_EQ : (int)OP_X, len, leader);
                    pos += len;
                }
                i -= c;
                jj -= c;
                if (c < G) {
                    const uint32_t code = nb & 3u;
                    if (!((vm >> c) & 1u) || code == 0 || hv_at <= 0) {
                        walking = false;  // off the matrix, or H <= 0: the alignment starts here
                    } else {
                        state = code == 2u ? 1 : 2;
                        v = hv_at;  // the gap state's value equals H here
                    }
                } else {
                    v -= total;
                }
            } else {
                const int gap_op = state == 1 ? (int)OP_I : (int)OP_D;
                int n;
                if (c == G) {
                    n = G;
                    v += G * a.gap_extend;
                } else if ((vm >> c) & 1u) {
                    n = c + 1;  // the cell that stops extending still emits its gap base
                    state = 0;
                    v += c * a.gap_extend + a.gap_open;  // H of the cell the gap opened from
                } else {
                    n = c;      // ran out of rows / columns
                }
                rw.add(gap_op, n, leader);
                if (gap_op == (int)OP_I)
                    i -= n;
                else
                    jj -= n;
            }
            if (i <= 0 || jj <= 0) walking = false;
        }
        __syncwarp();
    }
    i_out = i;
    j_out = jj;
}

// Copies the reversed runs into the dense CIGAR output and writes the pair's
// traceback results (group leader writes the scalars).
template <int G>
__device__ void finish_cigar(const SwArgs& a, const Grp<G>& grp, int p, bool active, RunWriter& rw,
                             bool runs_ok, int qs, int ts) {
    rw.flush(grp.k == 0);
    const int nruns = rw.n;
    unsigned long long cbase = 0;
    bool fits = runs_ok;
    if (grp.k == 0 && active && runs_ok && nruns > 0) cbase = atomicAdd(a.cigar_used, (unsigned long long)nruns);
    cbase = grp.shfl(cbase, 0);
    if (runs_ok && nruns > 0 && cbase + nruns > (unsigned long long)a.cigar_cap) {
        fits = false;
        if (grp.k == 0 && active) atomicOr(a.err, (int)GMF_SWF_CAPACITY);
    }
    __syncwarp();
    if (active && fits)
        for (int x = grp.k; x < nruns; x += G) a.cigar[cbase + x] = rw.buf[nruns - 1 - x];
    if (active && grp.k == 0) {
        if (a.q_start) a.q_start[p] = qs;
        if (a.t_start) a.t_start[p] = ts;
        if (a.op_counts) {
            a.op_counts[4 * p + 0] = rw.c_eq;
            a.op_counts[4 * p + 1] = rw.c_x;
            a.op_counts[4 * p + 2] = rw.c_i;
            a.op_counts[4 * p + 3] = rw.c_d;
        }
        a.cigar_start[p] = (int64_t)cbase;
        a.cigar_len[p] = fits ? nruns : -1;
    }
}

// Largest pipeline period of the cooperative classes (their rings hold P + 8
// entries per warp in shared memory).
constexpr int COOP_PMAX = 4088;

// Launch helpers implemented by the kernel translation units.
int launch_sw32(const SwArgs& a, bool tb, bool xd, int e_mode, bool queued, int grid, int wpb,
                cudaStream_t stream);
int launch_sw16(const SwArgs& a, int cls, bool tb, bool xd, int e_mode, int grid, int wpb,
                cudaStream_t stream);
int sw32_smem_per_warp(int ring);
int sw16_smem_per_warp(int cls, int ring);
int launch_sw16_coop(const SwArgs& a, int cls, bool tb, bool xd, int e_mode, cudaStream_t stream);
int launch_sw_walk(const SwArgs& a, cudaStream_t stream);
int sw16_coop_warps(int cls);

}  // namespace gmf
