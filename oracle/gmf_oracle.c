/*
 * gmf_oracle.c -- CPU restatement of GraphMambaFormer's classical alignment
 * hot path, used ONLY as test infrastructure (parity checker and the timed
 * CPU baseline).  Nothing in the shipped library links or calls this file.
 *
 * Parity anchor: every function below restates a reference function line by
 * line, with the reference's own arithmetic types, and was pinned against
 * outputs of the reference itself (golden fixtures in tests/golden/, made by
 * tests/golden/make_golden.py which imports the reference read-only).
 *
 *   oracle_sw_pair        graphmambaformer/alignment/extension.py L78-204
 *                         (banded_affine_sw_batch, called with B=1: f32
 *                         arithmetic, -1e30 sentinels, exclusive cummax scan
 *                         for E, first-index row max, strict '>' best update,
 *                         per-pair x-drop)
 *   oracle_sw_batch       the same with B > 1 per group: the group's row loop
 *                         stops after the first row on which every member
 *                         has dropped (L190-193); rows past a member's query
 *                         are empty (in_band needs i <= qlen)
 *   oracle_traceback_pair extension.py L207-302 (traceback_banded: f64
 *                         comparisons with tolerance 1e-3, out-of-matrix
 *                         cells read as -1e30, diag > F > E priority)
 *   oracle_chain_dp       alignment/chaining.py L129-180 (chain_dp_numpy:
 *                         f64 ((f[j] + adv) - pen) [+ bonus], first-max j,
 *                         take only when strictly > weight)
 *   oracle_chain_backtrack chaining.py L530-576 (_backtrack: stable argsort
 *                         of -f, claimed mask, partial-chain score)
 *   oracle_chain_select   chaining.py L579-617 (select + _read_overlap)
 *   oracle_wfa_align      extension.py L308-463 (WavefrontAligner.align +
 *                         _traceback: unit-cost global wavefronts from
 *                         diagonal 0, each candidate clipped on its own in
 *                         the forward pass, completion checked before the
 *                         max_distance test, traceback picks the first
 *                         largest of X, I, D without clipping)
 *   oracle_chain_read     chaining.py L620-642 (chain: strand +1 then -1,
 *                         for_strand / sorted_by_ref from alignment/types.py
 *                         L144-152, weight = length, no bonus)
 *
 * The penalty log2 term is never evaluated here: callers pass the table
 * pen_lut[g] = open + ext*g + coeff*log2(g+1) (0 for g = 0) computed with
 * numpy exactly as chaining.py L120-126 does, so the C code only performs
 * IEEE f64 add/sub/compare, in the reference's operation order.
 *
 * Build: oracle/build_oracle.py (gcc -O2 -ffp-contract=off -fno-fast-math).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NEG_F32 (-1e30f) /* torch.full(..., -1e30) in float32 */
#define NEG_F64 (-1e30)  /* the Python float returned by cell() for out-of-matrix */
#define N_CODE 5

/* CIGAR op codes shared with the CUDA library: = X I D S */
enum { OP_EQ = 0, OP_X = 1, OP_I = 2, OP_D = 3, OP_S = 4 };

typedef struct {
    float match, mismatch, gap_open, gap_extend, x_drop;
} sw_params;

/* ------------------------------------------------------------------------ */
/* Banded affine SW, one pair (extension.py L78-204, B = 1).                */
/* H/E/F are (qlen+1) x W row-major, row 0 initialised like the reference    */
/* (H zeros, E/F -1e30).  Returns the number of rows actually computed.     */
/* ------------------------------------------------------------------------ */
/* sw_rows: rows 1..min(qlen, max_rows); with own_xdrop the pair stops on   */
/* its own x-drop; row_best (optional) receives each computed row's best.   */
static int sw_rows(const int16_t* q, int32_t qlen, const int16_t* t, int32_t tlen, int32_t hb,
                   int32_t off, const sw_params* p, int32_t max_rows, int own_xdrop, float* H,
                   float* E, float* F, float* out_score, int64_t* out_qend, int64_t* out_tend,
                   float* row_best_out);

int oracle_sw_pair(const int16_t* q, int32_t qlen, const int16_t* t, int32_t tlen,
                   int32_t hb, int32_t off, const sw_params* p, float* H, float* E,
                   float* F, float* out_score, int64_t* out_qend, int64_t* out_tend) {
    return sw_rows(q, qlen, t, tlen, hb, off, p, qlen, 1, H, E, F, out_score, out_qend, out_tend, NULL);
}

static int sw_rows(const int16_t* q, int32_t qlen, const int16_t* t, int32_t tlen, int32_t hb,
                   int32_t off, const sw_params* p, int32_t max_rows, int own_xdrop, float* H,
                   float* E, float* F, float* out_score, int64_t* out_qend, int64_t* out_tend,
                   float* row_best_out) {
    const int W = 2 * hb + 1;
    const long rows = (long)qlen + 1;
    for (long k = 0; k < rows * W; ++k) {
        H[k] = 0.0f;
        E[k] = NEG_F32;
        F[k] = NEG_F32;
    }
    float* hprev = (float*)malloc(sizeof(float) * (W + 1));
    float* fprev = (float*)malloc(sizeof(float) * (W + 1));
    float* mrow = (float*)malloc(sizeof(float) * W);
    float* vrow = (float*)malloc(sizeof(float) * W);
    unsigned char* inb = (unsigned char*)malloc(W);
    float* scan_add = (float*)malloc(sizeof(float) * W);
    float* scan_sub = (float*)malloc(sizeof(float) * W);
    for (int d = 0; d < W; ++d) {
        /* d_index.to(float32) * ext ; open + (d - 1.0) * ext, all float32 */
        scan_add[d] = (float)d * p->gap_extend;
        scan_sub[d] = p->gap_open + ((float)d - 1.0f) * p->gap_extend;
    }
    for (int d = 0; d <= W; ++d) {
        hprev[d] = 0.0f;
        fprev[d] = NEG_F32;
    }
    float best = 0.0f, seen = 0.0f;
    int64_t bi = 0, bj = 0;
    int computed = 0;
    const int32_t last = max_rows < qlen ? max_rows : qlen;
    for (int i = 1; i <= last; ++i) {
        const int16_t qb = q[i - 1];
        for (int d = 0; d < W; ++d) {
            const long j = (long)i + off - hb + d;
            inb[d] = (j >= 1) && (j <= tlen);
            long tj = j - 1;
            if (tj < 0) tj = 0;
            if (tj > tlen - 1) tj = tlen - 1;
            const int16_t tb = (tlen > 0) ? t[tj] : (int16_t)-1;
            const int match = (qb == tb) && (qb >= 0) && (qb != N_CODE);
            const float sub = match ? p->match : -p->mismatch;
            const float diag = hprev[d] + sub;
            const float a = hprev[d + 1] - p->gap_open;
            const float b = fprev[d + 1] - p->gap_extend;
            const float vert = a > b ? a : b;
            float m = diag > vert ? diag : vert;
            if (m < 0.0f) m = 0.0f;
            mrow[d] = inb[d] ? m : NEG_F32;
            vrow[d] = vert;
        }
        /* inclusive = cummax(m + scan_add); exclusive shifted by one */
        float run = NEG_F32;
        float row_best = -1.0f;
        int row_slot = 0;
        for (int d = 0; d < W; ++d) {
            const float excl = (d == 0) ? NEG_F32 : run;
            float e = excl - scan_sub[d];
            if (!inb[d]) e = NEG_F32;
            const float x = mrow[d] + scan_add[d];
            run = (d == 0) ? x : (x > run ? x : run);
            float h = mrow[d] > e ? mrow[d] : e;
            if (h < 0.0f) h = 0.0f;
            if (!inb[d]) h = 0.0f;
            const float f = inb[d] ? vrow[d] : NEG_F32;
            H[(long)i * W + d] = h;
            E[(long)i * W + d] = e;
            F[(long)i * W + d] = f;
            if (h > row_best) { /* torch max: first index of the maximum */
                row_best = h;
                row_slot = d;
            }
        }
        if (row_best > best) {
            best = row_best;
            bi = i;
            bj = (int64_t)i + off - hb + row_slot;
        }
        if (row_best > seen) seen = row_best;
        for (int d = 0; d < W; ++d) {
            hprev[d] = H[(long)i * W + d];
            fprev[d] = F[(long)i * W + d];
        }
        hprev[W] = 0.0f;
        fprev[W] = NEG_F32;
        computed = i;
        if (row_best_out) row_best_out[i - 1] = row_best;
        if (own_xdrop && p->x_drop > 0.0f && (seen - row_best) > p->x_drop) break;
    }
    *out_score = best;
    *out_qend = bi;
    *out_tend = bj;
    free(hprev); free(fprev); free(mrow); free(vrow); free(inb);
    free(scan_add); free(scan_sub);
    return computed;
}

/* ------------------------------------------------------------------------ */
/* Traceback (extension.py L207-302).  ops_rev receives one op per column,  */
/* in the order they are emitted (end -> start).  Returns the op count.     */
/* ------------------------------------------------------------------------ */
static double cell(const float* M, long rows, int W, int hb, int off, long r, long c) {
    const long d = c - r - off + hb;
    if (r < 0 || r >= rows || d < 0 || d >= W) return NEG_F64;
    return (double)M[r * W + d];
}

long oracle_traceback_pair(const float* H, const float* E, const float* F, long rows,
                           int32_t hb, int32_t off, const int16_t* q, const int16_t* t,
                           int64_t qend, int64_t tend, const sw_params* p, unsigned char* ops_rev,
                           int64_t* read_start, int64_t* ref_start) {
    const int W = 2 * hb + 1;
    const double tol = 1e-3;
    const double match = p->match, mismatch = p->mismatch;
    const double gopen = p->gap_open, gext = p->gap_extend;
    long i = qend, j = tend, n = 0;
    int state = 0; /* 0 = H, 1 = F (vertical), 2 = E (horizontal) */
    while (i > 0 && j > 0) {
        if (state == 0) {
            const double h = cell(H, rows, W, hb, off, i, j);
            if (h <= 0.0) break;
            const int16_t qb = q[i - 1], tb = t[j - 1];
            const int matched = (qb == tb) && (qb >= 0) && (qb != N_CODE);
            const double sub = matched ? match : -mismatch;
            double up = cell(H, rows, W, hb, off, i - 1, j - 1);
            if (up < 0.0) up = 0.0;
            const double diag = up + sub;
            if (fabs(h - diag) <= tol) {
                ops_rev[n++] = matched ? OP_EQ : OP_X;
                i -= 1;
                j -= 1;
            } else if (fabs(h - cell(F, rows, W, hb, off, i, j)) <= tol) {
                state = 1;
            } else {
                state = 2;
            }
        } else if (state == 1) {
            const double cur = cell(F, rows, W, hb, off, i, j);
            ops_rev[n++] = OP_I;
            i -= 1;
            if (fabs(cur - (cell(H, rows, W, hb, off, i, j) - gopen)) <= tol)
                state = 0;
            else if (fabs(cur - (cell(F, rows, W, hb, off, i, j) - gext)) > tol)
                state = 0;
        } else {
            const double cur = cell(E, rows, W, hb, off, i, j);
            ops_rev[n++] = OP_D;
            j -= 1;
            if (fabs(cur - (cell(H, rows, W, hb, off, i, j) - gopen)) <= tol)
                state = 0;
            else if (fabs(cur - (cell(E, rows, W, hb, off, i, j) - gext)) > tol)
                state = 0;
        }
    }
    *read_start = i;
    *ref_start = j;
    return n;
}

/* Run-length encode forward ops (reverse of ops_rev) into (len << 4 | op). */
static long rle_reverse(const unsigned char* ops_rev, long n, uint32_t* out) {
    long runs = 0;
    for (long k = n - 1; k >= 0; --k) {
        const unsigned op = ops_rev[k];
        if (runs > 0 && (out[runs - 1] & 15u) == op)
            out[runs - 1] += 16u;
        else
            out[runs++] = (1u << 4) | op;
    }
    return runs;
}

/* ------------------------------------------------------------------------ */
/* Batched driver: SW + traceback, pthreads over x-drop groups.              */
/* A group is one call of the reference's banded_affine_sw_batch            */
/* (extension.py L78-204): its row loop stops only after the first row on   */
/* which every member has dropped (L190-193), and a member past its own     */
/* query length has an empty row (H = 0, row best 0).  group_off = NULL     */
/* makes every pair its own group.  cigar holds, for pair b, up to          */
/* cigar_cap[b] words at cigar_off[b].                                      */
/* ------------------------------------------------------------------------ */
typedef struct {
    int32_t n_pairs;
    const int16_t* q; const int64_t* q_off;
    const int16_t* t; const int64_t* t_off;
    const int32_t* hb; const int32_t* off;
    const sw_params* p;
    float* score; int64_t* q_end; int64_t* t_end; int64_t* q_start; int64_t* t_start;
    uint32_t* cigar; const int64_t* cigar_off; int32_t* cigar_n;
    int32_t* counts; /* 4 per pair: = X I D */
    int traceback;
    const int64_t* group_off; int32_t n_groups;
    int64_t next; /* work counter (groups) */
    pthread_mutex_t lock;
    int status;
} sw_job;

/* One pair: rows 1..min(qlen, max_rows), its own x-drop stop if own_xdrop,  */
/* then the traceback.  row_best: NULL, or one float per query row.         */
static int sw_member(sw_job* job, int64_t b, int32_t max_rows, int own_xdrop, int outputs,
                     float* row_best) {
    const int16_t* q = job->q + job->q_off[b];
    const int32_t qlen = (int32_t)(job->q_off[b + 1] - job->q_off[b]);
    const int16_t* t = job->t + job->t_off[b];
    const int32_t tlen = (int32_t)(job->t_off[b + 1] - job->t_off[b]);
    const int32_t hb = job->hb[b], off = job->off[b];
    const int W = 2 * hb + 1;
    const long rows = (long)qlen + 1;
    float* H = (float*)malloc(sizeof(float) * rows * W);
    float* E = (float*)malloc(sizeof(float) * rows * W);
    float* F = (float*)malloc(sizeof(float) * rows * W);
    if (!H || !E || !F) {
        free(H); free(E); free(F);
        return -1;
    }
    float sc; int64_t qe, te;
    sw_rows(q, qlen, t, tlen, hb, off, job->p, max_rows, own_xdrop, H, E, F, &sc, &qe, &te, row_best);
    if (outputs) {
        job->score[b] = sc;
        job->q_end[b] = qe;
        job->t_end[b] = te;
        if (job->traceback) {
            unsigned char* ops = (unsigned char*)malloc((size_t)qlen + (size_t)tlen + 2);
            int64_t rs, ts;
            const long n = oracle_traceback_pair(H, E, F, rows, hb, off, q, t, qe, te, job->p, ops,
                                                 &rs, &ts);
            job->q_start[b] = rs;
            job->t_start[b] = ts;
            int32_t c[4] = {0, 0, 0, 0};
            for (long k = 0; k < n; ++k) c[ops[k]]++;
            for (int k = 0; k < 4; ++k) job->counts[4 * b + k] = c[k];
            job->cigar_n[b] = (int32_t)rle_reverse(ops, n, job->cigar + job->cigar_off[b]);
            free(ops);
        }
    }
    free(H); free(E); free(F);
    return 0;
}

/* The row on which a group's loop stops: every member's rows without a stop, */
/* then the first row where (running max of row bests) - row best > x_drop   */
/* for all members.  Returns -1 when out of memory.                          */
static int32_t group_stop_row(sw_job* job, int64_t lo, int64_t hi) {
    int32_t maxq = 0;
    for (int64_t b = lo; b < hi; ++b) {
        const int32_t ql = (int32_t)(job->q_off[b + 1] - job->q_off[b]);
        if (ql > maxq) maxq = ql;
    }
    if (maxq == 0) return 0;
    const int64_t nm = hi - lo;
    float* rb = (float*)calloc((size_t)nm * (size_t)maxq, sizeof(float));
    float* seen = (float*)calloc((size_t)nm, sizeof(float));
    if (!rb || !seen) {
        free(rb); free(seen);
        return -1;
    }
    for (int64_t b = lo; b < hi; ++b) {
        const int32_t ql = (int32_t)(job->q_off[b + 1] - job->q_off[b]);
        if (sw_member(job, b, ql, 0, 0, rb + (b - lo) * maxq) != 0) {
            free(rb); free(seen);
            return -1;
        }
    }
    int32_t stop = maxq;
    for (int32_t i = 0; i < maxq; ++i) {
        int all = 1;
        for (int64_t m = 0; m < nm; ++m) {
            const float r = rb[m * maxq + i]; /* 0 past the member's query */
            if (r > seen[m]) seen[m] = r;
            if (!((seen[m] - r) > job->p->x_drop)) all = 0;
        }
        if (all) {
            stop = i + 1;
            break;
        }
    }
    free(rb); free(seen);
    return stop;
}

static void* sw_worker(void* arg) {
    sw_job* job = (sw_job*)arg;
    const int32_t n_groups = job->group_off ? job->n_groups : job->n_pairs;
    for (;;) {
        pthread_mutex_lock(&job->lock);
        const int64_t g = job->next++;
        pthread_mutex_unlock(&job->lock);
        if (g >= n_groups) break;
        const int64_t lo = job->group_off ? job->group_off[g] : g;
        const int64_t hi = job->group_off ? job->group_off[g + 1] : g + 1;
        const int grouped = (hi - lo > 1) && job->p->x_drop > 0.0f;
        const int32_t stop = grouped ? group_stop_row(job, lo, hi) : 0;
        if (stop < 0) {
            job->status = -1;
            continue;
        }
        for (int64_t b = lo; b < hi; ++b) {
            const int32_t ql = (int32_t)(job->q_off[b + 1] - job->q_off[b]);
            if (sw_member(job, b, grouped ? stop : ql, !grouped, 1, NULL) != 0) job->status = -1;
        }
    }
    return NULL;
}

int oracle_sw_batch(int32_t n_pairs, const int16_t* q, const int64_t* q_off, const int16_t* t,
                    const int64_t* t_off, const int32_t* hb, const int32_t* off,
                    const sw_params* p, int32_t traceback, int32_t n_threads, float* score,
                    int64_t* q_end, int64_t* t_end, int64_t* q_start, int64_t* t_start,
                    uint32_t* cigar, const int64_t* cigar_off, int32_t* cigar_n,
                    int32_t* counts, const int64_t* group_off, int32_t n_groups) {
    sw_job job = {n_pairs, q, q_off, t, t_off, hb, off, p, score, q_end, t_end, q_start, t_start,
                  cigar, cigar_off, cigar_n, counts, traceback, group_off, n_groups, 0,
                  PTHREAD_MUTEX_INITIALIZER, 0};
    if (n_threads < 1) n_threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * n_threads);
    for (int k = 0; k < n_threads; ++k) pthread_create(&th[k], NULL, sw_worker, &job);
    for (int k = 0; k < n_threads; ++k) pthread_join(th[k], NULL);
    free(th);
    return job.status;
}

/* ------------------------------------------------------------------------ */
/* Chaining DP (chaining.py L129-180).                                      */
/* bonus: NULL or (n, lookback) row-major; column c holds predecessor       */
/* i - lookback + c.                                                        */
/* ------------------------------------------------------------------------ */
void oracle_chain_dp(int64_t n, const int64_t* read_end, const int64_t* ref_end,
                     const double* weight, const double* bonus, int32_t max_lookback,
                     int64_t max_gap, const double* pen_lut, int64_t lut_len, double* f,
                     int64_t* parent) {
    const int64_t lookback = max_lookback > 1 ? max_lookback : 1;
    for (int64_t i = 0; i < n; ++i) {
        parent[i] = -1;
        const int64_t lo = i - lookback > 0 ? i - lookback : 0;
        if (lo == i) {
            f[i] = weight[i];
            continue;
        }
        double best = 0.0;
        int64_t best_j = -1;
        int any = 0;
        for (int64_t j = lo; j < i; ++j) {
            const int64_t dq = read_end[i] - read_end[j];
            const int64_t dr = ref_end[i] - ref_end[j];
            const int ok = dq > 0 && dr > 0 && dq <= max_gap && dr <= max_gap;
            double s;
            if (ok) {
                any = 1;
                const int64_t mn = dq < dr ? dq : dr;
                const double adv = (double)mn < weight[i] ? (double)mn : weight[i];
                const int64_t gap = dr > dq ? dr - dq : dq - dr;
                const double pen = gap < lut_len ? pen_lut[gap] : NAN;
                s = (f[j] + adv) - pen;
                if (bonus) s = s + bonus[i * lookback + (lookback - (i - lo)) + (j - lo)];
            } else {
                s = NEG_F64;
                /* the reference adds the bonus before masking, so masked
                   entries are exactly -1e30 */
            }
            if (best_j < 0 || s > best) { /* np.argmax: first maximum */
                best = s;
                best_j = j;
            }
        }
        if (!any) {
            f[i] = weight[i];
            continue;
        }
        if (best > weight[i]) {
            f[i] = best;
            parent[i] = best_j;
        } else {
            f[i] = weight[i];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Chain records.                                                           */
/* ------------------------------------------------------------------------ */
typedef struct {
    double score;
    int32_t strand;
    int64_t read_start, read_end, ref_start, ref_end;
    int64_t member_off; /* into a members scratch array */
    int64_t n_members;
    int32_t is_primary;
    int64_t order; /* position in the pre-select list (stable sort key) */
} oracle_chain;

typedef struct {
    const double* f;
    int64_t i;
} fidx;

static int cmp_f_desc(const void* a, const void* b) {
    const fidx* x = (const fidx*)a;
    const fidx* y = (const fidx*)b;
    /* argsort(-f, kind="stable"): ascending -f, ties by index */
    const double nx = -x->f[x->i], ny = -y->f[y->i];
    if (nx < ny) return -1;
    if (nx > ny) return 1;
    return (x->i > y->i) - (x->i < y->i);
}

/* _backtrack over one strand's sorted anchors.  global_idx maps sorted
   position -> original anchor index.  Appends to chains/members. */
static void backtrack(int64_t n, const double* f, const int64_t* parent, const int64_t* read_pos,
                      const int64_t* read_end, const int64_t* ref_pos, const int64_t* ref_end,
                      const int64_t* global_idx, int32_t strand, int64_t min_anchors,
                      double min_score, oracle_chain* chains, int64_t* n_chains,
                      int64_t* members, int64_t* n_members_total) {
    fidx* ord = (fidx*)malloc(sizeof(fidx) * (n > 0 ? n : 1));
    for (int64_t k = 0; k < n; ++k) {
        ord[k].f = f;
        ord[k].i = k;
    }
    qsort(ord, (size_t)n, sizeof(fidx), cmp_f_desc);
    unsigned char* claimed = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    int64_t* walk = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    for (int64_t k = 0; k < n; ++k) {
        const int64_t i = ord[k].i;
        if (claimed[i]) continue;
        int64_t m = 0, node = i;
        while (node >= 0 && !claimed[node]) {
            claimed[node] = 1;
            walk[m++] = node;
            node = parent[node];
        }
        const double score = f[i] - (node >= 0 ? f[node] : 0.0);
        if (m < min_anchors || score < min_score) continue;
        oracle_chain* c = &chains[(*n_chains)++];
        c->score = score;
        c->strand = strand;
        c->member_off = *n_members_total;
        c->n_members = m;
        c->is_primary = 0;
        int64_t rs = INT64_MAX, re = INT64_MIN, fs = INT64_MAX, fe = INT64_MIN;
        for (int64_t a = 0; a < m; ++a) {
            const int64_t loc = walk[m - 1 - a]; /* members.reverse(): read order */
            members[(*n_members_total)++] = global_idx[loc];
            if (read_pos[loc] < rs) rs = read_pos[loc];
            if (read_end[loc] > re) re = read_end[loc];
            if (ref_pos[loc] < fs) fs = ref_pos[loc];
            if (ref_end[loc] > fe) fe = ref_end[loc];
        }
        c->read_start = rs;
        c->read_end = re;
        c->ref_start = fs;
        c->ref_end = fe;
    }
    free(ord);
    free(claimed);
    free(walk);
}

void oracle_chain_backtrack(int64_t n, const double* f, const int64_t* parent,
                            const int64_t* read_pos, const int64_t* read_end,
                            const int64_t* ref_pos, const int64_t* ref_end,
                            const int64_t* global_idx, int32_t strand, int64_t min_anchors,
                            double min_score, double* c_score, int64_t* c_span /* 4/chain */,
                            int64_t* c_member_off, int64_t* c_n_members, int64_t* n_chains,
                            int64_t* members) {
    oracle_chain* chains = (oracle_chain*)malloc(sizeof(oracle_chain) * (n > 0 ? n : 1));
    int64_t nc = 0, nm = 0;
    backtrack(n, f, parent, read_pos, read_end, ref_pos, ref_end, global_idx, strand, min_anchors,
              min_score, chains, &nc, members, &nm);
    for (int64_t k = 0; k < nc; ++k) {
        c_score[k] = chains[k].score;
        c_span[4 * k + 0] = chains[k].read_start;
        c_span[4 * k + 1] = chains[k].read_end;
        c_span[4 * k + 2] = chains[k].ref_start;
        c_span[4 * k + 3] = chains[k].ref_end;
        c_member_off[k] = chains[k].member_off;
        c_n_members[k] = chains[k].n_members;
    }
    *n_chains = nc;
    free(chains);
}

static int cmp_chain_score(const void* a, const void* b) {
    const oracle_chain* x = (const oracle_chain*)a;
    const oracle_chain* y = (const oracle_chain*)b;
    const double nx = -x->score, ny = -y->score; /* sorted(key=-score), stable */
    if (nx < ny) return -1;
    if (nx > ny) return 1;
    return (x->order > y->order) - (x->order < y->order);
}

static double read_overlap(const oracle_chain* a, const oracle_chain* b) {
    const int64_t lo = a->read_start > b->read_start ? a->read_start : b->read_start;
    const int64_t hi = a->read_end < b->read_end ? a->read_end : b->read_end;
    if (hi <= lo) return 0.0;
    const int64_t sa = a->read_end - a->read_start, sb = b->read_end - b->read_start;
    int64_t den = sa < sb ? sa : sb;
    if (den < 1) den = 1;
    return (double)(hi - lo) / (double)den;
}

/* select (chaining.py L579-617).  chains[] is reordered in place; returns
   the number kept (they are chains[0..kept) afterwards). */
static int64_t select_chains(oracle_chain* chains, int64_t n, double ratio, double max_overlap,
                             int64_t max_chains) {
    if (n == 0) return 0;
    for (int64_t k = 0; k < n; ++k) chains[k].order = k;
    qsort(chains, (size_t)n, sizeof(oracle_chain), cmp_chain_score);
    const double cutoff = chains[0].score * ratio;
    int64_t kept = 0;
    for (int64_t k = 0; k < n; ++k) {
        oracle_chain c = chains[k];
        if (c.score < cutoff && kept) break;
        double overlap = 0.0;
        for (int64_t o = 0; o < kept; ++o) {
            if (!chains[o].is_primary) continue;
            const double ov = read_overlap(&c, &chains[o]);
            if (ov > overlap) overlap = ov;
        }
        if (overlap > max_overlap) continue;
        c.is_primary = kept == 0;
        chains[kept++] = c;
        if (kept >= max_chains) break;
    }
    return kept;
}

typedef struct {
    int32_t max_lookback;
    int64_t max_gap;
    int64_t min_chain_anchors;
    double min_chain_score;
    int64_t max_chains;
    double secondary_overlap;
    double secondary_score_ratio;
} chain_params;

typedef struct {
    int64_t i;
    const int64_t* re;
    const int64_t* fe;
} sidx;

static int cmp_lex(const void* a, const void* b) {
    /* np.lexsort((read_end, ref_end)): ref_end primary, read_end secondary,
       stable (original position as the last key) */
    const sidx* x = (const sidx*)a;
    const sidx* y = (const sidx*)b;
    if (x->fe[x->i] != y->fe[y->i]) return x->fe[x->i] < y->fe[y->i] ? -1 : 1;
    if (x->re[x->i] != y->re[y->i]) return x->re[x->i] < y->re[y->i] ? -1 : 1;
    return (x->i > y->i) - (x->i < y->i);
}

/* chain() for one read in fast mode (weight = length, no bonus).  Outputs up
   to max_chains chains; members_out receives each kept chain's global anchor
   indices back to back.  Returns the number of kept chains. */
int64_t oracle_chain_read(int64_t n, const int64_t* read_pos, const int64_t* ref_pos,
                          const int64_t* length, const int8_t* strand, const chain_params* cp,
                          const double* pen_lut, int64_t lut_len, double* out_score,
                          int32_t* out_strand, int64_t* out_span, int32_t* out_primary,
                          int64_t* out_n_members, int64_t* members_out) {
    if (n == 0) return 0;
    oracle_chain* chains = (oracle_chain*)malloc(sizeof(oracle_chain) * n);
    int64_t* members = (int64_t*)malloc(sizeof(int64_t) * n);
    int64_t nc = 0, nm = 0;
    int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * n);
    sidx* srt = (sidx*)malloc(sizeof(sidx) * n);
    int64_t *rp = malloc(8 * n), *re = malloc(8 * n), *fp = malloc(8 * n), *fe = malloc(8 * n);
    int64_t *gi = malloc(8 * n), *par = malloc(8 * n);
    double *w = malloc(8 * n), *f = malloc(8 * n);
    int64_t *re_all = malloc(8 * n), *fe_all = malloc(8 * n);
    for (int64_t k = 0; k < n; ++k) {
        re_all[k] = read_pos[k] + length[k];
        fe_all[k] = ref_pos[k] + length[k];
    }
    const int strands[2] = {1, -1};
    for (int s = 0; s < 2; ++s) {
        int64_t m = 0;
        for (int64_t k = 0; k < n; ++k)
            if (strand[k] == strands[s]) idx[m++] = k;
        if (m < cp->min_chain_anchors) continue;
        for (int64_t k = 0; k < m; ++k) {
            srt[k].i = idx[k];
            srt[k].re = re_all;
            srt[k].fe = fe_all;
        }
        qsort(srt, (size_t)m, sizeof(sidx), cmp_lex);
        for (int64_t k = 0; k < m; ++k) {
            const int64_t o = srt[k].i;
            rp[k] = read_pos[o];
            re[k] = re_all[o];
            fp[k] = ref_pos[o];
            fe[k] = fe_all[o];
            gi[k] = o;
            w[k] = (double)length[o];
        }
        oracle_chain_dp(m, re, fe, w, NULL, cp->max_lookback, cp->max_gap, pen_lut, lut_len, f, par);
        backtrack(m, f, par, rp, re, fp, fe, gi, strands[s], cp->min_chain_anchors,
                  cp->min_chain_score, chains, &nc, members, &nm);
    }
    const int64_t kept = select_chains(chains, nc, cp->secondary_score_ratio,
                                       cp->secondary_overlap, cp->max_chains);
    int64_t w_off = 0;
    for (int64_t k = 0; k < kept; ++k) {
        out_score[k] = chains[k].score;
        out_strand[k] = chains[k].strand;
        out_span[4 * k + 0] = chains[k].read_start;
        out_span[4 * k + 1] = chains[k].read_end;
        out_span[4 * k + 2] = chains[k].ref_start;
        out_span[4 * k + 3] = chains[k].ref_end;
        out_primary[k] = chains[k].is_primary;
        out_n_members[k] = chains[k].n_members;
        memcpy(members_out + w_off, members + chains[k].member_off,
               sizeof(int64_t) * chains[k].n_members);
        w_off += chains[k].n_members;
    }
    free(chains); free(members); free(idx); free(srt);
    free(rp); free(re); free(fp); free(fe); free(gi); free(par); free(w); free(f);
    free(re_all); free(fe_all);
    return kept;
}

/* Batched chain(): reads fanned out over pthreads.  Per read r the outputs
   occupy slots [r*max_chains, (r+1)*max_chains) and members occupy the read's
   own anchor range [read_off[r], read_off[r+1]). */
typedef struct {
    int64_t n_reads;
    const int64_t* read_off;
    const int64_t *read_pos, *ref_pos, *length;
    const int8_t* strand;
    const chain_params* cp;
    const double* lut;
    int64_t lut_len;
    double* score; int32_t* cstrand; int64_t* span; int32_t* primary; int64_t* n_members;
    int64_t* members; int32_t* n_chains;
    int64_t next;
    pthread_mutex_t lock;
} chain_job;

static void* chain_worker(void* arg) {
    chain_job* job = (chain_job*)arg;
    const int64_t mc = job->cp->max_chains;
    for (;;) {
        pthread_mutex_lock(&job->lock);
        const int64_t r = job->next++;
        pthread_mutex_unlock(&job->lock);
        if (r >= job->n_reads) break;
        const int64_t a0 = job->read_off[r], n = job->read_off[r + 1] - a0;
        job->n_chains[r] = (int32_t)oracle_chain_read(
            n, job->read_pos + a0, job->ref_pos + a0, job->length + a0, job->strand + a0, job->cp,
            job->lut, job->lut_len, job->score + r * mc, job->cstrand + r * mc,
            job->span + 4 * r * mc, job->primary + r * mc, job->n_members + r * mc,
            job->members + a0);
    }
    return NULL;
}

void oracle_chain_batch(int64_t n_reads, const int64_t* read_off, const int64_t* read_pos,
                        const int64_t* ref_pos, const int64_t* length, const int8_t* strand,
                        const chain_params* cp, const double* lut, int64_t lut_len,
                        int32_t n_threads, double* score, int32_t* cstrand, int64_t* span,
                        int32_t* primary, int64_t* n_members, int64_t* members,
                        int32_t* n_chains) {
    chain_job job = {n_reads, read_off, read_pos, ref_pos, length, strand, cp, lut, lut_len,
                     score, cstrand, span, primary, n_members, members, n_chains, 0,
                     PTHREAD_MUTEX_INITIALIZER};
    if (n_threads < 1) n_threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * n_threads);
    for (int k = 0; k < n_threads; ++k) pthread_create(&th[k], NULL, chain_worker, &job);
    for (int k = 0; k < n_threads; ++k) pthread_join(th[k], NULL);
    free(th);
}


/* ------------------------------------------------------------------------ */
/* Wavefront alignment (unit edit costs, global)                            */
/* ------------------------------------------------------------------------ */
static int64_t wfa_extend(int64_t i, int64_t k, const int16_t* q, int64_t n, const int16_t* t, int64_t m) {
    if (i < 0) return i;
    int64_t j = i - k;
    while (i < n && j >= 0 && j < m && q[i] == t[j] && q[i] >= 0 && q[i] != N_CODE) {
        ++i;
        ++j;
    }
    return i;
}

/* Edit distance and CIGAR words (run << 4 | op, op 0 '=', 1 'X', 2 'I',
 * 3 'D'); returns the distance, -1 when it exceeds max_distance, -2 when
 * out of memory.  *n_words receives the number of CIGAR words (cigar must
 * hold n + m + 2). */
int64_t oracle_wfa_align(const int16_t* q, int64_t n, const int16_t* t, int64_t m, int64_t max_distance,
                         uint32_t* cigar, int64_t* n_words) {
    *n_words = 0;
    if (n == 0 || m == 0) {
        if (n > 0) cigar[(*n_words)++] = ((uint32_t)n << 4) | 2u;
        if (m > 0) cigar[(*n_words)++] = ((uint32_t)m << 4) | 3u;
        return n > m ? n : m;
    }
    const int64_t final_k = n - m;
    /* history: wavefront s covers diagonals [-s, s], stored at s*s */
    int64_t cap = 1024;
    int64_t* H = (int64_t*)malloc(sizeof(int64_t) * cap);
    if (!H) return -2;
    H[0] = wfa_extend(0, 0, q, n, t, m);
    int64_t score = 0;
    for (;;) {
        /* completion of wavefront `score` */
        if (-score <= final_k && final_k <= score && H[score * score + (final_k + score)] >= n) break;
        if (score >= max_distance) {
            free(H);
            return -1;
        }
        ++score;
        const int64_t need = (score + 1) * (score + 1);
        if (need > cap) {
            while (cap < need) cap *= 2;
            int64_t* H2 = (int64_t*)realloc(H, sizeof(int64_t) * cap);
            if (!H2) {
                free(H);
                return -2;
            }
            H = H2;
        }
        const int64_t* prev = H + (score - 1) * (score - 1);
        const int64_t ps = score - 1;
        int64_t* cur = H + score * score;
        for (int64_t k = -score; k <= score; ++k) {
            int64_t cand[3];
            const int64_t pk[3] = {k, k - 1, k + 1};
            for (int c = 0; c < 3; ++c) {
                const int64_t idx = pk[c] + ps;
                int64_t v = (idx >= 0 && idx <= 2 * ps) ? prev[idx] : -1;
                if (c < 2) v = v >= 0 ? v + 1 : -1; /* substitution, insertion consume a query base */
                const int64_t col = v - k;
                if (v < 0 || v > n || col < 0 || col > m) v = -1;
                cand[c] = v;
            }
            int64_t best = cand[0] > cand[1] ? cand[0] : cand[1];
            best = best > cand[2] ? best : cand[2];
            cur[k + score] = wfa_extend(best, k, q, n, t, m);
        }
    }
    /* traceback */
    unsigned char* ops = (unsigned char*)malloc((size_t)(n + m + 2));
    if (!ops) {
        free(H);
        return -2;
    }
    int64_t n_ops = 0, k = final_k;
    for (int64_t s = score; s >= 1; --s) {
        const int64_t reach = H[s * s + (k + s)];
        const int64_t* prev = H + (s - 1) * (s - 1);
        const int64_t ps = s - 1;
        const int64_t pk[3] = {k, k - 1, k + 1};
        int64_t val[3];
        for (int c = 0; c < 3; ++c) {
            const int64_t idx = pk[c] + ps;
            const int64_t v = (idx >= 0 && idx <= 2 * ps && prev[idx] >= 0) ? prev[idx] : -1;
            val[c] = c < 2 ? (v >= 0 ? v + 1 : -1) : v;
        }
        int best = 0; /* first largest: X, then I, then D */
        for (int c = 1; c < 3; ++c)
            if (val[c] > val[best]) best = c;
        for (int64_t x = 0; x < reach - val[best]; ++x) ops[n_ops++] = 0; /* '=' */
        ops[n_ops++] = (unsigned char)(best == 0 ? 1 : (best == 1 ? 2 : 3));
        k = pk[best];
    }
    for (int64_t x = 0; x < H[k + 0]; ++x) ops[n_ops++] = 0; /* score-0 match run (k == 0) */
    *n_words = rle_reverse(ops, n_ops, cigar);
    free(ops);
    free(H);
    return score;
}
