/*
 * gmf_align.h -- C ABI of the B200 (sm_100a) alignment hot path:
 * minimap2-style anchor-chaining DP and banded affine-gap Smith-Waterman
 * extension with CIGAR traceback.
 *
 * Conventions
 *   - Every pointer in a gmf_* struct or argument is a DEVICE pointer unless
 *     its comment says "host".  Buffers are owned by the caller.
 *   - Work is enqueued on the caller's stream; no entry point synchronises
 *     except where documented (none of the compute calls do).
 *   - Every entry point returns an int status, GMF_OK (0) on success.  No C++
 *     exception crosses this boundary.  gmf_status_string() names a status.
 *   - Results are deterministic per pair / per read and independent of the
 *     other work in the same call (band, x-drop and tie rules are applied per
 *     pair), so a pair aligned alone or inside a large batch gives the same
 *     score, coordinates and CIGAR.
 *   - No compute call allocates device memory: scratch lives in the
 *     caller's workspace (size it with the *_workspace_bytes helpers).  The
 *     exceptions are gmf_ctx_create and the gmf_batch_* calls, whose
 *     contexts own their staging and device arenas.
 *   - A call enqueues on the device that owns its stream and leaves the
 *     calling thread's current device as it found it.  On a stream that is
 *     being captured into a CUDA graph the library cannot ask the stream for
 *     its device, so there the stream's device must be current
 *     (gmf_set_device) when the call is made.
 *
 * Reference interfaces these entry points replace (GraphMambaFormer):
 *   gmf_banded_sw     graphmambaformer/accel/cuda_kernels.py L504-566 (banded_sw)
 *                     + alignment/extension.py L78-302
 *                     (banded_affine_sw_batch + traceback_banded)
 *   gmf_chain_dp      accel/cuda_kernels.py L440-501 (chain_dp)
 *                     + alignment/chaining.py L129-180 (chain_dp_numpy)
 *   gmf_chain_sort    alignment/types.py L144-152 (for_strand, sorted_by_ref)
 *   gmf_chain_batch   alignment/chaining.py L620-745 (AffineChainer.chain /
 *                     chain_batch: sort, DP, _backtrack, select)
 *   gmf_ctx_*, gmf_batch_*  the asynchronous serving form of gmf_banded_sw on
 *                     host buffers (the reference has none: its wrappers run
 *                     synchronously on the caller's tensors)
 *   gmf_sam_count/fill  data/formats.py L343-397 + L476-500 (SAM records)
 *   gmf_wfa_distance  accel/cuda_kernels.py L569-600 (wfa_distance)
 *   gmf_wfa_align     alignment/extension.py L308-463 (WavefrontAligner)
 */
#ifndef GMF_ALIGN_H
#define GMF_ALIGN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* gmf_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* ---- status codes ------------------------------------------------------ */
#define GMF_OK 0
#define GMF_ERR_INVALID_ARGUMENT 1 /* malformed request (NULL pointer, bad size, bad parameter) */
#define GMF_ERR_CUDA 2             /* a CUDA runtime call failed */
#define GMF_ERR_WORKSPACE 3        /* workspace smaller than required */
#define GMF_ERR_CAPACITY 4         /* an output buffer (CIGAR words, chains) is too small */
#define GMF_ERR_LIMIT 5            /* input beyond a documented size limit */
#define GMF_ERR_TIMEOUT 6          /* a bounded device-side wait expired */
#define GMF_ERR_NOT_READY 7        /* asynchronous work still in flight */
#define GMF_ERR_HOST 8             /* a host-side resource failed (memory, threads) */

const char* gmf_status_string(int status);
int gmf_version(void); /* major*10000 + minor*100 + patch */

/* The library links its own CUDA runtime.  Calls given a non-NULL stream run
 * on that stream's device; calls on the legacy stream (NULL), and calls made
 * while their stream is being captured into a CUDA graph, run on the device
 * selected here (default 0). */
int gmf_set_device(int device);

/* Limits enforced by the entry points (GMF_ERR_LIMIT beyond them). */
#define GMF_MAX_HALF_BAND 4096      /* band width W = 2*half_band+1 <= 8193 */
#define GMF_MAX_SEQ_LEN (1 << 28)   /* query / target length */
#define GMF_MAX_READ_ANCHORS 16384  /* anchors per read for gmf_chain_sort/batch */
#define GMF_MAX_LOOKBACK 1024       /* chaining predecessor window */

/* ======================================================================== */
/* Banded affine-gap Smith-Waterman with traceback                          */
/* ======================================================================== */

/* Integer scoring (the reference's defaults and every configuration it ships
 * are integral; scores are exact int32).  x_drop <= 0 disables x-drop. */
typedef struct {
    int32_t match_score;      /* > 0 */
    int32_t mismatch_penalty; /* >= 0, subtracted */
    int32_t gap_open;         /* >= 0, cost of the first gap base */
    int32_t gap_extend;       /* >= 0, cost of each further gap base */
    int32_t x_drop;           /* stop when (best row max so far) - (row max) > x_drop */
} gmf_sw_params;

/* A batch of read/target pairs in CSR layout.  Base codes follow the
 * reference alphabet: A=1 C=2 G=3 T=4 N=5, negative = padding; a query code
 * matches a target code iff they are equal, >= 0 and != 5.
 * Band slot d of query row i maps to target column
 *     j = i + band_offset - half_band + d,   0 <= d < 2*half_band+1. */
typedef struct {
    int32_t n_pairs;
    const int8_t* query;       /* concatenated query codes */
    const int64_t* query_off;  /* n_pairs+1 offsets into query */
    const int8_t* target;      /* concatenated target codes */
    const int64_t* target_off; /* n_pairs+1 offsets into target */
    const int32_t* half_band;  /* per pair, 0..GMF_MAX_HALF_BAND */
    const int32_t* band_offset;/* per pair */
    const int32_t* order;      /* optional processing order (a permutation of
                                  0..n_pairs-1, e.g. longest first); NULL = 0..n-1.
                                  It changes scheduling only, never results. */
    int32_t max_half_band;     /* HOST value >= every half_band[p] (sizes shared memory) */
    /* Optional x-drop groups (used only when x_drop > 0): pairs
     * [xdrop_group_off[g], xdrop_group_off[g+1]) are aligned as one batch of
     * the reference's row loop, which stops after the first row on which
     * EVERY member has dropped (rows past a member's query read as 0), so a
     * member keeps improving while another has not dropped.  Offsets are
     * non-decreasing from 0 to n_pairs.  NULL = every pair is its own group. */
    const int32_t* xdrop_group_off; /* n_xdrop_groups+1 offsets, device */
    int32_t n_xdrop_groups;
} gmf_pairs;

/* Per-pair outputs.  Ends are 1-based (0 when score == 0), starts 0-based,
 * exactly as banded_affine_sw_batch / traceback_banded report them.  The
 * CIGAR of pair p is cigar[cigar_start[p] .. + cigar_len[p]) as words
 * (run_length << 4) | op with op 0 '=', 1 'X', 2 'I', 3 'D' (soft clips are
 * added by the caller).  Pairs are packed densely in completion order; the
 * device counter *cigar_used receives the total number of words. */
typedef struct {
    int32_t* score;
    int32_t* query_end;
    int32_t* target_end;
    int32_t* query_start;        /* NULL allowed when cigar == NULL */
    int32_t* target_start;       /* NULL allowed when cigar == NULL */
    int32_t* op_counts;          /* 4 per pair (= X I D) or NULL */
    uint32_t* cigar;             /* NULL = score/end only (no traceback) */
    int64_t cigar_capacity;      /* words available in cigar */
    int64_t* cigar_start;        /* per pair */
    int32_t* cigar_len;          /* per pair, -1 if the pair overflowed cigar_capacity */
    unsigned long long* cigar_used; /* one device word, written by the call */
    int32_t* error_flags;        /* one device word: OR of GMF_SWF_* flags (written by the call) */
} gmf_sw_results;

#define GMF_SWF_WORKSPACE 1u /* a pair's traceback did not fit the workspace */
#define GMF_SWF_CAPACITY 2u  /* cigar_capacity exceeded */
#define GMF_SWF_TIMEOUT 4u   /* a bounded wait between the warps sharing a pair gave up (that
                                pair's result is unreliable); not expected in normal operation */
#define GMF_SWF_INTERNAL 8u  /* an internal consistency check failed (a distance that does not
                                belong to the pair); the pair is reported without a CIGAR */

/* Bytes of workspace gmf_banded_sw needs for a batch.  HOST arrays. */
size_t gmf_banded_sw_workspace_bytes(int32_t n_pairs, const int32_t* query_len,
                                     const int32_t* target_len, const int32_t* half_band,
                                     int32_t with_traceback);

/* Banded local alignment + traceback of every pair, batched form: a device
 * classifier puts each pair in a work list (int16x2 cells with 8/16/32 lanes
 * per pair by band width, or int32 cells when a score could leave int16) and
 * one persistent kernel per list pulls pairs until it is empty.  Results are
 * identical to gmf_banded_sw_plain for every pair.
 * Replaces accel/cuda_kernels.py L504-566 and extension.py L78-302. */
int gmf_banded_sw(const gmf_pairs* pairs, const gmf_sw_params* params,
                  const gmf_sw_results* results, void* workspace, size_t workspace_bytes,
                  gmf_stream_t stream);

/* Plain per-batch form: one warp per pair in input order, int32 cells, one
 * launch (the baseline the batched form is measured against).  Same inputs,
 * outputs and workspace as gmf_banded_sw. */
int gmf_banded_sw_plain(const gmf_pairs* pairs, const gmf_sw_params* params,
                        const gmf_sw_results* results, void* workspace, size_t workspace_bytes,
                        gmf_stream_t stream);

/* Concatenates n segments of base codes: segment i is src[start[i] ..
 * start[i] + len[i]) -- reversed and complemented (1<->4, 2<->3, other codes
 * kept) when rc is non-NULL and rc[i] != 0 -- written to dst[dst_off[i] ..].
 * Positions outside [0, src_len) read as -1 (padding).  Builds the query and
 * target codes of an extension batch from a resident reference and resident
 * reads.  Replaces the host-side window slicing of alignment/extension.py
 * L489-509 (_window) and seeding.py L64-81 (reverse_complement_codes). */
int gmf_gather_segments(const int8_t* src, int64_t src_len, int32_t n, const int64_t* start,
                        const int32_t* len, const int8_t* rc, int8_t* dst, const int64_t* dst_off,
                        gmf_stream_t stream);

/* ======================================================================== */
/* Minimizer seeding                                                        */
/* ======================================================================== */

/* A (w, k) minimizer index of a reference, resident on the device: sorted
 * unique packed k-mers (int64, 2 bits per base, A=0 .. T=3), CSR offsets and
 * the ascending reference positions of each key -- the table
 * alignment/seeding.py L202-254 (KmerTable.build) makes for MinimizerIndex
 * L524-538, max_occ already applied. */
typedef struct {
    int32_t k;              /* 1..31 */
    int32_t w;              /* 1..256 */
    int64_t n_keys;
    const int64_t* keys;
    const int64_t* offsets; /* n_keys + 1 */
    const int32_t* positions;
} gmf_minimizer_index;

/* Pass 1 of seeding a batch of reads (codes CSR, read_off[n_reads + 1]):
 * counts[2r] = anchors of read r, counts[2r + 1] = anchors of its reverse
 * complement (0 unless both_strands).  Replaces MinimizerIndex.query
 * (seeding.py L540-545) applied per orientation by SeedingEngine.seed_read
 * (L1056-1101) before diagonal merging. */
int gmf_seed_count(const gmf_minimizer_index* index, int32_t n_reads, const int8_t* codes,
                   const int64_t* read_off, int32_t both_strands, int64_t* counts, gmf_stream_t stream);

/* Pass 2: the anchors, at anchor_off[2r] (forward) and anchor_off[2r + 1]
 * (reverse complement, read_pos in the reverse-complemented read) with
 * anchor_off the exclusive prefix sum of the counts (2 * n_reads + 1
 * entries); within an orientation in the reference's order (read position,
 * then reference position).  length = k, strand = +1 / -1. */
int gmf_seed_fill(const gmf_minimizer_index* index, int32_t n_reads, const int8_t* codes,
                  const int64_t* read_off, int32_t both_strands, const int64_t* anchor_off,
                  int32_t* read_pos, int32_t* ref_pos, int32_t* length, int8_t* strand,
                  gmf_stream_t stream);

/* Scheduling knobs of the batched form (per device, process-wide).  They
 * decide which kernel shape aligns which pair and how the kernels overlap;
 * results never depend on them.  graphmambaformer_b200.autotune times
 * candidate settings on a sample of a workload and keeps the fastest.  No
 * counterpart in the reference (its batched kernel has one fixed shape). */
typedef struct {
    int32_t l8_max_w;           /* bands W = 2*half_band+1 up to this take 8 lanes per pair */
    int32_t l16_max_w;          /* ... up to this 16 lanes (>= l8_max_w); wider take a warp */
    int32_t coop_min_strips[3]; /* 2-, 4-, 8-warp classes: fewest 64-row strips a pair needs
                                   to be shared by that many warps; 0 disables the class */
    int32_t warps_per_block;    /* one-warp classes: warps per CTA, 1..4 */
    int32_t side_streams;       /* 1: class kernels overlap on side streams; 0: caller's stream */
} gmf_sw_tuning;

/* Current settings of the calling thread's current device (defaults: 61,
 * 125, {4, 8, 16}, 4, 1). */
int gmf_sw_get_tuning(gmf_sw_tuning* tuning);
/* Replace them (GMF_ERR_INVALID_ARGUMENT for out-of-range values).  Takes
 * effect for later gmf_banded_sw calls on that device. */
int gmf_sw_set_tuning(const gmf_sw_tuning* tuning);

/* Test hook of the cooperative classes' bounded waits (no counterpart in the
 * reference, whose CPU path has no waits).  A warp of a cooperative class
 * polls its predecessor's progress flag; after `spin_limit` polls (0 = the
 * default, about 2^22) it records GMF_SWF_TIMEOUT in the results' error
 * flags and goes on, so a call never hangs.  With `stall_writers` = 1 no
 * warp publishes its progress, so every wait runs out: the call returns with
 * GMF_SWF_TIMEOUT set and meaningless alignments.  Applies to every later
 * gmf_banded_sw call in the process until reset with (0, 0). */
int gmf_sw_test_coop_wait(int32_t spin_limit, int32_t stall_writers);

/* ======================================================================== */
/* Anchor chaining                                                          */
/* ======================================================================== */

typedef struct {
    int32_t max_lookback;           /* predecessors considered per anchor (>= 1) */
    int32_t max_gap;                /* reject pairs separated by more than this */
    int32_t min_chain_anchors;      /* chain filter */
    int32_t max_chains;             /* chains kept per read (select) */
    double min_chain_score;         /* chain filter */
    double secondary_overlap;       /* select: drop chains overlapping the primary more */
    double secondary_score_ratio;   /* select: drop chains below ratio * best */
} gmf_chain_params;

/* Chaining DP over rows that are already split by strand and sorted by
 * (ref_end, read_end) -- chain_dp_numpy semantics, float64 exact:
 *   f[i] = max(w_i, max_j ((f[j] + min(min(dq, dr), w_i)) - pen_lut[|dr-dq|]) [+ bonus])
 * over j in [i - lookback, i) with 0 < dq, dr <= max_gap; the lowest j wins
 * ties; the predecessor is taken only when strictly above w_i.
 * pen_lut[g] must hold gap_open + gap_extend*g + log_coeff*log2(g+1) (0 at
 * g = 0) for g = 0..max_gap, computed by the caller (numpy reproduces the
 * reference's log2 exactly).  bonus: NULL or per anchor max_lookback values,
 * column c for predecessor i - max_lookback + c.  parent is the row-local
 * predecessor index or -1.  Replaces cuda_kernels.py L440-501. */
int gmf_chain_dp(int32_t n_rows, const int64_t* row_off, const int32_t* read_end,
                 const int32_t* ref_end, const double* weight, const double* bonus,
                 int32_t max_lookback, int32_t max_gap, const double* pen_lut, int32_t lut_len,
                 double* f, int32_t* parent, gmf_stream_t stream);

/* Anchors of many reads in CSR layout, in each read's original order. */
typedef struct {
    int32_t n_reads;
    const int64_t* read_off; /* n_reads+1 */
    const int32_t* read_pos;
    const int32_t* ref_pos;
    const int32_t* length;
    const int8_t* strand;    /* +1 / -1 (anything else is ignored, like for_strand) */
} gmf_anchor_batch;

/* Sorted layout (written by gmf_chain_sort): per read, the + strand anchors
 * sorted by (ref_end, read_end, original index) followed by the - strand
 * anchors sorted the same way, stored in the read's own range
 * [read_off[r], read_off[r] + n_plus[r] + n_minus[r]). */
typedef struct {
    int32_t* perm;     /* sorted slot -> original index within the read */
    int32_t* n_plus;   /* per read */
    int32_t* n_minus;  /* per read */
    int32_t* read_end; /* sorted read_pos + length */
    int32_t* ref_end;  /* sorted ref_pos + length */
} gmf_sorted_anchors;

/* workspace: >= 256 + 24 * n_anchors bytes (gmf_chain_workspace_bytes is
 * always enough); it holds the sort of reads too large for shared memory. */
int gmf_chain_sort(const gmf_anchor_batch* anchors, const gmf_sorted_anchors* sorted,
                   void* workspace, size_t workspace_bytes, gmf_stream_t stream);

/* Per-read chain records, max_chains slots per read (slot k of read r at
 * r*max_chains + k), ordered as select() returns them.  members: the
 * original (within-read) anchor indices of the kept chains, back to back in
 * slot order and in read order within a chain, stored in the read's own range
 * [read_off[r], read_off[r+1]). */
typedef struct {
    int32_t* n_chains;   /* per read */
    double* score;       /* per slot */
    int32_t* strand;     /* per slot */
    int32_t* span;       /* 4 per slot: read_start, read_end, ref_start, ref_end */
    int32_t* is_primary; /* per slot */
    int32_t* n_members;  /* per slot */
    int32_t* members;    /* per anchor */
} gmf_chain_results;

size_t gmf_chain_workspace_bytes(int32_t n_reads, int64_t n_anchors);

/* Full AffineChainer.chain for every read: strand split + sort, DP, chain
 * peeling (_backtrack) and select.  sorted_weight / sorted_bonus are optional
 * inputs in the layout gmf_chain_sort produces (hybrid mode: gated weights and
 * graph / learned-transition bonus); NULL = weight is the anchor length, no
 * bonus (fast mode).  When given, `sorted` must hold the output of a prior
 * gmf_chain_sort on the same anchors; otherwise `sorted` may be NULL and the
 * sort runs inside the call (in the workspace). */
int gmf_chain_batch(const gmf_anchor_batch* anchors, const gmf_chain_params* params,
                    const double* pen_lut, int32_t lut_len, const gmf_sorted_anchors* sorted,
                    const double* sorted_weight, const double* sorted_bonus,
                    const gmf_chain_results* results, void* workspace, size_t workspace_bytes,
                    gmf_stream_t stream);

/* Diagonal spread of every chain record of gmf_chain_batch: spread[r *
 * max_chains + k] = max - min of (ref_pos - read_pos) over the member
 * anchors of read r's slot k (0 for empty slots).  The extension window's
 * band widening term, computed where the chain records are: replaces the
 * member loop of alignment/extension.py L489-509 (_window). */
int gmf_chain_spread(const gmf_anchor_batch* anchors, const gmf_chain_results* chains, int32_t max_chains,
                     int32_t* spread, gmf_stream_t stream);

/* ======================================================================== */
/* Chaining without device allocation                                       */
/* ======================================================================== */

/* Scratch held by gmf_chain_batch_noalloc: a fixed array inside this library,
 * present on every GPU that loads it, for as long as the process runs. */
#define GMF_CHAIN_NOALLOC_SCRATCH_BYTES ((size_t)32 << 20)

/* gmf_chain_batch in fast mode (weight = anchor length, no bonus) for callers
 * that cannot allocate device memory: a plugin host that hands over only its
 * input and output buffers, a process whose HBM is all held by a pool it does
 * not control, or a latency-bound loop that must not call cudaMalloc/cudaFree
 * (they synchronise the device).  Inputs and outputs are the caller's, as in
 * gmf_chain_batch; the scratch is the library's fixed array, so the call takes
 * no workspace.  There is no counterpart in the reference.
 *   n_anchors  HOST value: total anchors of the batch (read_off[n_reads]).
 *              GMF_ERR_LIMIT when gmf_chain_workspace_bytes(n_reads, n_anchors)
 *              exceeds GMF_CHAIN_NOALLOC_SCRATCH_BYTES (about 390,000 anchors).
 *   The first call on a device looks up the array's device address (once per
 *   device, under a lock), so make that first call before any stream capture;
 *   during a capture the stream's device must be the current device (see the
 *   conventions above).  The address is kept for the life of the process: a
 *   cudaDeviceReset between calls is not supported.
 *   A read with more than GMF_MAX_READ_ANCHORS anchors, or whose anchors lie
 *   beyond n_anchors (an understated n_anchors), gets zero chains and the
 *   call still returns GMF_OK; gmf_chain_noalloc_error_flags reports it.
 *   Every call shares the one array per device: calls whose work overlaps on
 *   the GPU (other streams, other threads) race and corrupt each other's
 *   results; serialise them, e.g. on one stream.  The array keeps the last
 *   call's contents; each call clears the parts that must start at zero. */
int gmf_chain_batch_noalloc(const gmf_anchor_batch* anchors, const gmf_chain_params* params,
                            const double* pen_lut, int32_t lut_len, int64_t n_anchors,
                            const gmf_chain_results* results, gmf_stream_t stream);

/* Error word of the last gmf_chain_batch_noalloc call on the stream's device,
 * copied into *flags (device or host memory) on `stream`; with host memory,
 * read it after the stream has synchronised.  Bits: 1 = a read had more than
 * GMF_MAX_READ_ANCHORS anchors, 2 = a read's sort did not fit the scratch,
 * 4 = a read's anchors lay beyond n_anchors; each such read got zero chains.
 * 0 = every read was chained.  No counterpart in the reference (its chainer
 * raises on the host instead). */
int gmf_chain_noalloc_error_flags(int32_t* flags, gmf_stream_t stream);

/* ======================================================================== */
/* Contexts and asynchronous batches on HOST buffers                        */
/* ======================================================================== */

/* A context owns, on one device, `slots` (1..8) slots of a stream, pinned
 * staging memory and a device arena (inputs, outputs and workspace of one
 * batch): up to `slots` batches in flight.  A slot may hold up to
 * memory_budget / slots bytes of device memory (memory_budget 0 = no limit);
 * its arena grows, never shrinks.  One context serves any number of threads
 * (calls are serialised inside). */
typedef struct gmf_ctx gmf_ctx;

int gmf_ctx_create(int device, int32_t slots, size_t memory_budget, gmf_ctx** ctx);
int gmf_ctx_destroy(gmf_ctx* ctx); /* waits for the batches in flight */

/* A batch in HOST memory, read only during gmf_batch_submit (fields as in
 * gmf_pairs; the processing order is chosen inside). */
typedef struct {
    int32_t n_pairs;
    const int8_t* query;
    const int64_t* query_off;  /* n_pairs+1, from 0 */
    const int8_t* target;
    const int64_t* target_off; /* n_pairs+1, from 0 */
    const int32_t* half_band;
    const int32_t* band_offset;
    const int32_t* xdrop_group_off; /* optional, as in gmf_pairs */
    int32_t n_xdrop_groups;
} gmf_host_pairs;

/* HOST outputs (layout as in gmf_sw_results), written when the batch
 * completes: gmf_batch_poll returns GMF_OK, or gmf_batch_wait returns. */
typedef struct {
    int32_t* score;
    int32_t* query_end;
    int32_t* target_end;
    int32_t* query_start;      /* with cigar */
    int32_t* target_start;     /* with cigar */
    int32_t* op_counts;        /* 4 per pair or NULL */
    uint32_t* cigar;           /* NULL = score and ends only */
    int64_t cigar_capacity;    /* words */
    int64_t* cigar_start;      /* with cigar */
    int32_t* cigar_len;        /* with cigar */
    int64_t* cigar_used;       /* words written */
    int32_t* error_flags;      /* GMF_SWF_* of the batch */
} gmf_host_sw_results;

/* Enqueue one batch of gmf_banded_sw: the inputs go to the device in one
 * copy, the kernels run on the slot's stream and the fixed-size outputs come
 * back in one copy, all asynchronously.  Slots are taken in turn; when the
 * next one still holds a batch, that batch is completed first (its outputs
 * written; its ticket then reports GMF_OK once).  GMF_ERR_LIMIT when the
 * batch needs more than a slot's share of the budget.  *ticket identifies the
 * batch. */
int gmf_batch_submit(gmf_ctx* ctx, const gmf_host_pairs* pairs, const gmf_sw_params* params,
                     const gmf_host_sw_results* results, int64_t* ticket);

/* GMF_OK once the batch is complete and its outputs written (reported once
 * per ticket), GMF_ERR_NOT_READY while it is in flight,
 * GMF_ERR_INVALID_ARGUMENT for an unknown ticket. */
int gmf_batch_poll(gmf_ctx* ctx, int64_t ticket);

/* As gmf_batch_poll, blocking until the batch completes. */
int gmf_batch_wait(gmf_ctx* ctx, int64_t ticket);

/* ======================================================================== */
/* SAM text of alignment records                                            */
/* ======================================================================== */

/* Records to render as SAM lines (all device arrays; offsets from 0).  A
 * record is mapped when contig >= 0, it has bases, ref_end > ref_start and a
 * non-empty CIGAR; then, as the reference writes it, strand -1 reorients it
 * (FLAG 0x10, CIGAR runs reversed, SEQ reverse-complemented, QUAL reversed),
 * and a CIGAR whose query length (= X I S M) differs from the number of bases
 * makes it unmapped after all.  Unmapped: FLAG 0x4, RNAME '*', POS 0, MAPQ 0,
 * CIGAR '*'.  Columns 7-9 are '*', 0, 0 (single-end). */
typedef struct {
    int32_t n_records;
    const char* name;            /* QNAME bytes */
    const int64_t* name_off;     /* n_records+1 */
    const char* seq;             /* bases as given (ASCII) */
    const int64_t* seq_off;      /* n_records+1 */
    const uint8_t* qual;         /* Phred value per base (seq_off layout), NULL = all 0; clamped to 93 */
    const int32_t* contig;       /* per record: contig index, -1 = no alignment */
    const char* contig_names;    /* RNAME bytes of each contig */
    const int64_t* contig_off;   /* n_contigs+1 */
    int32_t n_contigs;
    const int64_t* ref_start;    /* 0-based */
    const int64_t* ref_end;
    const int8_t* strand;        /* +1 / -1 */
    const int32_t* mapq;
    const uint32_t* cigar;       /* words (run << 4) | op: 0 '=', 1 'X', 2 'I', 3 'D', 4 'S', 5 'M', 6 'N', 7 'H' */
    const int64_t* cigar_start;  /* per record */
    const int32_t* cigar_len;    /* per record, words */
    const int32_t* clip_left;    /* optional soft clips around the words (NULL = none), merged with an */
    const int32_t* clip_right;   /* adjacent S word */
    const char* tags;            /* optional tag text per record (tab-separated fields), NULL = none */
    const int64_t* tag_off;      /* n_records+1 with tags */
    int64_t max_seq_len;         /* HOST value: the longest record's bases (splits the fill pass over
                                    more warps; 0 or too low costs speed, never correctness) */
} gmf_sam_records;

/* Length in bytes of every record's line (newline included). */
int gmf_sam_count(const gmf_sam_records* records, int64_t* line_len, gmf_stream_t stream);

/* Write every record's line at text + line_off[r], where line_off holds
 * n_records+1 entries: the exclusive scan of the lengths and their total.  Replaces data/formats.py L343-397 (_make_segment) and the SAM
 * rendering of write_sam (L476-500) for single-end records. */
int gmf_sam_fill(const gmf_sam_records* records, const int64_t* line_off, char* text, gmf_stream_t stream);

/* ======================================================================== */
/* Unit-cost global wavefront alignment (WFA)                               */
/* ======================================================================== */

#define GMF_MAX_WFA_DISTANCE (1 << 16) /* distance bound of a call */

/* Pairs aligned end to end (codes and matching as in gmf_pairs). */
typedef struct {
    int32_t n_pairs;
    const int8_t* query;       /* concatenated query codes */
    const int64_t* query_off;  /* n_pairs+1 offsets into query */
    const int8_t* target;      /* concatenated target codes */
    const int64_t* target_off; /* n_pairs+1 offsets into target */
    const int32_t* order;      /* optional processing order (a permutation); NULL = 0..n-1.
                                  It changes scheduling only, never results. */
    int64_t query_total;       /* HOST value: query_off[n_pairs] */
    int64_t target_total;      /* HOST value: target_off[n_pairs] */
    int32_t max_len;           /* HOST value >= every query and target length */
} gmf_wfa_pairs;

/* Per-pair outputs of gmf_wfa_align.  The CIGAR of pair p is
 * cigar[cigar_start[p] .. + cigar_len[p]) as words (run << 4) | op, op 0 '=',
 * 1 'X', 2 'I', 3 'D', packed densely in completion order; cigar_len[p] is -1
 * when the pair has no alignment (distance -1), its history did not fit the
 * workspace (GMF_SWF_WORKSPACE) or its words did not fit cigar_capacity
 * (GMF_SWF_CAPACITY). */
typedef struct {
    int32_t* op_counts;          /* 4 per pair (= X I D) or NULL */
    uint32_t* cigar;
    int64_t cigar_capacity;      /* words available in cigar (n + m + 1 per pair always suffice) */
    int64_t* cigar_start;        /* per pair */
    int32_t* cigar_len;          /* per pair */
    unsigned long long* cigar_used; /* one device word, written by the call */
    int32_t* error_flags;        /* one device word: OR of GMF_SWF_* flags (written by the call) */
} gmf_wfa_results;

/* Bytes of workspace for a WFA call: gmf_wfa_distance needs
 * history_entries = 0; gmf_wfa_align needs the total of (d+1)^2 over its pairs
 * (gmf_wfa_history_entries), or less, in which case the pairs that do not fit
 * are reported and can be retried.  max_distance: the call's bound
 * (gmf_wfa_align: >= every distance). */
size_t gmf_wfa_workspace_bytes(int32_t n_pairs, int32_t max_len, int32_t max_distance,
                               int64_t history_entries);

/* Sum over pairs of (distance+1)^2 (pairs with distance -1 or an empty side
 * count 0).  HOST arrays; -1 on a bad argument. */
int64_t gmf_wfa_history_entries(int32_t n_pairs, const int32_t* query_len, const int32_t* target_len,
                                const int32_t* distance);

/* Edit distance of every pair, or -1 when it exceeds max_distance (where the
 * reference raises).  An empty side answers max(n, m) whatever the bound.
 * Replaces accel/cuda_kernels.py L569-600 (wfa_distance) and the distance of
 * alignment/extension.py L353-408 (WavefrontAligner.align). */
int gmf_wfa_distance(const gmf_wfa_pairs* pairs, int32_t max_distance, int32_t* distance,
                     void* workspace, size_t workspace_bytes, gmf_stream_t stream);

/* CIGAR of every pair from the distances of a prior gmf_wfa_distance (device
 * array) on the same pairs: the wavefronts are recomputed to that distance
 * with their history kept, then walked back (ties: X, then I, then D).
 * max_distance: HOST value >= every distance[p].  Replaces
 * alignment/extension.py L410-463 (WavefrontAligner._traceback). */
int gmf_wfa_align(const gmf_wfa_pairs* pairs, const int32_t* distance, int32_t max_distance,
                  const gmf_wfa_results* results, void* workspace, size_t workspace_bytes,
                  gmf_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* GMF_ALIGN_H */
