// SAM text of alignment records, rendered on the device.
//
// Semantics (graphmambaformer/data/formats.py L343-397, _make_segment, with
// data/alignment_io.py L55-106 and formats.py L287-289): a record is mapped
// when it names a known contig, has bases, a non-empty reference span and a
// non-empty CIGAR.  A mapped record on strand -1 is reoriented to the forward
// strand: FLAG 0x10, CIGAR runs in reverse order, SEQ reverse-complemented
// (A<->T, C<->G, anything else N), QUAL reversed.  Then, if the CIGAR's
// query-consuming length (= X I S) differs from the number of bases, the
// record is written unmapped after all, keeping 0x10 and the reoriented SEQ
// and QUAL.  Unmapped records: FLAG |= 0x4, RNAME '*', POS 0, MAPQ 0, CIGAR
// '*'.  Single-end records: RNEXT '*', PNEXT 0, TLEN 0.  QUAL is Phred+33 of
// the values clamped to [0, 93].  POS is 1-based.
//
// Layout: one warp per record.  A count pass gives every line's length; the
// caller scans them to offsets; the fill pass writes each line at its
// offset.  Lanes copy the name, bases, qualities and tags in parallel; the
// CIGAR runs are rendered 32 at a time with a warp scan of their text
// lengths.  The fill grid's second dimension splits the bases and qualities
// of long records into chunks of 2,048, each copied by a warp of its own
// (chunk 0 by the warp that writes the rest of the line), so a 20 kb read
// does not hold one warp for the whole pass.

#include "gmf_common.cuh"

namespace {

constexpr int SAM_WARPS = 4;

__device__ __forceinline__ int n_digits(long long v) {
    int d = 1;
    while (v >= 10) {
        v /= 10;
        ++d;
    }
    return d;
}

__device__ __forceinline__ char* put_num(char* p, long long v) {
    const int d = n_digits(v);
    for (int i = d - 1; i >= 0; --i) {
        p[i] = (char)('0' + (int)(v % 10));
        v /= 10;
    }
    return p + d;
}

__device__ __forceinline__ char comp_base(char b) {
    switch (b) {
        case 'A': return 'T';
        case 'C': return 'G';
        case 'G': return 'C';
        case 'T': return 'A';
        default: return 'N';
    }
}

__device__ __constant__ char k_ops[8] = {'=', 'X', 'I', 'D', 'S', 'M', 'N', 'H'};

// The record's CIGAR as runs: optional left clip, the words, optional right
// clip, with a clip merged into an adjacent S word (or the two clips into one
// run when there are no words).
struct Runs {
    const uint32_t* w;
    int nw;
    int cl, cr;      // clips, 0 when absent
    int lead, trail; // 1 when the clip is a run of its own
    int total;
    __device__ void init(const uint32_t* words, int n, int clip_l, int clip_r) {
        w = words;
        nw = n;
        cl = clip_l > 0 ? clip_l : 0;
        cr = clip_r > 0 ? clip_r : 0;
        if (nw == 0) {
            lead = (cl + cr) > 0 ? 1 : 0;
            trail = 0;
            cl += cr;
            cr = 0;
        } else {
            lead = (cl > 0 && (w[0] & 15u) != gmf::OP_S) ? 1 : 0;
            trail = (cr > 0 && (w[nw - 1] & 15u) != gmf::OP_S) ? 1 : 0;
        }
        total = lead + nw + trail;
    }
    // run i in forward order: (op, length)
    __device__ void get(int i, int& op, long long& len) const {
        if (i < lead) {
            op = gmf::OP_S;
            len = cl;
            return;
        }
        const int k = i - lead;
        if (k >= nw) {
            op = gmf::OP_S;
            len = cr;
            return;
        }
        op = (int)(w[k] & 15u);
        len = (long long)(w[k] >> 4);
        if (k == 0 && !lead && op == gmf::OP_S) len += cl;
        if (k == nw - 1 && !trail && op == gmf::OP_S) len += cr;
    }
};

struct Rec {
    long long name0, name_len, seq0, seq_len, tag0, tag_len;
    int contig, flag, mapq;
    long long pos;  // 1-based, 0 when unmapped
    bool mapped, rev;
    Runs runs;
    long long cigar_text;  // characters of the CIGAR column
};

// Everything about record r that the line needs; all lanes get the same.
__device__ Rec load_rec(const gmf_sam_records& R, int r, int lane) {
    Rec x;
    x.name0 = R.name_off[r];
    x.name_len = R.name_off[r + 1] - x.name0;
    x.seq0 = R.seq_off[r];
    x.seq_len = R.seq_off[r + 1] - x.seq0;
    x.tag0 = R.tag_off ? R.tag_off[r] : 0;
    x.tag_len = R.tag_off ? R.tag_off[r + 1] - x.tag0 : 0;
    x.contig = R.contig[r];
    const int nw = R.cigar_len[r] > 0 ? R.cigar_len[r] : 0;
    x.runs.init(R.cigar + (nw ? R.cigar_start[r] : 0), nw, R.clip_left ? R.clip_left[r] : 0,
                R.clip_right ? R.clip_right[r] : 0);
    bool mapped = x.contig >= 0 && x.contig < R.n_contigs && x.seq_len > 0 && R.ref_end[r] > R.ref_start[r] &&
                  x.runs.total > 0;
    int flag = 0;
    x.rev = false;
    if (mapped && R.strand[r] == -1) {
        flag |= 0x10;
        x.rev = true;
    }
    // query-consuming length and CIGAR text length, summed over the lanes
    long long qlen = 0, text = 0;
    for (int i = lane; i < x.runs.total; i += 32) {
        int op;
        long long len;
        x.runs.get(i, op, len);
        if (op == gmf::OP_EQ || op == gmf::OP_X || op == gmf::OP_I || op == gmf::OP_S || op == 5) qlen += len;
        text += n_digits(len) + 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        qlen += __shfl_xor_sync(gmf::FULL_MASK, qlen, o);
        text += __shfl_xor_sync(gmf::FULL_MASK, text, o);
    }
    if (mapped && qlen != x.seq_len) mapped = false;
    x.mapped = mapped;
    if (!mapped) flag |= 0x4;
    x.flag = flag;
    x.mapq = mapped ? R.mapq[r] : 0;
    x.pos = mapped ? R.ref_start[r] + 1 : 0;
    x.cigar_text = mapped ? text : 1;
    return x;
}

__device__ long long line_length(const gmf_sam_records& R, const Rec& x) {
    const long long rname = x.mapped ? (R.contig_off[x.contig + 1] - R.contig_off[x.contig]) : 1;
    long long n = x.name_len + 1 + n_digits(x.flag) + 1 + rname + 1 + n_digits(x.pos) + 1 + n_digits(x.mapq) + 1 +
                  x.cigar_text + 1 + 6 /* "*\t0\t0\t" */ + x.seq_len + 1 + x.seq_len;
    if (x.tag_len > 0) n += 1 + x.tag_len;
    return n + 1;  // newline
}

// Bases [lo, hi) of a record's SEQ and QUAL columns (SEQ at p, QUAL at
// p + L + 1): each lane loads 8 bases (and qualities) before it stores any,
// so a long stretch keeps 8 loads per lane in flight.
__device__ __forceinline__ void copy_bases(const gmf_sam_records& R, long long seq0, long long L, bool rev, char* p,
                                           long long lo, long long hi, int lane) {
    constexpr int U = 8;
    for (long long i0 = lo; i0 < hi; i0 += 32 * U) {
        char b[U];
        int qv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long i = i0 + u * 32 + lane;
            b[u] = 'N';
            qv[u] = 0;
            if (i < hi) {
                const long long src = seq0 + (rev ? L - 1 - i : i);
                b[u] = __ldg(R.seq + src);
                qv[u] = R.qual ? (int)__ldg(R.qual + src) : 0;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long i = i0 + u * 32 + lane;
            if (i < hi) {
                p[i] = rev ? comp_base(b[u]) : b[u];
                const int q = qv[u] > 93 ? 93 : qv[u];
                p[L + 1 + i] = (char)(33 + q);
            }
        }
    }
}

// Bases of chunk `y` of a record: [y*ch, (y+1)*ch), the last chunk of the
// grid taking everything to the end (so a low length hint stays correct).
__device__ __forceinline__ void chunk_range(long long L, long long ch, int y, int ny, long long& lo, long long& hi) {
    lo = (long long)y * ch;
    hi = (y == ny - 1) ? L : (lo + ch < L ? lo + ch : L);
    if (lo > L) lo = L;
}

template <bool FILL>
__global__ void __launch_bounds__(SAM_WARPS * 32) sam_kernel(gmf_sam_records R, int64_t* line_len,
                                                           const int64_t* line_off, char* out, long long ch) {
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    const int y = FILL ? (int)blockIdx.y : 0, ny = FILL ? (int)gridDim.y : 1;
    if (FILL && y > 0) {  // a later chunk of the bases: placed from the end of the line
        for (int r = gw; r < R.n_records; r += nw) {
            const long long s0 = R.seq_off[r], L = R.seq_off[r + 1] - s0;
            long long lo, hi;
            chunk_range(L, ch, y, ny, lo, hi);
            if (lo >= hi) continue;
            const long long tag_len = R.tag_off ? R.tag_off[r + 1] - R.tag_off[r] : 0;
            const int c = R.contig[r];
            const bool words = R.cigar_len[r] > 0 || (R.clip_left && R.clip_left[r] > 0) ||
                               (R.clip_right && R.clip_right[r] > 0);
            const bool rev = c >= 0 && c < R.n_contigs && L > 0 && R.ref_end[r] > R.ref_start[r] && words &&
                             R.strand[r] == -1;  // reoriented before the length check, as the first chunk is
            char* p = out + line_off[r + 1] - 1 - (tag_len > 0 ? 1 + tag_len : 0) - (2 * L + 1);
            copy_bases(R, s0, L, rev, p, lo, hi, lane);
        }
        return;
    }
    for (int r = gw; r < R.n_records; r += nw) {
        const Rec x = load_rec(R, r, lane);
        if (!FILL) {
            if (lane == 0) line_len[r] = line_length(R, x);
            continue;
        }
        char* p = out + line_off[r];
        // QNAME
        for (long long i = lane; i < x.name_len; i += 32) p[i] = R.name[x.name0 + i];
        p += x.name_len;
        // FLAG RNAME POS MAPQ (lane 0), then the CIGAR column
        long long at = 0;
        if (lane == 0) {
            char* q = p;
            *q++ = '\t';
            q = put_num(q, x.flag);
            *q++ = '\t';
            if (x.mapped) {
                const long long c0 = R.contig_off[x.contig], c1 = R.contig_off[x.contig + 1];
                for (long long i = c0; i < c1; ++i) *q++ = R.contig_names[i];
            } else {
                *q++ = '*';
            }
            *q++ = '\t';
            q = put_num(q, x.pos);
            *q++ = '\t';
            q = put_num(q, x.mapq);
            *q++ = '\t';
            at = q - p;
        }
        at = __shfl_sync(gmf::FULL_MASK, at, 0);
        p += at;
        if (!x.mapped) {
            if (lane == 0) p[0] = '*';
            p += 1;
        } else {
            long long base = 0;
            const int total = x.runs.total;
            for (int c0 = 0; c0 < total; c0 += 32) {
                const int i = c0 + lane;
                int op = 0;
                long long len = 0, w = 0;
                if (i < total) {
                    x.runs.get(x.rev ? total - 1 - i : i, op, len);
                    w = n_digits(len) + 1;
                }
                long long incl = w;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const long long u = __shfl_up_sync(gmf::FULL_MASK, incl, o);
                    if (lane >= o) incl += u;
                }
                if (i < total) {
                    char* q = put_num(p + base + incl - w, len);
                    *q = k_ops[op & 7];
                }
                base += __shfl_sync(gmf::FULL_MASK, incl, 31);
            }
            p += base;
        }
        if (lane == 0) {
            p[0] = '\t';
            p[1] = '*';
            p[2] = '\t';
            p[3] = '0';
            p[4] = '\t';
            p[5] = '0';
            p[6] = '\t';
        }
        p += 7;
        // SEQ and QUAL: this warp copies chunk 0 of the bases
        const long long L = x.seq_len;
        {
            long long lo, hi;
            chunk_range(L, ch, 0, ny, lo, hi);
            copy_bases(R, x.seq0, L, x.rev, p, lo, hi, lane);
        }
        if (lane == 0) p[L] = '\t';
        p += 2 * L + 1;
        if (x.tag_len > 0) {
            if (lane == 0) p[0] = '\t';
            for (long long i = lane; i < x.tag_len; i += 32) p[1 + i] = R.tags[x.tag0 + i];
            p += 1 + x.tag_len;
        }
        if (lane == 0) p[0] = '\n';
    }
}

int check(const gmf_sam_records* R) {
    if (!R || R->n_records < 0 || R->n_contigs < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (R->n_records == 0) return GMF_OK;
    if (!R->name || !R->name_off || !R->seq || !R->seq_off || !R->contig || !R->ref_start || !R->ref_end ||
        !R->strand || !R->mapq || !R->cigar || !R->cigar_start || !R->cigar_len)
        return GMF_ERR_INVALID_ARGUMENT;
    if (R->n_contigs > 0 && (!R->contig_names || !R->contig_off)) return GMF_ERR_INVALID_ARGUMENT;
    if (!R->tags != !R->tag_off) return GMF_ERR_INVALID_ARGUMENT;
    return GMF_OK;
}

int grid_of(int n) {
    const long long blocks = ((long long)n + SAM_WARPS - 1) / SAM_WARPS;
    return (int)(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

constexpr long long SAM_CHUNK = 2048;  // bases per warp in the fill pass

}  // namespace

extern "C" int gmf_sam_count(const gmf_sam_records* records, int64_t* line_len, gmf_stream_t stream) {
    GMF_TRY(check(records));
    if (records->n_records == 0) return GMF_OK;
    if (!line_len) return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    sam_kernel<false><<<grid_of(records->n_records), SAM_WARPS * 32, 0, (cudaStream_t)stream>>>(
        *records, line_len, nullptr, nullptr, SAM_CHUNK);
    return gmf::cuda_status(cudaGetLastError());
}

extern "C" int gmf_sam_fill(const gmf_sam_records* records, const int64_t* line_off, char* text,
                            gmf_stream_t stream) {
    GMF_TRY(check(records));
    if (records->n_records == 0) return GMF_OK;
    if (!line_off || !text) return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    // chunks of the longest record's bases (the last chunk takes any remainder)
    const long long mx = records->max_seq_len > 0 ? records->max_seq_len : 0;
    long long ny = (mx + SAM_CHUNK - 1) / SAM_CHUNK;
    ny = ny < 1 ? 1 : (ny > 65535 ? 65535 : ny);
    const long long ch = ny > 1 ? (mx + ny - 1) / ny : SAM_CHUNK;
    const dim3 grid((unsigned)grid_of(records->n_records), (unsigned)ny);
    sam_kernel<true><<<grid, SAM_WARPS * 32, 0, (cudaStream_t)stream>>>(*records, nullptr, line_off, text,
                                                                     ch < SAM_CHUNK ? SAM_CHUNK : ch);
    return gmf::cuda_status(cudaGetLastError());
}
