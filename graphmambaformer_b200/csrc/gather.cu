// Segment gather of base codes (extension stage input building).
//
// The extension stage aligns each chain's query (the read, reverse-
// complemented for strand -1: graphmambaformer/alignment/seeding.py L64-81,
// reverse_complement_codes, complement table A<->T, C<->G, N and padding
// kept) against a window of the reference (alignment/extension.py L489-509,
// _window).  With the reference and the batch's reads resident on the
// device, both are slices of resident buffers; this kernel concatenates the
// slices of a batch into the CSR layout gmf_banded_sw reads.

#include "gmf_common.cuh"

namespace {

__device__ __forceinline__ int8_t complement_code(int8_t c) { return (c >= 1 && c <= 4) ? (int8_t)(5 - c) : c; }

__global__ void __launch_bounds__(256) gather_segments_kernel(const int8_t* __restrict__ src, int64_t src_len,
                                                              int n, const int64_t* __restrict__ start,
                                                              const int32_t* __restrict__ len,
                                                              const int8_t* __restrict__ rc, int8_t* __restrict__ dst,
                                                              const int64_t* __restrict__ dst_off) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int64_t s = start[i];
        const int L = len[i];
        const bool rev = rc != nullptr && rc[i] != 0;
        int8_t* d = dst + dst_off[i];
        for (int x = threadIdx.x; x < L; x += blockDim.x) {
            const int64_t pos = rev ? s + (L - 1 - x) : s + x;
            const int8_t c = (pos >= 0 && pos < src_len) ? src[pos] : (int8_t)-1;
            d[x] = rev ? complement_code(c) : c;
        }
    }
}

}  // namespace

extern "C" int gmf_gather_segments(const int8_t* src, int64_t src_len, int32_t n, const int64_t* start,
                                   const int32_t* len, const int8_t* rc, int8_t* dst, const int64_t* dst_off,
                                   gmf_stream_t stream) {
    if (n < 0 || src_len < 0) return GMF_ERR_INVALID_ARGUMENT;
    if (n == 0) return GMF_OK;
    if (!src || !start || !len || !dst || !dst_off) return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    const int blocks = n < 148 * 16 ? n : 148 * 16;
    gather_segments_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(src, src_len, n, start, len, rc, dst, dst_off);
    return gmf::cuda_status(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Diagonal spread of every kept chain: max - min of (ref_pos - read_pos) over
// the chain's member anchors, the widening term of the extension band
// (alignment/extension.py L489-509, _window: half_band + diagonal spread).
// One warp per read walks its chain records in slot order; lanes take the
// members of a chain in turn and a warp reduction gives the spread.
// ---------------------------------------------------------------------------
namespace {

__global__ void __launch_bounds__(128) chain_spread_kernel(int32_t n_reads, const int64_t* __restrict__ read_off,
                                                           const int32_t* __restrict__ read_pos,
                                                           const int32_t* __restrict__ ref_pos,
                                                           const int32_t* __restrict__ n_chains,
                                                           const int32_t* __restrict__ n_members,
                                                           const int32_t* __restrict__ members, int32_t max_chains,
                                                           int32_t* __restrict__ spread) {
    const int lane = threadIdx.x & 31;
    const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    for (int r = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5); r < n_reads; r += nw) {
        const int64_t a0 = read_off[r];
        const int nc = min(max(n_chains[r], 0), max_chains);
        int64_t m0 = a0;  // the members of slot k follow those of slots < k in the read's range
        for (int k = 0; k < max_chains; ++k) {
            int lo = 0x7fffffff, hi = (int)0x80000000;
            const int m = k < nc ? n_members[(int64_t)r * max_chains + k] : 0;
            for (int x = lane; x < m; x += 32) {
                const int64_t g = a0 + members[m0 + x];
                const int dg = ref_pos[g] - read_pos[g];
                lo = min(lo, dg);
                hi = max(hi, dg);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(gmf::FULL_MASK, lo, o));
                hi = max(hi, __shfl_xor_sync(gmf::FULL_MASK, hi, o));
            }
            if (lane == 0) spread[(int64_t)r * max_chains + k] = m > 0 ? hi - lo : 0;
            m0 += m;
        }
    }
}

}  // namespace

extern "C" int gmf_chain_spread(const gmf_anchor_batch* anchors, const gmf_chain_results* chains,
                                int32_t max_chains, int32_t* spread, gmf_stream_t stream) {
    if (!anchors || !chains || !spread || anchors->n_reads < 0 || max_chains < 1) return GMF_ERR_INVALID_ARGUMENT;
    if (anchors->n_reads == 0) return GMF_OK;
    if (!anchors->read_off || !anchors->read_pos || !anchors->ref_pos || !chains->n_chains || !chains->n_members ||
        !chains->members)
        return GMF_ERR_INVALID_ARGUMENT;
    GMF_BIND_STREAM(stream);
    const long long warps = anchors->n_reads < 148 * 32 ? anchors->n_reads : 148 * 32;
    chain_spread_kernel<<<(int)((warps + 3) / 4), 128, 0, (cudaStream_t)stream>>>(
        anchors->n_reads, anchors->read_off, anchors->read_pos, anchors->ref_pos, chains->n_chains,
        chains->n_members, chains->members, max_chains, spread);
    return gmf::cuda_status(cudaGetLastError());
}
