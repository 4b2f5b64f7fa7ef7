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
