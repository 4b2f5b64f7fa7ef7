// Integer-ALU throughput probe for sm_100a: the roofline denominator of the
// banded SW kernel (MEASURED_PEAKS-style copy / GEMM figures do not cover the
// integer pipe).  Each thread runs 8 independent dependency chains so the
// measurement is throughput-bound, not latency-bound.
//   kind 0: x = max(x + a, y); y = max(y - b, x)      4 scalar int ops / chain step
//   kind 1: x = viaddmax(x, a, y); y = viaddmax(y, -b, x)  (DPX), 4 scalar-equivalent ops
//   kind 2: packed 16x2: x = vmax(vadd(x, a), y); y = ...  8 lane-ops (2 halves) per step
//   kinds 3-6 time single intrinsics (16x2 compares, DPX max forms, byte
//   permute / funnel shift) so their cost relative to one int32 op is known
//   kinds 7-9 time the unsigned 16x2 forms (max, min, three-way max, DPX
//   add-max) the biased-unsigned SW cells use
//   kinds 10-14 time single forms against a plain add / xor pair (kind 12):
//   packed add / sub, byte permute, DPX add-min + three-way max, multiply-add
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

template <int KIND>
__global__ void int_probe_kernel(int iters, int a, int b, int* out) {
    int x[8], y[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = threadIdx.x * 3 + k;
        y[k] = blockIdx.x + 7 * k;
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (KIND == 0) {
                x[k] = max(x[k] + a, y[k]);
                y[k] = max(y[k] - b, x[k]);
            } else if (KIND == 1) {
                x[k] = __viaddmax_s32(x[k], a, y[k]);
                y[k] = __viaddmax_s32(y[k], -b, x[k]);
            } else if (KIND == 2) {
                x[k] = (int)__vmaxs2(__vadd2((unsigned)x[k], (unsigned)a), (unsigned)y[k]);
                y[k] = (int)__vmaxs2(__vsub2((unsigned)y[k], (unsigned)b), (unsigned)x[k]);
            } else if (KIND == 3) {  // 16x2 compares (the traceback-bit primitives)
                x[k] = (int)__vcmpgts2((unsigned)x[k], (unsigned)y[k]) ^ a;
                y[k] = (int)__vcmpeq2((unsigned)y[k], (unsigned)x[k]) + b;
            } else if (KIND == 4) {  // DPX 16x2 max with relu and three-way max
                x[k] = (int)__vimax_s16x2_relu((unsigned)x[k], (unsigned)y[k]) + a;
                y[k] = (int)__vimax3_s16x2((unsigned)y[k], (unsigned)x[k], (unsigned)b);
            } else if (KIND == 5) {  // DPX max with predicate outputs
                bool p0, p1;
                x[k] = (int)__vibmax_s16x2((unsigned)x[k], (unsigned)y[k], &p0, &p1);
                y[k] = y[k] + (p0 ? a : b) + (p1 ? b : a);
            } else if (KIND == 7) {  // unsigned 16x2 max / min
                x[k] = (int)__vmaxu2((unsigned)x[k], (unsigned)y[k]) + a;
                y[k] = (int)__vminu2((unsigned)y[k], (unsigned)x[k]) ^ b;
            } else if (KIND == 8) {  // unsigned 16x2 three-way max + packed sub
                x[k] = (int)__vimax3_u16x2((unsigned)x[k], (unsigned)y[k], (unsigned)a);
                y[k] = (int)__vsub2((unsigned)y[k], (unsigned)x[k]);
            } else if (KIND == 9) {  // DPX unsigned 16x2 add-max
                x[k] = (int)__viaddmax_u16x2((unsigned)x[k], (unsigned)a, (unsigned)y[k]);
                y[k] = (int)__viaddmax_u16x2((unsigned)y[k], (unsigned)b, (unsigned)x[k]);
            } else if (KIND == 10) {  // packed 16x2 add / sub alone
                x[k] = (int)__vadd2((unsigned)x[k], (unsigned)a);
                y[k] = (int)__vsub2((unsigned)y[k], (unsigned)x[k]);
            } else if (KIND == 11) {  // byte permutes alone
                x[k] = (int)__byte_perm((unsigned)x[k], (unsigned)y[k], 0x5410);
                y[k] = (int)__byte_perm((unsigned)y[k], (unsigned)x[k], 0x7632) + a;
            } else if (KIND == 12) {  // plain add / xor (reference pair)
                x[k] = x[k] + a;
                y[k] = y[k] ^ x[k];
            } else if (KIND == 13) {  // DPX add-min (0/1 flags) and three-way max
                x[k] = (int)__viaddmin_u16x2((unsigned)x[k], 0u, (unsigned)y[k]);
                y[k] = (int)__vimax3_u16x2((unsigned)y[k], (unsigned)x[k], (unsigned)a);
            } else if (KIND == 14) {  // multiply-add
                x[k] = x[k] * a + y[k];
                y[k] = y[k] * b + x[k];
            } else {  // byte permute + funnel shift (exchange and bit packing)
                x[k] = (int)__byte_perm((unsigned)x[k], (unsigned)y[k], 0x5432) + a;
                y[k] = (int)__funnelshift_r((unsigned)y[k], (unsigned)x[k], 8);
            }
        }
    }
    int s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s ^= x[k] + y[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Float64 add / max chains (the chaining DP's arithmetic): 4 f64 ops per
// step on each of 8 independent chains per thread.
__global__ void f64_probe_kernel(int iters, double a, double b, double* out) {
    double x[8], y[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        x[k] = threadIdx.x * 0.5 + k;
        y[k] = blockIdx.x + 0.25 * k;
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            x[k] = fmax(x[k] + a, y[k]);
            y[k] = fmax(y[k] - b, x[k]);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k] + y[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Launch the float64 probe (4 * 8 * iters ops per thread).
extern "C" int gmf_probe_f64(int blocks, int threads, int iters, double* out, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    f64_probe_kernel<<<blocks, threads, 0, s>>>(iters, 0.75, 0.5, out);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Launch one probe; the caller times it with events on `stream`.
extern "C" int gmf_probe_int(int kind, int blocks, int threads, int iters, int* out, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    switch (kind) {
        case 0: int_probe_kernel<0><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
        case 1: int_probe_kernel<1><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
        case 2: int_probe_kernel<2><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 3: int_probe_kernel<3><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 4: int_probe_kernel<4><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 5: int_probe_kernel<5><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
        case 6: int_probe_kernel<6><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
        case 7: int_probe_kernel<7><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 8: int_probe_kernel<8><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 9: int_probe_kernel<9><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 10: int_probe_kernel<10><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        case 11: int_probe_kernel<11><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
        case 12: int_probe_kernel<12><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
        case 13: int_probe_kernel<13><<<blocks, threads, 0, s>>>(iters, 0x00030003, 0x00050005, out); break;
        default: int_probe_kernel<14><<<blocks, threads, 0, s>>>(iters, 3, 5, out); break;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Scalar-equivalent integer operations one probe launch performs.
extern "C" double gmf_probe_int_ops(int kind, int blocks, int threads, int iters) {
    // kind 2 counts 2 halves per op; the others count 2 ops (one pair of
    // intrinsic calls plus the int32 op that keeps each chain dependent)
    const double per_step = (kind == 2) ? 8.0 : 4.0;
    return per_step * 8.0 * (double)iters * blocks * threads;
}
