// Shared definitions of the gmf CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gmf_align.h"

namespace gmf {

constexpr unsigned FULL_MASK = 0xffffffffu;

// "Minus infinity" of the integer DP.  Every value the recurrences derive
// from it stays far below any real score (E and F never fall more than two
// gap penalties under it, because out-of-band cells are reset to it), and no
// sum involving it can overflow int32 for the parameter limits enforced by
// the host (penalties <= 2^20).
constexpr int NEG = -(1 << 29);

// CIGAR operation codes of the packed words (run << 4 | op).
enum : uint32_t { OP_EQ = 0, OP_X = 1, OP_I = 2, OP_D = 3, OP_S = 4 };

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? GMF_OK : GMF_ERR_CUDA; }

// Make the device that owns `stream` current for this thread (the library's
// CUDA runtime is private, so its current device follows the caller's stream
// rather than another runtime's state).  The legacy stream keeps the current
// device, and so does a stream that is being captured into a CUDA graph:
// asking a capturing stream for its device invalidates the capture, so a
// caller that captures makes the stream's device current first
// (gmf_set_device).  `prev` receives the device that was current when this
// call switched it, else stays -1.
inline int bind_stream_device(cudaStream_t stream, int* prev) {
    if (stream == nullptr) return GMF_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) return GMF_ERR_CUDA;
    if (cs != cudaStreamCaptureStatusNone) return GMF_OK;
    int dev = -1, cur = -1;
    if (cudaStreamGetDevice(stream, &dev) != cudaSuccess) return GMF_ERR_CUDA;
    if (cudaGetDevice(&cur) != cudaSuccess) return GMF_ERR_CUDA;
    if (dev != cur) {
        if (cudaSetDevice(dev) != cudaSuccess) return GMF_ERR_CUDA;
        *prev = cur;
    }
    return GMF_OK;
}

// An entry point's binding to its stream's device: the device that was
// current before the call is current again when the entry point returns, so
// no call changes its caller's current device.
struct StreamDeviceScope {
    int prev = -1;
    int status = GMF_OK;
    explicit StreamDeviceScope(cudaStream_t stream) { status = bind_stream_device(stream, &prev); }
    ~StreamDeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    StreamDeviceScope(const StreamDeviceScope&) = delete;
    StreamDeviceScope& operator=(const StreamDeviceScope&) = delete;
};

}  // namespace gmf

#define GMF_TRY(expr)              \
    do {                           \
        int _s = (expr);           \
        if (_s != GMF_OK) return _s; \
    } while (0)

// Binds the enclosing entry point to the device of `stream` until it returns.
#define GMF_BIND_STREAM(stream)                                         \
    gmf::StreamDeviceScope _gmf_device_scope((cudaStream_t)(stream));   \
    if (_gmf_device_scope.status != GMF_OK) return _gmf_device_scope.status

#define GMF_CUDA_TRY(expr)                          \
    do {                                            \
        cudaError_t _e = (expr);                    \
        if (_e != cudaSuccess) return GMF_ERR_CUDA; \
    } while (0)
