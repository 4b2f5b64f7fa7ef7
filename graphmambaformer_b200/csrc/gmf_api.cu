// Library-level entry points of the C ABI (status strings, version).
#include "gmf_common.cuh"

extern "C" const char* gmf_status_string(int status) {
    switch (status) {
        case GMF_OK: return "ok";
        case GMF_ERR_INVALID_ARGUMENT: return "invalid argument";
        case GMF_ERR_CUDA: return "CUDA runtime error";
        case GMF_ERR_WORKSPACE: return "workspace too small";
        case GMF_ERR_CAPACITY: return "output capacity exceeded";
        case GMF_ERR_LIMIT: return "input beyond a supported size limit";
        case GMF_ERR_TIMEOUT: return "bounded device wait expired";
        case GMF_ERR_NOT_READY: return "work still in flight";
        case GMF_ERR_HOST: return "host resource failure";
        default: return "unknown status";
    }
}

extern "C" int gmf_version(void) { return 1 * 10000 + 0 * 100 + 0; }

extern "C" int gmf_set_device(int device) {
    return gmf::cuda_status(cudaSetDevice(device));
}
