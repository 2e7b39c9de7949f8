// api.cu -- status strings and version of the C ABI.
#include "common.cuh"

extern "C" const char* aerial_error_string(int status) {
    switch (status) {
        case AERIAL_OK: return "ok";
        case AERIAL_ERR_INVALID_ARG: return "invalid argument (null pointer, size out of range or misaligned buffer)";
        case AERIAL_ERR_UNSUPPORTED: return "shape or option outside the supported envelope";
        case AERIAL_ERR_NO_DEVICE: return "no usable sm_100 device";
        case AERIAL_ERR_BUDGET: return "request exceeds the device-memory budget";
        case AERIAL_ERR_QUEUE_FULL: return "submission queue full";
        case AERIAL_ERR_TIMEOUT: return "bounded wait ran out";
        case AERIAL_ERR_NOT_FOUND: return "unknown cell or request";
        case AERIAL_ERR_SCRATCH_LIMIT: return "request needs more than the library's static scratch (16 MiB)";
        default:
            if (status > 0 && status < 1000) return cudaGetErrorString((cudaError_t)status);
            return "unknown status";
    }
}

extern "C" int aerial_version(void) { return 10000; /* 1.0.0 */ }

namespace aeq {
int prepare_fused_kernels();
int prepare_srs_kernels();
int prepare_plain_kernels();
}

// Load the library's kernels on the current device (see the header).
extern "C" int aerial_prepare(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return AERIAL_ERR_NO_DEVICE;
    int s = aeq::prepare_fused_kernels();
    if (!s) s = aeq::prepare_srs_kernels();
    if (!s) s = aeq::prepare_plain_kernels();
    return s;
}
