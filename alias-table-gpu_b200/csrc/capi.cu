// capi.cu — status strings, device check and version of the C ABI.
#include <cuda_runtime.h>

#include "host_util.h"

extern "C" const char* wrs_status_string(wrs_status s) {
    switch (s) {
        case WRS_SUCCESS: return "success";
        case WRS_ERR_INVALID_ARGUMENT: return "invalid argument";
        case WRS_ERR_INVALID_WEIGHT: return "a weight is NaN, negative or infinite";
        case WRS_ERR_ZERO_TOTAL: return "all weights are zero";
        case WRS_ERR_SCRATCH_TOO_SMALL: return "scratch buffer too small";
        case WRS_ERR_CUDA: return "CUDA runtime error";
        case WRS_ERR_DEVICE_TIMEOUT: return "bounded device wait timed out";
        case WRS_ERR_TOO_MANY_TRIES: return "rejection sampling exhausted max_tries";
        case WRS_ERR_UNSUPPORTED: return "unsupported device or option";
        case WRS_ERR_CAPACITY: return "output buffer too small";
        default: return "unknown status";
    }
}

extern "C" wrs_status wrs_check_device(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WRS_ERR_CUDA;
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return WRS_ERR_CUDA;
    return major == 10 ? WRS_SUCCESS : WRS_ERR_UNSUPPORTED;
}

extern "C" int wrs_version(void) { return WRS_VERSION_MAJOR * 100 + WRS_VERSION_MINOR; }
