// capi.cu — status strings, device check and version of the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>

#include "host_util.h"

namespace {
std::atomic<uint64_t> g_wait_limit_ns{0};      // 0: the default, wrs::kWaitLimitNs
std::atomic<uint32_t> g_hold{0xffffffffu};     // ~0u: no look-back block is held
}  // namespace

namespace wrs {
WaitCfg current_wait_cfg() {
    WaitCfg c;
    const uint64_t l = g_wait_limit_ns.load(std::memory_order_relaxed);
    c.limit_ns = l ? l : kWaitLimitNs;
    c.hold = g_hold.load(std::memory_order_relaxed);
    c.pad = 0;
    return c;
}
}  // namespace wrs

extern "C" wrs_status wrs_set_device_wait_limit(uint64_t limit_ns) {
    if (limit_ns > 60ull * 1000000000ull) return WRS_ERR_INVALID_ARGUMENT;
    g_wait_limit_ns.store(limit_ns, std::memory_order_relaxed);
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_debug_hold_lookback(int64_t block) {
    if (block < -1 || block >= 0xffffffffll) return WRS_ERR_INVALID_ARGUMENT;
    g_hold.store(block < 0 ? 0xffffffffu : (uint32_t)block, std::memory_order_relaxed);
    return WRS_SUCCESS;
}

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

// The reference's table format (TableStorage, construction/aliasTable/TableStorage.cuh:6-128,
// structure-of-arrays form): per row an absolute FP64 weight in [0, W/N] and an int alias, so
// code written against the reference (AliasTable::verifyTableCorrectness, AliasTable.cu:24-65;
// doSample, sampling/aliasTable/SamplerGpuBasic.cu:28-69) can consume a table built here.
namespace {
__global__ void export_reference_kernel(const uint2* __restrict__ table, uint64_t n, double W_N,
                                        double* __restrict__ weight, int32_t* __restrict__ alias) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 r = table[i];
        weight[i] = (double)__uint_as_float(r.x) * W_N;
        alias[i] = (int32_t)r.y;
    }
}
}  // namespace

extern "C" wrs_status wrs_export_reference_table(const wrs_alias_row* d_table, int64_t n, double W, double* d_weight,
                                                 int32_t* d_alias, void* stream) {
    if (!d_table || !d_weight || !d_alias || n < 1 || n > 0x7fffffffll || !(W > 0.0)) return WRS_ERR_INVALID_ARGUMENT;
    const uint64_t blocks = std::min<uint64_t>(((uint64_t)n + 255) / 256, 148ull * 32);
    export_reference_kernel<<<(uint32_t)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const uint2*>(d_table), (uint64_t)n, W / (double)n, d_weight, d_alias);
    return wrs::launch_status();
}
