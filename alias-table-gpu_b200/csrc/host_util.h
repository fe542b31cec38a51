// host_util.h — host helpers shared by the C ABI translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <utility>

#include "wrs.h"
#include "wrs_common.cuh"

namespace wrs {

// The wait limits of launches made now (wrs_set_device_wait_limit, wrs_debug_hold_lookback).
WaitCfg current_wait_cfg();

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct DeviceInfo {
    int sm_count;
    int major;
    int minor;
    size_t smem_optin;
    int wsum_blocks_per_sm;  // resident CTAs of the weight-total kernel per SM
};

// Cached per device ordinal.
DeviceInfo device_info();

inline wrs_status cuda_status(cudaError_t e) { return e == cudaSuccess ? WRS_SUCCESS : WRS_ERR_CUDA; }

// Launch-error check after a kernel launch.
inline wrs_status launch_status() { return cuda_status(cudaGetLastError()); }

// A launch with programmatic stream serialisation (see pdl_enter): the kernel may be scheduled
// before the previous kernel on `stream` has completed, and waits for it on the device.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Synchronise `stream` and read a device status word.
wrs_status read_device_status(const uint32_t* d_status, cudaStream_t stream);

// Simple linear carve of a scratch buffer.
struct Carver {
    unsigned char* base;
    size_t off;
    explicit Carver(void* p) : base(static_cast<unsigned char*>(p)), off(0) {}
    template <typename T>
    T* take(size_t count, size_t align = 256) {
        off = align_up(off, align);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
};

constexpr int kWsumBlock = 256;
constexpr uint32_t kWsumMaxGrid = 2048;
uint32_t wsum_grid(uint64_t n);

}  // namespace wrs
