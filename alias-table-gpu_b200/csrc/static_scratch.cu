// static_scratch.cu — an alias build for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocating routine) at the point where they
// need a table: code running under an allocator that forbids it, plugins that must not
// touch the host process's memory pools, or paths that may not block on an allocation.
// wrs_alias_build_f32_static_scratch builds tables of up to kStaticMaxItems items with
// its scratch in a fixed device array of kStaticScratchBytes (8 MiB) that lives in this
// library: every GPU that loads the library holds that array until the process exits.
// The caller still passes the weights, the table and the optional W output.
//
// The array's name is only a host-side stand-in in host code, so its device address is
// looked up with cudaGetSymbolAddress, once per device, with that device current; the
// first call on each device does this set-up (make it before any stream capture).
// All calls on a device share the one array: calls that overlap on the GPU race and
// corrupt each other's results, so serialise them (one stream, or events). The build
// itself clears what must start at zero (the scratch header) on every call.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "host_util.h"

namespace {

constexpr int64_t kStaticMaxItems = (int64_t)1 << 18;  // 262,144 items
constexpr size_t kStaticScratchBytes = (size_t)8 << 20;  // 8 MiB (>= the build's need at the limit, any tile size)

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_mu;
std::vector<void*> g_dev_ptr;  // per device ordinal: device address of g_static_scratch

wrs_status static_scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WRS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if ((int)g_dev_ptr.size() <= dev) g_dev_ptr.resize(dev + 1, nullptr);
    if (g_dev_ptr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr) return WRS_ERR_CUDA;
        g_dev_ptr[dev] = p;
    }
    *out = g_dev_ptr[dev];
    return WRS_SUCCESS;
}

}  // namespace

extern "C" wrs_status wrs_alias_build_f32_static_scratch(const float* d_w, int64_t n, const wrs_build_opts* opts,
                                                         wrs_alias_row* d_table, double* d_W, void* stream) {
    if (n < 1 || n > kStaticMaxItems) return WRS_ERR_INVALID_ARGUMENT;
    const size_t need = wrs_alias_build_scratch_bytes(n, opts);
    if (need == 0 || need > kStaticScratchBytes) return WRS_ERR_INVALID_ARGUMENT;
    void* scratch = nullptr;
    const wrs_status st = static_scratch_address(&scratch);
    if (st != WRS_SUCCESS) return st;
    return wrs_alias_build_f32(d_w, n, opts, d_table, d_W, scratch, kStaticScratchBytes, stream);
}
