// static_scratch.cu — an alias build for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocating routine) at the point where they
// need a table: code running under an allocator that forbids it, plugins that must not
// touch the host process's memory pools, or paths that may not block on an allocation.
// wrs_alias_build_f32_static_scratch builds tables of up to kStaticMaxItems items with
// its scratch in a fixed device array of kStaticScratchBytes (8 MiB) that lives in this
// library: every GPU that loads the library holds that array until the process exits. The
// driver reserves it when it loads this library's device code on a device, which with lazy
// module loading (the CUDA default) is the first call of any entry point on that device.
// The caller still passes the weights, the table and the optional W output.
//
// The array's name is only a host-side stand-in in host code, so its device address is
// looked up with cudaGetSymbolAddress, with the device current, at the first call on each
// device (make that call before any stream capture). The address is kept per device and
// per CUDA context: after a device reset (a new primary context) the next call looks it up
// again. All calls on a device share the one array: calls that overlap on the GPU race and
// corrupt each other's results, so serialise them (one stream, or events). The build itself
// clears what must start at zero (the scratch header) on every call; the header's status
// word then keeps the last call's device-side status until the next call on that device
// (wrs_static_scratch_status reads it).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "host_util.h"

namespace {

constexpr int64_t kStaticMaxItems = (int64_t)1 << 18;  // 262,144 items
constexpr size_t kStaticScratchBytes = (size_t)8 << 20;  // 8 MiB (>= the build's need at the limit, any tile size)

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

struct DeviceSlot {
    CUcontext ctx = nullptr;  // the context the address belongs to
    void* ptr = nullptr;      // device address of g_static_scratch in that context
};

std::mutex g_mu;
std::vector<DeviceSlot> g_slots;  // per device ordinal
CtxGetCurrentFn g_ctx_get_current = nullptr;
bool g_ctx_fn_looked_up = false;

// The current CUDA context, through the driver entry point the runtime hands out (this
// library links only the CUDA runtime). nullptr when the driver does not provide it.
CUcontext current_context() {
    if (!g_ctx_fn_looked_up) {
        g_ctx_fn_looked_up = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    CUcontext c = nullptr;
    if (g_ctx_get_current == nullptr || g_ctx_get_current(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

wrs_status static_scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WRS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if ((int)g_slots.size() <= dev) g_slots.resize(dev + 1);
    DeviceSlot& s = g_slots[dev];
    const CUcontext ctx = current_context();
    if (s.ptr == nullptr || ctx == nullptr || ctx != s.ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr) return WRS_ERR_CUDA;
        s.ptr = p;
        s.ctx = ctx;
    }
    *out = s.ptr;
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

extern "C" wrs_status wrs_static_scratch_status(void* stream) {
    void* scratch = nullptr;
    const wrs_status st = static_scratch_address(&scratch);
    if (st != WRS_SUCCESS) return st;
    return wrs_scratch_status(scratch, stream);
}
