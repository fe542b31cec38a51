// sample.cu — C ABI of the alias samplers and of rejection sampling.
//
// wrs_alias_sample        <- SamplerGpuBasic / SamplerGpuSectioned[Shared]::executeBenchmarkSampling
//                            (sampling/aliasTable/SamplerGpuBasic.cu:109-133,
//                             SamplerGpuSectioned.cu:138-166, SamplerGpuSectionedShared.cu:90-111)
// wrs_rejection_build_f32 <- RejectionSampling::build + fillA
//                            (construction/rejectionSampling/RejectionSampling.cu:35-56)
// wrs_rejection_sample    <- SamplerRejection[GiveUp]::executeBenchmarkSampling
//                            (sampling/rejectionSampling/SamplerRejection.cu:63-72)
#include <cuda_runtime.h>

#include <mutex>

#include "host_util.h"
#include "rejection_kernels.cuh"
#include "sample_kernels.cuh"

using namespace wrs;

namespace {
constexpr int64_t kMaxItems = (int64_t)0x7fffffff - 8192;
constexpr uint32_t kDefaultSection = 65536;
constexpr size_t kStageMaxBytes = 96 * 1024;  // sections up to this size are staged in smem
constexpr uint32_t kSectLargeRows = 32768;    // L2-form sections from this size draw 4 positions a step

inline uint32_t seed_k0(uint64_t seed) { return (uint32_t)seed; }
inline uint32_t seed_k1(uint64_t seed) { return (uint32_t)(seed >> 32); }
}  // namespace

extern "C" wrs_status wrs_alias_sample(const wrs_alias_row* d_table, int64_t n, uint64_t num_samples, uint64_t seed,
                                       uint64_t counter_base, const wrs_sample_opts* opts, uint32_t* d_out,
                                       uint64_t* d_section_counts, void* stream_) {
    if (!d_table || n < 1 || n > kMaxItems || (num_samples > 0 && !d_out)) return WRS_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)d_table & 7u) != 0 || ((uintptr_t)d_out & 3u) != 0) return WRS_ERR_INVALID_ARGUMENT;
    const uint32_t mode = opts ? opts->mode : WRS_SAMPLE_PLAIN;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const DeviceInfo dev = device_info();
    const uint2* table = reinterpret_cast<const uint2*>(d_table);
    if (mode == WRS_SAMPLE_PLAIN || mode == WRS_SAMPLE_HISTOGRAM || mode == WRS_SAMPLE_DISCARD) {
        if (num_samples == 0) return WRS_SUCCESS;
        const uint64_t noct = (num_samples + 7) / 8;
        const uint32_t threads = (opts && opts->threads) ? opts->threads : 256u;
        if (threads != 256u) return WRS_ERR_INVALID_ARGUMENT;
        uint64_t grid = (noct + threads - 1) / threads;
        const uint64_t cap = (uint64_t)dev.sm_count * 16;
        if (grid > cap) grid = cap;
        if (mode == WRS_SAMPLE_HISTOGRAM)
            sample_plain_kernel<1><<<(uint32_t)grid, threads, 0, stream>>>(
                table, (uint32_t)n, num_samples, seed_k0(seed), seed_k1(seed), counter_base, d_out);
        else if (mode == WRS_SAMPLE_DISCARD)
            sample_plain_kernel<2><<<(uint32_t)grid, threads, 0, stream>>>(
                table, (uint32_t)n, num_samples, seed_k0(seed), seed_k1(seed), counter_base, d_out);
        else
            sample_plain_kernel<0><<<(uint32_t)grid, threads, 0, stream>>>(
                table, (uint32_t)n, num_samples, seed_k0(seed), seed_k1(seed), counter_base, d_out);
    } else if (mode == WRS_SAMPLE_SECTIONED) {
        const uint32_t S = (opts && opts->section_items) ? opts->section_items : kDefaultSection;
        if (S < 2 || (S & 1u)) return WRS_ERR_INVALID_ARGUMENT;
        const uint64_t K = ((uint64_t)n + S - 1) / S;
        const size_t sec_bytes = (size_t)S * sizeof(uint2);
        const bool stage = sec_bytes <= kStageMaxBytes && ((uintptr_t)d_table & 15u) == 0;
        const uint32_t threads = kSectThreads;
        if (stage) {
            const int per_sm = (int)(200 * 1024 / sec_bytes) < 4 ? (int)(200 * 1024 / sec_bytes) : 4;
            uint64_t grid = (uint64_t)dev.sm_count * (per_sm > 0 ? per_sm : 1);
            if (grid > K) grid = K;
            cudaError_t e = cudaFuncSetAttribute(sample_sectioned_kernel<true, 8>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sec_bytes);
            if (e != cudaSuccess) return WRS_ERR_CUDA;
            sample_sectioned_kernel<true, 8><<<(uint32_t)grid, threads, sec_bytes, stream>>>(
                table, (uint32_t)n, num_samples, S, (uint32_t)K, seed_k0(seed), seed_k1(seed), counter_base, d_out,
                d_section_counts);
        } else {
            // one CTA per SM: the sections in flight (SMs x section bytes) stay L2-resident
            uint64_t grid = (uint64_t)dev.sm_count;
            if (grid > K) grid = K;
            if (S >= kSectLargeRows)
                sample_sectioned_kernel<false, 4><<<(uint32_t)grid, threads, 0, stream>>>(
                    table, (uint32_t)n, num_samples, S, (uint32_t)K, seed_k0(seed), seed_k1(seed), counter_base,
                    d_out, d_section_counts);
            else
                sample_sectioned_kernel<false, 8><<<(uint32_t)grid, threads, 0, stream>>>(
                    table, (uint32_t)n, num_samples, S, (uint32_t)K, seed_k0(seed), seed_k1(seed), counter_base,
                    d_out, d_section_counts);
        }
    } else {
        return WRS_ERR_INVALID_ARGUMENT;
    }
    const wrs_status st = launch_status();
    if (st != WRS_SUCCESS) return st;
    if (opts && (opts->flags & WRS_FLAG_SYNC)) return cuda_status(cudaStreamSynchronize(stream));
    return WRS_SUCCESS;
}

// ---------------------------------------------------------------- sampling into host memory
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_copy_mu;
cudaStream_t g_copy_stream[kMaxDevices] = {};

// The library's device-to-host copy stream of the current device (created on first use).
wrs_status copy_stream(cudaStream_t* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return WRS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_copy_mu);
    if (!g_copy_stream[dev] && cudaStreamCreateWithFlags(&g_copy_stream[dev], cudaStreamNonBlocking) != cudaSuccess) {
        g_copy_stream[dev] = nullptr;
        return WRS_ERR_CUDA;
    }
    *out = g_copy_stream[dev];
    return WRS_SUCCESS;
}
}  // namespace

extern "C" wrs_status wrs_alias_sample_to_host(const wrs_alias_row* d_table, int64_t n, uint64_t num_samples,
                                               uint64_t seed, uint64_t counter_base, uint64_t chunk_samples,
                                               uint32_t* d_out, uint32_t* h_out, void* stream_) {
    if (!d_table || n < 1 || n > kMaxItems || (num_samples > 0 && (!d_out || !h_out))) return WRS_ERR_INVALID_ARGUMENT;
    if (num_samples == 0) return WRS_SUCCESS;
    uint64_t chunk = chunk_samples ? chunk_samples : (1ull << 25);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    cudaStream_t copy = nullptr;
    wrs_status st = copy_stream(&copy);
    if (st != WRS_SUCCESS) return st;
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return WRS_ERR_CUDA;
    for (uint64_t s0 = 0; s0 < num_samples && st == WRS_SUCCESS; s0 += chunk) {
        const uint64_t c = num_samples - s0 < chunk ? num_samples - s0 : chunk;
        st = wrs_alias_sample(d_table, n, c, seed, counter_base + s0, nullptr, d_out + s0, nullptr, stream_);
        if (st != WRS_SUCCESS) break;
        // the copy stream takes the chunk once it is written (a wait binds the latest record)
        if (cudaEventRecord(ev, stream) != cudaSuccess || cudaStreamWaitEvent(copy, ev, 0) != cudaSuccess ||
            cudaMemcpyAsync(h_out + s0, d_out + s0, c * sizeof(uint32_t), cudaMemcpyDeviceToHost, copy) !=
                cudaSuccess)
            st = WRS_ERR_CUDA;
    }
    // later work on `stream` (and a later call reusing d_out) waits for every copy
    if (cudaEventRecord(ev, copy) != cudaSuccess || cudaStreamWaitEvent(stream, ev, 0) != cudaSuccess)
        st = st == WRS_SUCCESS ? WRS_ERR_CUDA : st;
    cudaEventDestroy(ev);
    return st;
}

// ---------------------------------------------------------------- rejection
namespace {
struct RejLayout {
    BuildHeader* hdr;
    double2* partials;
    uint64_t* tile_words;
    RejBigEntry* big;
    uint64_t big_capacity;
    uint32_t* huge;
    uint64_t huge_capacity;
    size_t bytes;
};
constexpr int kRejIpt = 8;
RejLayout carve_rej(void* scratch, uint64_t n) {
    const uint64_t T = (uint64_t)kBuildThreads * kRejIpt;
    const uint64_t nt = (n + T - 1) / T;
    Carver c(scratch);
    RejLayout L;
    L.hdr = c.take<BuildHeader>(1);
    L.partials = c.take<double2>(kWsumMaxGrid);
    L.tile_words = c.take<uint64_t>(nt);
    L.big_capacity = (2 * n) / kRejBig + 16;
    L.big = c.take<RejBigEntry>(L.big_capacity);
    L.huge_capacity = (2 * n) / kRejHugeSlots + 16;
    L.huge = c.take<uint32_t>(L.huge_capacity);
    L.bytes = c.off;
    return L;
}
}  // namespace

extern "C" size_t wrs_rejection_build_scratch_bytes(int64_t n) {
    if (n < 1) return 0;
    return carve_rej(nullptr, (uint64_t)n).bytes;
}

extern "C" wrs_status wrs_rejection_build_f32(const float* d_w, int64_t n, uint32_t* d_A, uint64_t a_capacity,
                                              float* d_frac, uint64_t* d_A_size, double* d_W, void* d_scratch,
                                              size_t scratch_bytes, uint32_t flags, void* stream_) {
    if (!d_w || !d_A || !d_frac || !d_scratch || n < 1 || n > kMaxItems / 2) return WRS_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < carve_rej(nullptr, (uint64_t)n).bytes) return WRS_ERR_SCRATCH_TOO_SMALL;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const RejLayout L = carve_rej(d_scratch, (uint64_t)n);
    const uint64_t T = (uint64_t)kBuildThreads * kRejIpt;
    const uint64_t nt = ((uint64_t)n + T - 1) / T;
    if (cudaMemsetAsync(L.hdr, 0, sizeof(BuildHeader), stream) != cudaSuccess) return WRS_ERR_CUDA;
    wsum_kernel<kWsumBlock><<<wsum_grid((uint64_t)n), kWsumBlock, 0, stream>>>(
        d_w, (uint64_t)n, L.hdr, L.partials, reinterpret_cast<uint32_t*>(L.tile_words), 2 * nt, d_W);
    // the kernels after wsum are programmatic dependents (launch_pdl)
    if (launch_pdl(rejection_tile_kernel<kRejIpt>, dim3((uint32_t)nt), dim3(kBuildThreads), 0, stream, d_w,
                   (uint64_t)n, L.hdr, L.tile_words, (uint32_t)nt, d_A, a_capacity, d_frac, L.big, L.big_capacity,
                   d_A_size, current_wait_cfg()) != cudaSuccess)
        return WRS_ERR_CUDA;
    const DeviceInfo dev = device_info();
    if (launch_pdl(rejection_big_kernel, dim3((uint32_t)dev.sm_count * 4), dim3(256), 0, stream, L.hdr, L.big,
                   L.big_capacity, d_A, a_capacity, L.huge, L.huge_capacity) != cudaSuccess)
        return WRS_ERR_CUDA;
    if (launch_pdl(rejection_huge_kernel, dim3((uint32_t)dev.sm_count * 4), dim3(256), 0, stream, L.hdr, L.big,
                   L.huge, L.huge_capacity, d_A, a_capacity) != cudaSuccess)
        return WRS_ERR_CUDA;
    const wrs_status st = launch_status();
    if (st != WRS_SUCCESS) return st;
    if (flags & WRS_FLAG_SYNC) return read_device_status(&L.hdr->status, stream);
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_rejection_sample(const uint32_t* d_A, const uint64_t* d_A_size, const float* d_frac,
                                           int64_t n, uint64_t num_samples, uint64_t seed, uint64_t counter_base,
                                           uint32_t max_tries, uint32_t* d_out, uint32_t* d_status, uint32_t flags,
                                           void* stream_) {
    if (!d_A || !d_A_size || !d_frac || n < 1 || (num_samples > 0 && !d_out)) return WRS_ERR_INVALID_ARGUMENT;
    if (num_samples == 0) return WRS_SUCCESS;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const DeviceInfo dev = device_info();
    const uint32_t tries = max_tries ? max_tries : 64u;
    uint64_t grid = ((num_samples + kRejJ - 1) / kRejJ + 255) / 256;
    const uint64_t cap = (uint64_t)dev.sm_count * 8;
    if (grid > cap) grid = cap;
    rejection_sample_kernel<<<(uint32_t)grid, 256, 0, stream>>>(d_A, d_A_size, d_frac, num_samples, seed_k0(seed),
                                                               seed_k1(seed), counter_base, tries, d_out, d_status);
    const wrs_status st = launch_status();
    if (st != WRS_SUCCESS) return st;
    if (flags & WRS_FLAG_SYNC) {
        if (d_status) return read_device_status(d_status, stream);
        return cuda_status(cudaStreamSynchronize(stream));
    }
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_rejection_pack(const uint32_t* d_A, const uint64_t* d_A_size, const float* d_frac,
                                         int64_t n, uint64_t a_capacity, uint64_t* d_slots, void* stream_) {
    if (!d_A || !d_A_size || !d_frac || !d_slots || n < 1 || n > kMaxItems) return WRS_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)d_slots & 7u) != 0) return WRS_ERR_INVALID_ARGUMENT;
    if (a_capacity == 0) return WRS_SUCCESS;
    const DeviceInfo dev = device_info();
    uint64_t grid = (a_capacity + 255) / 256;
    const uint64_t cap = (uint64_t)dev.sm_count * 8;
    if (grid > cap) grid = cap;
    rejection_pack_kernel<<<(uint32_t)grid, 256, 0, static_cast<cudaStream_t>(stream_)>>>(
        d_A, d_A_size, d_frac, (uint32_t)n, a_capacity, reinterpret_cast<uint2*>(d_slots));
    return launch_status();
}

extern "C" wrs_status wrs_rejection_sample_packed(const uint64_t* d_slots, uint64_t slot_capacity,
                                                  const uint64_t* d_A_size, int64_t n,
                                                  uint64_t num_samples, uint64_t seed, uint64_t counter_base,
                                                  uint32_t max_tries, uint32_t* d_out, uint32_t* d_status,
                                                  uint32_t flags, void* stream_) {
    if (!d_slots || !d_A_size || n < 1 || (num_samples > 0 && !d_out)) return WRS_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)d_slots & 7u) != 0) return WRS_ERR_INVALID_ARGUMENT;
    if (num_samples == 0) return WRS_SUCCESS;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const DeviceInfo dev = device_info();
    const uint32_t tries = max_tries ? max_tries : 64u;
    const uint64_t per = (uint64_t)kRejPackedR * 256;  // samples per CTA and chunk
    uint64_t grid = (num_samples + per - 1) / per;
    const uint64_t cap = (uint64_t)dev.sm_count * 8;
    if (grid > cap) grid = cap;
    rejection_sample_packed_kernel<<<(uint32_t)grid, 256, 0, stream>>>(
        reinterpret_cast<const uint2*>(d_slots), slot_capacity, d_A_size, num_samples, seed_k0(seed), seed_k1(seed), counter_base,
        tries, d_out, d_status);
    const wrs_status st = launch_status();
    if (st != WRS_SUCCESS) return st;
    if (flags & WRS_FLAG_SYNC) {
        if (d_status) return read_device_status(d_status, stream);
        return cuda_status(cudaStreamSynchronize(stream));
    }
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_random_gather_probe(const wrs_alias_row* d_table, int64_t n, uint64_t num_gathers,
                                              uint64_t seed, uint32_t* d_sink, void* stream_) {
    if (!d_table || !d_sink || n < 1 || n > kMaxItems) return WRS_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)d_table & 7u) != 0 || ((uintptr_t)d_sink & 3u) != 0) return WRS_ERR_INVALID_ARGUMENT;
    if (num_gathers == 0) return WRS_SUCCESS;
    const DeviceInfo dev = device_info();
    uint64_t grid = ((num_gathers + 7) / 8 + 255) / 256;
    const uint64_t cap = (uint64_t)dev.sm_count * 16;
    if (grid > cap) grid = cap;
    gather_probe_kernel<<<(uint32_t)grid, 256, 0, static_cast<cudaStream_t>(stream_)>>>(
        reinterpret_cast<const uint2*>(d_table), (uint32_t)n, num_gathers, seed, d_sink);
    return launch_status();
}
