// autotune.cu — launch shapes of the single-table build and of the sectioned sampler, chosen by
// timing on the device and kept per (GPU, table-size bucket) in a JSON cache.
//
// The reference fixes its launch shapes at compile time (AliasTableSplitGpu.cuh:60-94) and
// picks its split count p from n by a fixed rule (AliasTableSplitGpu.cu:53-75), and its
// sectioned samplers take the section size as a constructor argument
// (SamplerGpuSectioned.cu:7-9). Here wrs_autotune_build times the split build at every tile size
// and wrs_autotune_sections times the sectioned sampler at a range of section sizes on the
// caller's own table; each result is recorded under the current device's name and
// ceil(log2 n), wrs_autotune_lookup returns it, and the cache is saved to / loaded from a JSON
// file:
//   {"entries": [{"gpu": "NVIDIA B200", "log2n": 26, "tile_items": 2048, "section_items": 16384}]}
// (a value of 0 means not tuned).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "host_util.h"

namespace {

struct Entry {
    uint32_t tile_items = 0;
    uint32_t section_items = 0;
};

std::mutex g_mu;
std::map<std::pair<std::string, int>, Entry> g_cache;

int log2_bucket(int64_t n) {
    int b = 0;
    while (b < 62 && ((int64_t)1 << b) < n) ++b;
    return b;
}

wrs_status device_name(std::string* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return WRS_ERR_CUDA;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return WRS_ERR_CUDA;
    *out = p.name;
    return WRS_SUCCESS;
}

// Median-free timing: the best of `reps` runs after one warm-up run.
template <typename F>
wrs_status time_best(F&& run, cudaStream_t stream, int reps, float* best_ms) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return WRS_ERR_CUDA;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return WRS_ERR_CUDA;
    }
    wrs_status st = run();
    float best = 1e30f;
    for (int r = 0; st == WRS_SUCCESS && r < reps; ++r) {
        cudaEventRecord(e0, stream);
        st = run();
        cudaEventRecord(e1, stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = WRS_ERR_CUDA;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *best_ms = best;
    return st;
}

// JSON of the flat form written below: finds `"key": value` after `from`.
bool json_field(const std::string& s, size_t from, size_t to, const char* key, std::string* val) {
    const std::string k = std::string("\"") + key + "\"";
    size_t p = s.find(k, from);
    if (p == std::string::npos || p >= to) return false;
    p = s.find(':', p + k.size());
    if (p == std::string::npos || p >= to) return false;
    ++p;
    while (p < to && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) ++p;
    if (p < to && s[p] == '"') {
        const size_t q = s.find('"', p + 1);
        if (q == std::string::npos || q > to) return false;
        *val = s.substr(p + 1, q - p - 1);
        return true;
    }
    size_t q = p;
    while (q < to && (isdigit((unsigned char)s[q]) || s[q] == '-')) ++q;
    if (q == p) return false;
    *val = s.substr(p, q - p);
    return true;
}

}  // namespace

extern "C" wrs_status wrs_autotune_build(const float* d_w, int64_t n, wrs_alias_row* d_table, void* d_scratch,
                                         size_t scratch_bytes, wrs_build_opts* opts, void* stream_) {
    if (!d_w || !d_table || !d_scratch || !opts || n < 1) return WRS_ERR_INVALID_ARGUMENT;
    if (opts->method != WRS_METHOD_SPLIT || opts->precision != WRS_PRECISION_MIXED) return WRS_ERR_INVALID_ARGUMENT;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    static const uint32_t kTiles[] = {1024, 2048, 4096};
    float best_ms = 1e30f;
    uint32_t best = 0;
    for (uint32_t t : kTiles) {
        wrs_build_opts o = *opts;
        o.tile_items = t;
        o.flags = 0;
        if (wrs_alias_build_scratch_bytes(n, &o) > scratch_bytes) continue;
        float ms = 0.0f;
        wrs_status st = time_best(
            [&]() { return wrs_alias_build_f32(d_w, n, &o, d_table, nullptr, d_scratch, scratch_bytes, stream); },
            stream, 3, &ms);
        if (st == WRS_SUCCESS) st = wrs_scratch_status(d_scratch, stream);
        if (st != WRS_SUCCESS) return st;
        if (ms < best_ms) {
            best_ms = ms;
            best = t;
        }
    }
    if (best == 0) return WRS_ERR_SCRATCH_TOO_SMALL;
    opts->tile_items = best;
    std::string gpu;
    if (device_name(&gpu) == WRS_SUCCESS) {
        std::lock_guard<std::mutex> lock(g_mu);
        g_cache[{gpu, log2_bucket(n)}].tile_items = best;
    }
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_autotune_sections(const wrs_alias_row* d_table, int64_t n, uint64_t num_samples,
                                            uint32_t* d_out, uint32_t* section_items, void* stream_) {
    if (!d_table || !d_out || !section_items || n < 2 || num_samples == 0) return WRS_ERR_INVALID_ARGUMENT;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    float best_ms = 1e30f;
    uint32_t best = 0;
    for (uint32_t S = 512; S <= 65536; S *= 2) {
        if (S > 2 * (uint64_t)n && best != 0) break;  // one section already holds the table
        wrs_sample_opts o{};
        o.mode = WRS_SAMPLE_SECTIONED;
        o.section_items = S;
        float ms = 0.0f;
        const wrs_status st = time_best(
            [&]() { return wrs_alias_sample(d_table, n, num_samples, 1, 0, &o, d_out, nullptr, stream); }, stream, 3,
            &ms);
        if (st != WRS_SUCCESS) return st;
        if (ms < best_ms) {
            best_ms = ms;
            best = S;
        }
    }
    *section_items = best;
    std::string gpu;
    if (device_name(&gpu) == WRS_SUCCESS) {
        std::lock_guard<std::mutex> lock(g_mu);
        g_cache[{gpu, log2_bucket(n)}].section_items = best;
    }
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_autotune_lookup(int64_t n, uint32_t* tile_items, uint32_t* section_items) {
    if (n < 1) return WRS_ERR_INVALID_ARGUMENT;
    std::string gpu;
    const wrs_status st = device_name(&gpu);
    if (st != WRS_SUCCESS) return st;
    std::lock_guard<std::mutex> lock(g_mu);
    const auto it = g_cache.find({gpu, log2_bucket(n)});
    const Entry e = it == g_cache.end() ? Entry{} : it->second;
    if (tile_items) *tile_items = e.tile_items;
    if (section_items) *section_items = e.section_items;
    return it == g_cache.end() ? WRS_ERR_INVALID_ARGUMENT : WRS_SUCCESS;
}

extern "C" wrs_status wrs_autotune_cache_save(const char* path) {
    if (!path) return WRS_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "w");
    if (!f) return WRS_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_mu);
    std::fprintf(f, "{\"entries\": [");
    bool first = true;
    for (const auto& kv : g_cache) {
        std::string gpu;
        for (char c : kv.first.first)
            if (c != '"' && c != '\\') gpu += c;
        std::fprintf(f, "%s\n  {\"gpu\": \"%s\", \"log2n\": %d, \"tile_items\": %u, \"section_items\": %u}",
                     first ? "" : ",", gpu.c_str(), kv.first.second, kv.second.tile_items, kv.second.section_items);
        first = false;
    }
    std::fprintf(f, "\n]}\n");
    return std::fclose(f) == 0 ? WRS_SUCCESS : WRS_ERR_INVALID_ARGUMENT;
}

extern "C" wrs_status wrs_autotune_cache_load(const char* path) {
    if (!path) return WRS_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "r");
    if (!f) return WRS_ERR_INVALID_ARGUMENT;
    std::string s;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, k);
    std::fclose(f);
    if (s.find("\"entries\"") == std::string::npos) return WRS_ERR_INVALID_ARGUMENT;
    std::map<std::pair<std::string, int>, Entry> loaded;
    size_t p = 0;
    while ((p = s.find('{', p + 1)) != std::string::npos) {
        const size_t q = s.find('}', p);
        if (q == std::string::npos) return WRS_ERR_INVALID_ARGUMENT;
        std::string gpu, l, t, sec;
        if (!json_field(s, p, q, "gpu", &gpu) || !json_field(s, p, q, "log2n", &l) ||
            !json_field(s, p, q, "tile_items", &t) || !json_field(s, p, q, "section_items", &sec))
            return WRS_ERR_INVALID_ARGUMENT;
        Entry e;
        e.tile_items = (uint32_t)std::strtoul(t.c_str(), nullptr, 10);
        e.section_items = (uint32_t)std::strtoul(sec.c_str(), nullptr, 10);
        loaded[{gpu, (int)std::strtol(l.c_str(), nullptr, 10)}] = e;
        p = q;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    for (const auto& kv : loaded) g_cache[kv.first] = kv.second;
    return WRS_SUCCESS;
}
