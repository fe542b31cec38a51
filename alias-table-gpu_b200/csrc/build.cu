// build.cu — C ABI of the weight total and the single-table alias build.
//
// wrs_sum_f32          <- Adder::addGpuCub (utils/Adder.cu:144-157)
// wrs_alias_build_f32  <- AliasTableSplitGpu<TableStorage>::build()
//                         (construction/aliasTable/buildMethod/AliasTableSplitGpu.cu:388-468)
//
// Unlike the reference build (>= 5 blocking device-to-host copies and >= 3 cudaMalloc/cudaFree
// pairs inside build()), the whole build is stream-ordered work on caller memory: a 128-byte
// memset of the scratch header, then the wsum, scan, link and pack kernels (split method), or
// the wsum, tile_reduce, tile_prefix, psa_local and leftover passes (PSA+).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "build_kernels.cuh"
#include "psa_kernels.cuh"
#include "split_kernels.cuh"
#include "precision_kernels.cuh"
#include "host_util.h"

namespace wrs {

DeviceInfo device_info() {
    static std::mutex mu;
    static std::vector<DeviceInfo> cache;
    static std::vector<bool> have;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if ((int)cache.size() <= dev) {
        cache.resize(dev + 1);
        have.resize(dev + 1, false);
    }
    if (!have[dev]) {
        DeviceInfo d{};
        cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&d.major, cudaDevAttrComputeCapabilityMajor, dev);
        cudaDeviceGetAttribute(&d.minor, cudaDevAttrComputeCapabilityMinor, dev);
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        d.smem_optin = (size_t)optin;
        if (d.sm_count <= 0) d.sm_count = 148;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.wsum_blocks_per_sm, wsum_kernel<kWsumBlock>, kWsumBlock,
                                                          0) != cudaSuccess ||
            d.wsum_blocks_per_sm < 1)
            d.wsum_blocks_per_sm = 1;
        cache[dev] = d;
        have[dev] = true;
    }
    return cache[dev];
}

wrs_status read_device_status(const uint32_t* d_status, cudaStream_t stream) {
    uint32_t h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, d_status, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return WRS_ERR_CUDA;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return WRS_ERR_CUDA;
    return (wrs_status)h;
}

uint32_t wsum_grid(uint64_t n) {
    const DeviceInfo d = device_info();
    uint64_t g = (n + 2047) / 2048;
    // one wave: a second, partial wave of CTAs would run the tail at low occupancy
    const uint64_t cap = (uint64_t)d.sm_count * (uint64_t)d.wsum_blocks_per_sm;
    if (g > cap) g = cap;
    if (g > kWsumMaxGrid) g = kWsumMaxGrid;
    if (g < 1) g = 1;
    return (uint32_t)g;
}

namespace {

constexpr int64_t kMaxItems = (int64_t)0x7fffffff - 8192;

// Items per tile of the scan and pack passes (0 = the default: 2048, and 1024 for PSA+, whose
// local pass is faster on smaller tiles).
int64_t tile_items_for(const wrs_build_opts* opts) {
    const uint32_t t = opts ? opts->tile_items : 0u;
    switch (t) {
        case 0: return (opts && opts->method == WRS_METHOD_PSA_PLUS) ? 1024 : 2048;
        case 2048: return 2048;
        case 1024: return 1024;
        case 4096: return 4096;
        default: return -1;
    }
}

// The split method: wsum (W, class thresholds, look-back flags cleared), scan (tile sums,
// look-back prefixes over groups of tiles, tile starts, compact heavy list), link (the split
// search per tile boundary), pack_walk (the merge, walk form; it lists the tiles whose heavies
// exceed its arrays) and split_pack's chunked form over that list.
struct SplitLayout {
    BuildHeader* hdr;
    double2* partials;
    LbWord* lb;          // scan: look-back word per group of tiles
    BlockWord* blocks;   // tile_prefix: look-back record per block of tiles
    uint64_t num_groups;
    uint64_t num_blocks;
    TileVals* agg;
    TileVals* incl;
    TileStart* starts;
    uint32_t* chunk_list;
    uint32_t* heavy_item;
    uint64_t* heavy_E;
    size_t bytes;
};

SplitLayout carve_split(void* scratch, uint64_t n, uint64_t num_tiles) {
    Carver c(scratch);
    SplitLayout L;
    L.hdr = c.take<BuildHeader>(1);
    L.partials = c.take<double2>(kWsumMaxGrid);
    L.num_groups = (num_tiles + scan_group_tiles(num_tiles) - 1) / scan_group_tiles(num_tiles);
    L.num_blocks = (num_tiles + kPrefixTiles - 1) / kPrefixTiles;
    L.lb = c.take<LbWord>(L.num_groups);
    L.blocks = c.take<BlockWord>(L.num_blocks);  // right after lb: one zeroing covers both
    L.agg = c.take<TileVals>(num_tiles);
    L.incl = c.take<TileVals>(num_tiles);
    L.starts = c.take<TileStart>(num_tiles + 1);
    L.chunk_list = c.take<uint32_t>(num_tiles);
    L.heavy_item = c.take<uint32_t>(n);
    L.heavy_E = c.take<uint64_t>(n);
    L.bytes = c.off;
    return L;
}

template <int T>
struct SplitShape;
template <>
struct SplitShape<1024> {
    static constexpr int SCAN_IPT = 4, NT = 128, IPT = 8;
};
template <>
struct SplitShape<2048> {
    static constexpr int SCAN_IPT = 8, NT = 256, IPT = 8;
};
template <>
struct SplitShape<4096> {
    static constexpr int SCAN_IPT = 16, NT = 256, IPT = 16;
};

template <int T>
wrs_status launch_split(const float* d_w, uint64_t n, wrs_alias_row* d_table, double* d_W, const SplitLayout& L,
                        uint64_t num_tiles, cudaStream_t stream) {
    using S = SplitShape<T>;
    static_assert(S::NT * S::IPT == T && kScanThreads * S::SCAN_IPT == T, "tile shapes");
    const uint32_t nt = (uint32_t)num_tiles;
    if (cudaMemsetAsync(L.hdr, 0, sizeof(BuildHeader), stream) != cudaSuccess) return WRS_ERR_CUDA;
    // wsum clears the look-back words of scan and tile_prefix (adjacent in the scratch)
    const uint64_t zero_words =
        (uint64_t)(reinterpret_cast<const char*>(L.blocks + L.num_blocks) - reinterpret_cast<const char*>(L.lb)) / 4;
    wsum_kernel<kWsumBlock><<<wsum_grid(n), kWsumBlock, 0, stream>>>(d_w, n, L.hdr, L.partials,
                                                                     reinterpret_cast<uint32_t*>(L.lb), zero_words,
                                                                     d_W);
    const WaitCfg wc = current_wait_cfg();
    // the kernels after wsum are launched as programmatic dependents: each starts while its
    // predecessor's last wave runs and waits for the predecessor's completion on entry
    if (launch_pdl(scan_kernel<S::SCAN_IPT>, dim3((uint32_t)L.num_groups), dim3(kScanThreads), 0, stream, d_w, n,
                   L.hdr, L.lb, nt, L.agg, L.heavy_item, L.heavy_E, wc, scan_group_tiles(nt)) != cudaSuccess)
        return WRS_ERR_CUDA;
    if (launch_pdl(tile_prefix_kernel, dim3((uint32_t)L.num_blocks), dim3(kPrefixThreads), 0, stream, L.hdr, L.agg,
                   L.incl, L.blocks, nt, wc) != cudaSuccess)
        return WRS_ERR_CUDA;
    if (launch_pdl(link_kernel, dim3(((nt + 1) * (uint32_t)kLinkLanes + 255) / 256), dim3(256), 0, stream, L.hdr,
                   L.incl, nt, L.heavy_E, L.starts) != cudaSuccess)
        return WRS_ERR_CUDA;
    {
        const size_t smem = pack_walk_smem_bytes(T, S::IPT);
        if (cudaFuncSetAttribute(pack_walk_kernel<S::NT, S::IPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return WRS_ERR_CUDA;
        if (launch_pdl(pack_walk_kernel<S::NT, S::IPT>, dim3(nt), dim3(S::NT), smem, stream, d_w, n, L.hdr,
                       L.starts, L.heavy_item, L.heavy_E, nt, d_table, L.chunk_list) != cudaSuccess)
            return WRS_ERR_CUDA;
    }
    {
        constexpr int NT = PackShape<T>::NT, IPT = PackShape<T>::IPT;
        const size_t smem = pack_smem_bytes(T);
        if (cudaFuncSetAttribute(split_pack_kernel<NT, IPT, false, false, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return WRS_ERR_CUDA;
        const TileMap map{nullptr, nullptr, nullptr, n, nt};
        // the tiles pack_walk listed; a small grid, so that an empty list costs one short launch
        const uint32_t grid = std::min<uint32_t>(nt, (uint32_t)device_info().sm_count * 2u);
        if (launch_pdl(split_pack_kernel<NT, IPT, false, false, true>, dim3(grid), dim3(NT), smem, stream, d_w,
                       L.hdr, nullptr, L.starts, L.heavy_item, L.heavy_E, nt, d_table, map, nullptr,
                       L.chunk_list) != cudaSuccess)
            return WRS_ERR_CUDA;
    }
    return launch_status();
}

// The comparison builds in one floating-point type R (WRS_PRECISION_FP64 / _FP32): weight tile
// sums, the total W, deficit/excess tile sums, the tiles' line bases, the two lines in item
// order, and the merge.
template <typename R>
struct PrecLayout {
    BuildHeader* hdr;
    PrecTile<R>* tiles;
    PrecTile<R>* prefix;  // num_tiles + 1: the last holds the totals
    R* Lkey;
    uint32_t* Litem;
    float* Lprob;
    R* Hkey;
    uint32_t* Hitem;
    size_t bytes;
};

template <typename R>
PrecLayout<R> carve_prec(void* scratch, uint64_t n) {
    const uint64_t nt = (n + kPrecTile - 1) / kPrecTile;
    Carver c(scratch);
    PrecLayout<R> L;
    L.hdr = c.take<BuildHeader>(1);
    L.tiles = c.take<PrecTile<R>>(nt);
    L.prefix = c.take<PrecTile<R>>(nt + 1);
    L.Lkey = c.take<R>(n);
    L.Litem = c.take<uint32_t>(n);
    L.Lprob = c.take<float>(n);
    L.Hkey = c.take<R>(n);
    L.Hitem = c.take<uint32_t>(n);
    L.bytes = c.off;
    return L;
}

template <typename R>
wrs_status launch_prec(const float* d_w, uint64_t n, wrs_alias_row* d_table, double* d_W, const PrecLayout<R>& L,
                       cudaStream_t stream) {
    const uint32_t nt = (uint32_t)((n + kPrecTile - 1) / kPrecTile);
    if (cudaMemsetAsync(L.hdr, 0, sizeof(BuildHeader), stream) != cudaSuccess) return WRS_ERR_CUDA;
    prec_weight_tiles_kernel<R><<<nt, kPrecThreads, 0, stream>>>(d_w, n, L.hdr, L.tiles);
    prec_weight_total_kernel<R><<<1, kPrecScanThreads, 0, stream>>>(L.hdr, L.tiles, nt, n, d_W);
    const uint32_t lgrid = (nt + 127) / 128;
    prec_lines_kernel<R, false><<<lgrid, 128, 0, stream>>>(d_w, n, L.hdr, L.tiles, nullptr, nt, nullptr, nullptr,
                                                           nullptr, nullptr, nullptr);
    prec_line_bases_kernel<R><<<1, 32, 0, stream>>>(L.hdr, L.tiles, L.prefix, nt);
    prec_lines_kernel<R, true><<<lgrid, 128, 0, stream>>>(d_w, n, L.hdr, L.tiles, L.prefix, nt, L.Lkey, L.Litem,
                                                          L.Lprob, L.Hkey, L.Hitem);
    const uint64_t threads = (n + kPrecMergeChunk - 1) / kPrecMergeChunk;
    prec_merge_kernel<R><<<(uint32_t)((threads + 255) / 256), 256, 0, stream>>>(
        L.hdr, L.prefix + nt, L.Lkey, L.Litem, L.Lprob, L.Hkey, L.Hitem, n, d_table);
    return launch_status();
}

// PSA+: the split passes up to the tile prefixes, the local pass, and the split passes again
// over the leftovers (second header, prefix records, tile starts and heavy list).
struct PsaLayout {
    BuildHeader* hdr;  // hdr[0]: the build; hdr[1]: the leftover passes (one memset clears both)
    BuildHeader* hdr2;
    double2* partials;
    BlockWord* blocks;
    BlockWord* blocks2;
    uint64_t num_blocks;
    TileVals* agg;
    TileVals* incl;
    TileVals* agg2;
    TileVals* incl2;
    TileStart* starts2;
    uint32_t* hmask;
    LeftSlot* slots;
    uint32_t* heavy_item2;
    uint4* heavy_E2;
    size_t bytes;
};

PsaLayout carve_psa(void* scratch, uint64_t n, uint64_t num_tiles, uint64_t tile_items) {
    Carver c(scratch);
    PsaLayout L;
    L.hdr = c.take<BuildHeader>(2);
    L.hdr2 = L.hdr + 1;
    L.partials = c.take<double2>(kWsumMaxGrid);
    L.num_blocks = (num_tiles + kPrefixTiles - 1) / kPrefixTiles;
    L.blocks = c.take<BlockWord>(L.num_blocks);
    L.blocks2 = c.take<BlockWord>(L.num_blocks);
    L.agg = c.take<TileVals>(num_tiles);
    L.incl = c.take<TileVals>(num_tiles);
    L.agg2 = c.take<TileVals>(num_tiles);
    L.incl2 = c.take<TileVals>(num_tiles);
    L.starts2 = c.take<TileStart>(num_tiles + 1);
    L.hmask = c.take<uint32_t>(num_tiles * (tile_items / 32));
    L.slots = c.take<LeftSlot>(num_tiles * tile_items);
    L.heavy_item2 = c.take<uint32_t>(n);
    L.heavy_E2 = c.take<uint4>(n);
    L.bytes = c.off;
    return L;
}

template <int T>
wrs_status launch_psa(const float* d_w, uint64_t n, wrs_alias_row* d_table, double* d_W, const PsaLayout& L,
                      uint64_t num_tiles, cudaStream_t stream) {
    constexpr int NT = PackShape<T>::NT, IPT = PackShape<T>::IPT;
    const uint32_t nt = (uint32_t)num_tiles;
    if (cudaMemsetAsync(L.hdr, 0, 2 * sizeof(BuildHeader), stream) != cudaSuccess) return WRS_ERR_CUDA;
    if (cudaMemsetAsync(L.blocks2, 0, L.num_blocks * sizeof(BlockWord), stream) != cudaSuccess) return WRS_ERR_CUDA;
    const uint64_t zero_words = L.num_blocks * sizeof(BlockWord) / sizeof(uint32_t);
    wsum_kernel<kWsumBlock><<<wsum_grid(n), kWsumBlock, 0, stream>>>(d_w, n, L.hdr, L.partials,
                                                                     reinterpret_cast<uint32_t*>(L.blocks), zero_words,
                                                                     d_W);
    const TileMap map{nullptr, nullptr, nullptr, n, nt};
    // the kernels after wsum are programmatic dependents (launch_pdl)
    const auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    if (!ok(launch_pdl(tile_reduce_kernel<T, false>, dim3(nt), dim3(kReduceThreads), 0, stream, d_w, L.hdr, L.agg,
                       L.hmask, map)))
        return WRS_ERR_CUDA;
    const WaitCfg wc = current_wait_cfg();
    if (!ok(launch_pdl(tile_prefix_kernel, dim3((uint32_t)L.num_blocks), dim3(kPrefixThreads), 0, stream, L.hdr, L.agg,
                       L.incl, L.blocks, nt, wc)))
        return WRS_ERR_CUDA;
    {
        const size_t smem = psa_local_smem_bytes(T);
        if (cudaFuncSetAttribute(psa_local_kernel<NT, IPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return WRS_ERR_CUDA;
        if (!ok(launch_pdl(psa_local_kernel<NT, IPT>, dim3(nt), dim3(NT), smem, stream, d_w, n, L.hdr, L.incl, d_table,
                           L.slots, L.agg2, L.hdr2)))
            return WRS_ERR_CUDA;
    }
    if (!ok(launch_pdl(tile_prefix_kernel, dim3((uint32_t)L.num_blocks), dim3(kPrefixThreads), 0, stream, L.hdr2,
                       L.agg2, L.incl2, L.blocks2, nt, wc)))
        return WRS_ERR_CUDA;
    if (!ok(launch_pdl(psa_heavy_list_kernel<T>, dim3((nt + 3) / 4), dim3(128), 0, stream, L.hdr2, L.agg2, L.incl2,
                       L.slots, nt, L.heavy_item2, L.heavy_E2)))
        return WRS_ERR_CUDA;
    const uint32_t link_grid = ((nt + 1) * (uint32_t)kTileLinkLanes + 255) / 256;
    if (!ok(launch_pdl(tile_link_kernel<false>, dim3(link_grid), dim3(256), 0, stream, L.hdr2, L.incl2, nt, 1u,
                       L.heavy_E2, L.starts2, map)))
        return WRS_ERR_CUDA;
    {
        const size_t smem = pack_smem_bytes(T);
        if (cudaFuncSetAttribute(split_pack_kernel<NT, IPT, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return WRS_ERR_CUDA;
        if (!ok(launch_pdl(split_pack_kernel<NT, IPT, false, true>, dim3(nt), dim3(NT), smem, stream, d_w, L.hdr2,
                           L.incl2, L.starts2, L.heavy_item2, L.heavy_E2, nt, d_table, map, L.slots, nullptr)))
            return WRS_ERR_CUDA;
    }
    if (!ok(launch_pdl(copy_status_kernel, dim3(1), dim3(1), 0, stream, L.hdr2, L.hdr))) return WRS_ERR_CUDA;
    return launch_status();
}

}  // namespace
}  // namespace wrs

using namespace wrs;

extern "C" size_t wrs_sum_scratch_bytes(int64_t n) {
    (void)n;
    Carver c(nullptr);
    c.take<BuildHeader>(1);
    c.take<double2>(kWsumMaxGrid);
    return c.off;
}

extern "C" wrs_status wrs_sum_f32(const float* d_w, int64_t n, double* d_total, void* d_scratch,
                                  size_t scratch_bytes, void* stream_) {
    if (!d_w || !d_total || !d_scratch || n < 1 || n > kMaxItems) return WRS_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < wrs_sum_scratch_bytes(n)) return WRS_ERR_SCRATCH_TOO_SMALL;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    Carver c(d_scratch);
    BuildHeader* hdr = c.take<BuildHeader>(1);
    double2* partials = c.take<double2>(kWsumMaxGrid);
    if (cudaMemsetAsync(hdr, 0, sizeof(BuildHeader), stream) != cudaSuccess) return WRS_ERR_CUDA;
    wsum_kernel<kWsumBlock><<<wsum_grid((uint64_t)n), kWsumBlock, 0, stream>>>(d_w, (uint64_t)n, hdr, partials,
                                                                               nullptr, 0, d_total);
    return launch_status();
}

extern "C" size_t wrs_alias_build_scratch_bytes(int64_t n, const wrs_build_opts* opts) {
    const int64_t T = tile_items_for(opts);
    if (n < 1 || T < 0) return 0;
    const uint32_t prec = opts ? opts->precision : WRS_PRECISION_MIXED;
    if (prec != WRS_PRECISION_MIXED) {
        if (prec > WRS_PRECISION_FP32 || opts->method != WRS_METHOD_SPLIT) return 0;
        return prec == WRS_PRECISION_FP64 ? carve_prec<double>(nullptr, (uint64_t)n).bytes
                                          : carve_prec<float>(nullptr, (uint64_t)n).bytes;
    }
    const uint64_t nt = ((uint64_t)n + T - 1) / T;
    if (opts && opts->method == WRS_METHOD_PSA_PLUS) return carve_psa(nullptr, (uint64_t)n, nt, T).bytes;
    return carve_split(nullptr, (uint64_t)n, nt).bytes;
}

extern "C" wrs_status wrs_alias_build_f32(const float* d_w, int64_t n, const wrs_build_opts* opts,
                                          wrs_alias_row* d_table, double* d_W, void* d_scratch,
                                          size_t scratch_bytes, void* stream_) {
    if (!d_w || !d_table || !d_scratch || n < 1 || n > kMaxItems) return WRS_ERR_INVALID_ARGUMENT;
    const int64_t T = tile_items_for(opts);
    const uint32_t method = opts ? opts->method : WRS_METHOD_SPLIT;
    if (T < 0 || method > WRS_METHOD_PSA_PLUS) return WRS_ERR_INVALID_ARGUMENT;
    const uint64_t nt = ((uint64_t)n + T - 1) / T;
    const uint32_t prec = opts ? opts->precision : WRS_PRECISION_MIXED;
    if (prec != WRS_PRECISION_MIXED) {
        if (prec > WRS_PRECISION_FP32 || method != WRS_METHOD_SPLIT) return WRS_ERR_INVALID_ARGUMENT;
        cudaStream_t stream = static_cast<cudaStream_t>(stream_);
        wrs_status st;
        BuildHeader* hdr;
        if (prec == WRS_PRECISION_FP64) {
            if (scratch_bytes < carve_prec<double>(nullptr, (uint64_t)n).bytes) return WRS_ERR_SCRATCH_TOO_SMALL;
            const PrecLayout<double> L = carve_prec<double>(d_scratch, (uint64_t)n);
            hdr = L.hdr;
            st = launch_prec<double>(d_w, (uint64_t)n, d_table, d_W, L, stream);
        } else {
            if (scratch_bytes < carve_prec<float>(nullptr, (uint64_t)n).bytes) return WRS_ERR_SCRATCH_TOO_SMALL;
            const PrecLayout<float> L = carve_prec<float>(d_scratch, (uint64_t)n);
            hdr = L.hdr;
            st = launch_prec<float>(d_w, (uint64_t)n, d_table, d_W, L, stream);
        }
        if (st != WRS_SUCCESS) return st;
        if (opts->flags & WRS_FLAG_SYNC) return read_device_status(&hdr->status, stream);
        return WRS_SUCCESS;
    }
    if (method == WRS_METHOD_PSA_PLUS) {
        if (scratch_bytes < carve_psa(nullptr, (uint64_t)n, nt, T).bytes) return WRS_ERR_SCRATCH_TOO_SMALL;
        cudaStream_t stream = static_cast<cudaStream_t>(stream_);
        const PsaLayout L = carve_psa(d_scratch, (uint64_t)n, nt, T);
        wrs_status st;
        switch (T) {
            case 1024: st = launch_psa<1024>(d_w, (uint64_t)n, d_table, d_W, L, nt, stream); break;
            case 4096: st = launch_psa<4096>(d_w, (uint64_t)n, d_table, d_W, L, nt, stream); break;
            default: st = launch_psa<2048>(d_w, (uint64_t)n, d_table, d_W, L, nt, stream); break;
        }
        if (st != WRS_SUCCESS) return st;
        if (opts->flags & WRS_FLAG_SYNC) return read_device_status(&L.hdr->status, stream);
        return WRS_SUCCESS;
    }
    if (scratch_bytes < carve_split(nullptr, (uint64_t)n, nt).bytes) return WRS_ERR_SCRATCH_TOO_SMALL;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const SplitLayout L = carve_split(d_scratch, (uint64_t)n, nt);
    wrs_status st;
    switch (T) {
        case 1024: st = launch_split<1024>(d_w, (uint64_t)n, d_table, d_W, L, nt, stream); break;
        case 4096: st = launch_split<4096>(d_w, (uint64_t)n, d_table, d_W, L, nt, stream); break;
        default: st = launch_split<2048>(d_w, (uint64_t)n, d_table, d_W, L, nt, stream); break;
    }
    if (st != WRS_SUCCESS) return st;
    if (opts && (opts->flags & WRS_FLAG_SYNC)) return read_device_status(&L.hdr->status, stream);
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_scratch_status(const void* d_scratch, void* stream) {
    if (!d_scratch) return WRS_ERR_INVALID_ARGUMENT;
    return read_device_status(&static_cast<const BuildHeader*>(d_scratch)->status, static_cast<cudaStream_t>(stream));
}
