// batched.cu — C ABI of the batched (CSR) alias build, its sampler and its autotuner.
//
// wrs_batched_build_f32 / wrs_batched_sample replace a loop of AliasTableSplitGpu objects
// (construction/aliasTable/buildMethod/AliasTableSplitGpu.cu:388-468) and of
// SamplerGpuBasic::executeBenchmarkSampling (sampling/aliasTable/SamplerGpuBasic.cu:109-133),
// one per table, with a fixed launch sequence for the whole batch; wrs_batched_autotune
// replaces the reference's compile-time launch constants (AliasTableSplitGpu.cuh:60-94).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "batched_kernels.cuh"
#include "batched_rejection_kernels.cuh"
#include "host_util.h"

namespace wrs {
namespace {

constexpr uint32_t kDefaultSmall = 128;

// The library's side streams of the current device (created on first use): the listed tables
// of a batch are built and sampled on the first kSideStreams - 1, by size class, at the lowest
// stream priority; the tiled passes run on the last one, at the highest priority, so that their
// short grids (the longest chain of the call) get SMs first as the list kernels' CTAs retire.
constexpr int kMaxDevices = 64;
constexpr int kSideStreams = 5;
std::mutex g_side_mu;
cudaStream_t g_side[kMaxDevices][kSideStreams] = {};
wrs_status side_streams(cudaStream_t (&out)[kSideStreams]) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return WRS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_side_mu);
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (int k = 0; k < kSideStreams; ++k) {
        if (!g_side[dev][k] && cudaStreamCreateWithPriority(&g_side[dev][k], cudaStreamNonBlocking,
                                                            k == kSideStreams - 1 ? greatest : least) != cudaSuccess) {
            g_side[dev][k] = nullptr;
            return WRS_ERR_CUDA;
        }
        out[k] = g_side[dev][k];
    }
    return WRS_SUCCESS;
}

// Side streams forked from `stream` and joined back into it by events (which a stream capture
// records as a fork and a join). `mid` orders work between the side streams.
struct Fork {
    cudaStream_t side[kSideStreams];
    cudaEvent_t fork = nullptr, mid = nullptr, join[kSideStreams] = {};
    bool open = false;

    wrs_status begin(cudaStream_t stream) {
        for (int k = 0; k < kSideStreams; ++k) side[k] = stream;
        if (side_streams(side) != WRS_SUCCESS) return WRS_ERR_CUDA;
        bool ok = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess &&
                  cudaEventCreateWithFlags(&mid, cudaEventDisableTiming) == cudaSuccess;
        for (int k = 0; ok && k < kSideStreams; ++k)
            ok = cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaEventRecord(fork, stream) == cudaSuccess;
        for (int k = 0; ok && k < kSideStreams; ++k) ok = cudaStreamWaitEvent(side[k], fork, 0) == cudaSuccess;
        open = ok;
        return ok ? WRS_SUCCESS : WRS_ERR_CUDA;
    }
    // joins every side stream that was forked, so that a capture stays well formed
    wrs_status end(cudaStream_t stream) {
        bool ok = true;
        if (open)
            for (int k = 0; k < kSideStreams; ++k)
                ok = cudaEventRecord(join[k], side[k]) == cudaSuccess &&
                     cudaStreamWaitEvent(stream, join[k], 0) == cudaSuccess && ok;
        open = false;
        return ok ? WRS_SUCCESS : WRS_ERR_CUDA;
    }
    ~Fork() {
        if (fork) cudaEventDestroy(fork);
        if (mid) cudaEventDestroy(mid);
        for (int k = 0; k < kSideStreams; ++k)
            if (join[k]) cudaEventDestroy(join[k]);
    }
};

const uint32_t kSmallChoices[] = {32, 64, 128, 256, 512};
const uint32_t kTileChoices[] = {1024, 2048, 4096};

bool valid_small(uint32_t s) {
    for (uint32_t c : kSmallChoices)
        if (c == s) return true;
    return false;
}
bool valid_tile(uint32_t t) {
    for (uint32_t c : kTileChoices)
        if (c == t) return true;
    return false;
}

struct Shape {
    uint32_t small_max;
    uint32_t tile;
};

bool shape_of(const wrs_build_opts* opts, Shape* sh) {
    sh->small_max = (opts && opts->small_table_items) ? opts->small_table_items : kDefaultSmall;
    sh->tile = (opts && opts->tile_items) ? opts->tile_items : 2048u;
    return valid_small(sh->small_max) && valid_tile(sh->tile);
}

// The host's view of the batch for one shape (from h_offsets and h_kinds).
struct HostPlan {
    uint32_t listed_tables;          // alias tables with 1 <= n <= kMediumMax
    uint32_t empty_tables;           // tables with n = 0
    uint32_t list_tables[kLists];    // ... of them per list (table_list)
    uint64_t list_items[kLists];     // items of each list's tables
    uint64_t table_sum;              // sum over listed tables of (t + 1) * n_t (mod 2^64)
    uint32_t big_tables;             // alias tables with n > kMediumMax (tiled passes)
    uint32_t tiles;                  // tiles of the big tables
    uint64_t big_items;
    uint64_t rej_warp_tables;        // rejection tables with 1 <= n <= kRejWarpMax
    uint64_t rej_block_tables;       // larger rejection tables
    bool valid;
};

HostPlan host_plan(const int64_t* h_offsets, int64_t num_tables, const Shape& sh, const uint8_t* h_kinds = nullptr) {
    HostPlan p{};
    p.valid = true;
    if (!h_offsets || num_tables < 1 || h_offsets[0] != 0) {
        p.valid = false;
        return p;
    }
    uint64_t tiles = 0, tables = 0, listed = 0;
    for (int64_t t = 0; t < num_tables; ++t) {
        const int64_t n = h_offsets[t + 1] - h_offsets[t];
        if (n < 0 || n > (int64_t)0x7fffffff - 8192) {
            p.valid = false;
            return p;
        }
        if (n == 0) {
            ++p.empty_tables;
            continue;
        }
        const uint8_t kind = h_kinds ? h_kinds[t] : (uint8_t)WRS_TABLE_ALIAS;
        if (kind == WRS_TABLE_REJECTION) {
            if (n <= (int64_t)kRejWarpMax) ++p.rej_warp_tables; else ++p.rej_block_tables;
            continue;
        }
        if (kind != WRS_TABLE_ALIAS) continue;
        const int c = table_list(n, sh.small_max);
        if (c >= 0) {
            ++listed;
            ++p.list_tables[c];
            p.list_items[c] += (uint64_t)n;
            p.table_sum += (uint64_t)(t + 1) * (uint64_t)n;
        } else {
            ++tables;
            tiles += (uint64_t)((n + sh.tile - 1) / sh.tile);
            p.big_items += (uint64_t)n;
        }
    }
    // table ids of the lists are 32-bit
    if (tables > 0x7fffffffull || tiles > 0x7fffffffull || (listed > 0 && num_tables > (int64_t)0xffffffffll))
        p.valid = false;
    p.listed_tables = (uint32_t)listed;
    p.big_tables = (uint32_t)tables;
    p.tiles = (uint32_t)tiles;
    return p;
}

struct BatchLayout {
    BuildHeader* hdr0;  // batch status word
    uint32_t* plan_status;
    BuildHeader* hdrs;  // one per big table
    PlanCounts* blk;
    TableDesc* desc;
    uint32_t* tile_table;
    double2* partials;
    TileVals* agg;
    TileVals* incl;
    TileStart* starts;
    uint32_t* hmask;
    uint32_t* heavy_item;
    uint4* heavy_E;
    uint32_t* list;        // the listed tables' ids by list
    // build and sample only: the spill list, and the chunked sampler's tables and chunk prefix
    uint32_t* spill;
    uint32_t spill_cap;
    uint32_t* gen;
    uint64_t* gen_prefix;
    size_t bytes;
};

BatchLayout carve_batch(void* scratch, int64_t num_tables, const HostPlan& p, uint32_t tile,
                        bool sampling = false) {
    Carver c(scratch);
    BatchLayout L;
    // the batch header, the plan header and the per-table headers are contiguous: one memset
    // clears them all; the batch header comes first, so wrs_scratch_status reads its status
    L.hdr0 = c.take<BuildHeader>(2 + (size_t)p.big_tables);
    L.plan_status = &(L.hdr0 + 1)->status;
    L.hdrs = L.hdr0 + 2;
    L.blk = c.take<PlanCounts>((size_t)((num_tables + kPlanBlock - 1) / kPlanBlock));
    L.desc = c.take<TableDesc>(p.big_tables);
    L.tile_table = c.take<uint32_t>(p.tiles);
    L.partials = c.take<double2>(p.tiles);
    L.agg = c.take<TileVals>(p.tiles);
    L.incl = c.take<TileVals>(p.tiles);
    L.starts = c.take<TileStart>((size_t)p.tiles + p.big_tables);
    L.hmask = c.take<uint32_t>((size_t)p.tiles * (tile / 32));
    L.heavy_item = c.take<uint32_t>(p.big_items);
    L.heavy_E = c.take<uint4>(p.big_items);
    L.list = c.take<uint32_t>(p.listed_tables);
    L.spill_cap = sampling ? p.listed_tables + p.empty_tables : 0u;
    L.spill = c.take<uint32_t>(L.spill_cap);
    const size_t ngen = sampling ? (size_t)p.big_tables + L.spill_cap : 0;
    L.gen = c.take<uint32_t>(ngen);
    L.gen_prefix = c.take<uint64_t>(sampling ? ngen + 1 : 0);
    L.bytes = c.off;
    return L;
}

// Build and sample: where the samples go (wrs_batched_build_sample).
struct SampleArgs {
    const int64_t* d_sample_offsets;
    uint64_t total;
    uint64_t seed;
    uint64_t counter_base;
    uint32_t* d_out;
};

// The samples of list `cls`'s tables (those with at most kListSampleMax), on the list's stream.
wrs_status launch_list_sample(const wrs_alias_row* d_table, const int64_t* d_offsets, const TableLists& sl, int cls,
                              const SampleArgs& sa, const BatchLayout& L, uint32_t* status, cudaStream_t stream) {
    const uint32_t count = sl.cap[cls];
    if (count == 0) return WRS_SUCCESS;
    const DeviceInfo d = device_info();
    const uint64_t want = (count + kListSampleWarps - 1) / kListSampleWarps;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)d.sm_count * 8));
    list_sample_kernel<<<grid, 32 * kListSampleWarps, 0, stream>>>(
        d_table, d_offsets, sa.d_sample_offsets, sl.list + sl.base[cls], sl.cnt->list_fill + cls, count, sa.seed,
        sa.counter_base, sa.d_out, L.spill, &sl.cnt->spill_fill, L.spill_cap, status);
    return launch_status();
}

// The tables of one size class's list, a group of GW lanes each.
template <int SPL, int GW>
wrs_status launch_small_class(const float* d_w, const int64_t* d_offsets, const TableLists& sl, int cls,
                              wrs_alias_row* d_table, double* d_W, uint32_t* status, cudaStream_t stream) {
    const uint32_t count = sl.cap[cls];
    if (count == 0) return WRS_SUCCESS;
    constexpr int GPW = 32 / GW;
    const size_t smem = sizeof(SmallSmem<SPL, GW>) * kSmallWarps * GPW;
    cudaError_t e = cudaFuncSetAttribute(small_tables_kernel<SPL, GW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return WRS_ERR_CUDA;
    const DeviceInfo d = device_info();
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, small_tables_kernel<SPL, GW>, 32 * kSmallWarps, smem);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    const uint64_t want = ((uint64_t)count + kSmallWarps * GPW - 1) / (kSmallWarps * GPW);
    const uint64_t cap = (uint64_t)d.sm_count * per_sm;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min(want, cap));
    small_tables_kernel<SPL, GW><<<grid, 32 * kSmallWarps, smem, stream>>>(
        d_w, d_offsets, sl.list + sl.base[cls], sl.cnt->list_fill + cls, count, d_table, d_W, status);
    return launch_status();
}

// The medium tables of list `cls`, a CTA of MT threads each.
template <int MT>
wrs_status launch_medium(const float* d_w, const int64_t* d_offsets, const TableLists& sl, int cls,
                         wrs_alias_row* d_table, double* d_W, uint32_t* status, cudaStream_t stream) {
    const uint32_t count = sl.cap[cls];
    if (count == 0) return WRS_SUCCESS;
    constexpr size_t smem = medium_smem_bytes<MT>();
    cudaError_t e = cudaFuncSetAttribute(medium_tables_kernel<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return WRS_ERR_CUDA;
    const DeviceInfo d = device_info();
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, medium_tables_kernel<MT>, MT, smem);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(count, (uint64_t)d.sm_count * per_sm));
    medium_tables_kernel<MT><<<grid, MT, smem, stream>>>(d_w, d_offsets, sl.list + sl.base[cls], sl.cnt->list_fill + cls,
                                                         count, d_table, d_W, status);
    return launch_status();
}

// The listed tables (n <= kMediumMax): the lists on the first side stream, then one
// launch per list, the lists spread over the side streams (a launch waits for its slowest
// table, so lists run side by side).
template <int SPL>
wrs_status launch_lists(const float* d_w, const int64_t* d_offsets, const uint8_t* d_kinds, int64_t num_tables,
                        wrs_alias_row* d_table, double* d_W, const BatchLayout& L, const HostPlan& p, Fork& f,
                        const SampleArgs* sa) {
    BatchCounters* bc = reinterpret_cast<BatchCounters*>(L.hdr0);  // cleared with the headers
    uint32_t* status = &bc->status;
    TableLists sl;
    sl.cnt = bc;
    sl.list = L.list;
    uint32_t base = 0;
    for (int c = 0; c < kLists; ++c) {
        sl.base[c] = base;
        sl.cap[c] = p.list_tables[c];
        sl.items[c] = p.list_items[c];
        base += sl.cap[c];
    }
    sl.table_sum = p.table_sum;
    const uint64_t nblk = ((uint64_t)num_tables + kListThreads - 1) / kListThreads;
    const cudaStream_t* ss = f.side;
    table_lists_kernel<<<(uint32_t)nblk, kListThreads, 0, ss[0]>>>(d_offsets, d_kinds, num_tables, 32u * SPL, sl,
                                                                  status, sa ? sa->d_sample_offsets : nullptr,
                                                                  L.spill, L.spill_cap);
    lists_check_kernel<<<1, 32, 0, ss[0]>>>(sl, status);
    wrs_status st = launch_status();
    if (st != WRS_SUCCESS) return st;
    if (cudaEventRecord(f.mid, ss[0]) != cudaSuccess) return WRS_ERR_CUDA;
    for (int k = 1; k < kSideStreams - 1; ++k)  // the list streams (the last one runs the tiled passes)
        if (cudaStreamWaitEvent(ss[k], f.mid, 0) != cudaSuccess) return WRS_ERR_CUDA;
    // each list's samples (build and sample) right after the list, on the same stream
    auto sampled = [&](wrs_status s2, int cls, cudaStream_t strm) {
        if (s2 != WRS_SUCCESS || !sa) return s2;
        return launch_list_sample(d_table, d_offsets, sl, cls, *sa, L, status, strm);
    };
    if (st == WRS_SUCCESS)
        st = sampled(launch_medium<1024>(d_w, d_offsets, sl, 7, d_table, d_W, status, ss[3]), 7, ss[3]);
    if (st == WRS_SUCCESS)
        st = sampled(launch_small_class<2, 2>(d_w, d_offsets, sl, 0, d_table, d_W, status, ss[0]), 0, ss[0]);
    if (st == WRS_SUCCESS)
        st = sampled(launch_medium<256>(d_w, d_offsets, sl, 6, d_table, d_W, status, ss[1]), 6, ss[1]);
    if (st == WRS_SUCCESS)
        st = sampled(launch_small_class<2, 4>(d_w, d_offsets, sl, 1, d_table, d_W, status, ss[2]), 1, ss[2]);
    if (st == WRS_SUCCESS)
        st = sampled(launch_small_class<2, 8>(d_w, d_offsets, sl, 2, d_table, d_W, status, ss[2]), 2, ss[2]);
    if (st == WRS_SUCCESS)
        st = sampled(launch_small_class<2, 16>(d_w, d_offsets, sl, 3, d_table, d_W, status, ss[1]), 3, ss[1]);
    if constexpr (SPL >= 2) {
        if (st == WRS_SUCCESS)
            st = sampled(launch_small_class<2, 32>(d_w, d_offsets, sl, 4, d_table, d_W, status, ss[3]), 4, ss[3]);
    }
    if constexpr (SPL > 2) {
        if (st == WRS_SUCCESS)
            st = sampled(launch_small_class<SPL, 32>(d_w, d_offsets, sl, 5, d_table, d_W, status, ss[2]), 5, ss[2]);
    }
    return st;
}

template <int T>
wrs_status launch_big(const float* d_w, const int64_t* d_offsets, const uint8_t* d_kinds, int64_t num_tables,
                      wrs_alias_row* d_table, double* d_W, const BatchLayout& L, const HostPlan& p,
                      cudaStream_t stream) {
    const uint32_t big_min = (uint32_t)kMediumMax;  // the tiled passes take the tables above it
    constexpr int NT = PackShape<T>::NT, IPT = PackShape<T>::IPT;
    const uint32_t nblk = (uint32_t)((num_tables + kPlanBlock - 1) / kPlanBlock);
    const PlanCounts cap{p.big_tables, p.tiles, p.big_items};
    plan_count_kernel<<<nblk, kPlanBlock, 0, stream>>>(d_offsets, d_kinds, num_tables, big_min, T, L.blk);
    // the kernels after plan_count are launched as programmatic dependents: each starts while its
    // predecessor's last wave runs and waits for the predecessor's completion on entry
    const auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    if (!ok(launch_pdl(plan_scan_kernel, dim3(1), dim3(kPlanBlock), 0, stream, L.blk, nblk, cap, L.plan_status)))
        return WRS_ERR_CUDA;
    if (!ok(launch_pdl(plan_fill_kernel, dim3(nblk), dim3(kPlanBlock), 0, stream, d_offsets, d_kinds, num_tables,
                       big_min, (uint32_t)T, L.blk, cap, L.desc, L.tile_table)))
        return WRS_ERR_CUDA;
    const TileMap map{L.tile_table, L.desc, L.plan_status, 0, 0};
    const uint32_t nt = p.tiles;
    if (!ok(launch_pdl(batch_wsum_kernel<T>, dim3(nt), dim3(kBatchWsumThreads), 0, stream, d_w, L.hdrs, L.partials,
                       map, d_W)))
        return WRS_ERR_CUDA;
    if (!ok(launch_pdl(tile_reduce_kernel<T, true>, dim3(nt), dim3(kReduceThreads), 0, stream, d_w, L.hdrs, L.agg,
                       L.hmask, map)))
        return WRS_ERR_CUDA;
    if (!ok(launch_pdl(batch_prefix_kernel, dim3(p.big_tables), dim3(kPrefixThreads), 0, stream, L.hdrs, L.agg,
                       L.incl, L.desc, L.plan_status)))
        return WRS_ERR_CUDA;
    if (!ok(launch_pdl(heavy_list_kernel<T, true>, dim3((nt + heavy_warps(T) - 1) / heavy_warps(T)),
                       dim3(32 * heavy_warps(T)), 0, stream, d_w, L.hdrs, L.agg, L.incl, L.hmask, nt, L.heavy_item,
                       L.heavy_E, map)))
        return WRS_ERR_CUDA;
    const uint32_t link_grid = ((nt + p.big_tables) * (uint32_t)kTileLinkLanes + 255) / 256;
    if (!ok(launch_pdl(tile_link_kernel<true>, dim3(link_grid), dim3(256), 0, stream, L.hdrs, L.incl, nt,
                       p.big_tables, L.heavy_E, L.starts, map)))
        return WRS_ERR_CUDA;
    const size_t smem = pack_smem_bytes(T);
    const cudaError_t e = cudaFuncSetAttribute(split_pack_kernel<NT, IPT, true, false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return WRS_ERR_CUDA;
    if (!ok(launch_pdl(split_pack_kernel<NT, IPT, true, false>, dim3(nt), dim3(NT), smem, stream, d_w, L.hdrs, L.incl,
                       L.starts, L.heavy_item, L.heavy_E, nt, d_table, map, nullptr, nullptr)))
        return WRS_ERR_CUDA;
    if (!ok(launch_pdl(batch_status_kernel, dim3((p.big_tables + 1 + 255) / 256), dim3(256), 0, stream, L.hdr0 + 1,
                       p.big_tables + 1, &L.hdr0->status)))
        return WRS_ERR_CUDA;
    return launch_status();
}

// Rejection structures of the batch's rejection tables (errors into the batch status word).
struct RejOut {
    uint32_t* A;
    float* frac;
    uint64_t* a_size;
};

wrs_status launch_rejection(const float* d_w, const int64_t* d_offsets, const uint8_t* d_kinds, int64_t num_tables,
                            const HostPlan& p, const RejOut& r, double* d_W, uint32_t* status, cudaStream_t stream) {
    const DeviceInfo d = device_info();
    if (p.rej_warp_tables > 0) {
        const uint64_t want = (p.rej_warp_tables + kRejWarps - 1) / kRejWarps;
        const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)d.sm_count * 8));
        rej_warp_tables_kernel<<<grid, 32 * kRejWarps, 0, stream>>>(d_w, d_offsets, d_kinds, num_tables, r.A, r.frac,
                                                                   r.a_size, d_W, status);
    }
    if (p.rej_block_tables > 0) {
        const uint32_t grid =
            (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(p.rej_block_tables, (uint64_t)d.sm_count * 2));
        rej_block_tables_kernel<<<grid, kRejBlockThreads, 0, stream>>>(d_w, d_offsets, d_kinds, num_tables,
                                                                      kRejWarpMax, r.A, r.frac, r.a_size, d_W,
                                                                      status);
    }
    return launch_status();
}

wrs_status batched_build(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets, int64_t num_tables,
                         const Shape& sh, wrs_alias_row* d_table, double* d_W, void* d_scratch, size_t scratch_bytes,
                         cudaStream_t stream, BatchLayout* out_layout, const uint8_t* d_kinds = nullptr,
                         const uint8_t* h_kinds = nullptr, const RejOut* rej = nullptr,
                         const SampleArgs* sa = nullptr) {
    const HostPlan p = host_plan(h_offsets, num_tables, sh, h_kinds);
    if (!p.valid) return WRS_ERR_INVALID_ARGUMENT;
    const BatchLayout L = carve_batch(d_scratch, num_tables, p, sh.tile, sa != nullptr);
    if (scratch_bytes < L.bytes) return WRS_ERR_SCRATCH_TOO_SMALL;
    if (out_layout) *out_layout = L;
    if (cudaMemsetAsync(L.hdr0, 0, sizeof(BuildHeader) * (2 + (size_t)p.big_tables), stream) != cudaSuccess)
        return WRS_ERR_CUDA;
    wrs_status st = WRS_SUCCESS;
    // the listed tables and the tiled tables are independent: the former run on the side streams
    // (with samples, the lists pass also finds the empty tables that have samples)
    const bool lists = p.listed_tables > 0 || (sa && p.empty_tables > 0);
    Fork f;
    if (lists && f.begin(stream) != WRS_SUCCESS) {
        f.end(stream);
        return WRS_ERR_CUDA;
    }
    if (lists) {
        switch (sh.small_max) {
            case 32: st = launch_lists<1>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, f, sa); break;
            case 64: st = launch_lists<2>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, f, sa); break;
            case 128: st = launch_lists<4>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, f, sa); break;
            case 256: st = launch_lists<8>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, f, sa); break;
            default: st = launch_lists<16>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, f, sa); break;
        }
    }
    if (st == WRS_SUCCESS && p.big_tables > 0) {
        const cudaStream_t bs = lists ? f.side[kSideStreams - 1] : stream;
        switch (sh.tile) {
            case 1024: st = launch_big<1024>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, bs); break;
            case 4096: st = launch_big<4096>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, bs); break;
            default: st = launch_big<2048>(d_w, d_offsets, d_kinds, num_tables, d_table, d_W, L, p, bs); break;
        }
    }
    if (f.end(stream) != WRS_SUCCESS && st == WRS_SUCCESS) st = WRS_ERR_CUDA;
    if (st != WRS_SUCCESS) return st;
    if (sa) {  // the tiled tables' samples and the spilled ones, after every build
        BatchCounters* bc = reinterpret_cast<BatchCounters*>(L.hdr0);
        const uint32_t* plan_status = p.big_tables > 0 ? L.plan_status : nullptr;
        chunks_plan_kernel<<<1, 1024, 0, stream>>>(L.desc, p.big_tables, plan_status, L.spill, &bc->spill_fill,
                                                   L.spill_cap, sa->d_sample_offsets, num_tables, sa->total, L.gen,
                                                   L.gen_prefix, &bc->chunks, &bc->status);
        const DeviceInfo d = device_info();
        chunk_sample_kernel<<<d.sm_count * 8, kChunkThreads, 0, stream>>>(
            d_table, d_offsets, sa->d_sample_offsets, L.gen, L.gen_prefix, &bc->spill_fill, L.spill_cap, plan_status,
            p.big_tables, &bc->chunks, sa->seed, sa->counter_base, sa->d_out, &bc->status);
        st = launch_status();
    }
    if (rej && (p.rej_warp_tables > 0 || p.rej_block_tables > 0))
        st = launch_rejection(d_w, d_offsets, d_kinds, num_tables, p, *rej, d_W, &L.hdr0->status, stream);
    return st;
}

}  // namespace
}  // namespace wrs

using namespace wrs;

extern "C" size_t wrs_batched_build_scratch_bytes(const int64_t* h_offsets, int64_t num_tables,
                                                  const wrs_build_opts* opts) {
    if (opts) {
        Shape sh;
        if (!shape_of(opts, &sh)) return 0;
        const HostPlan p = host_plan(h_offsets, num_tables, sh);
        return p.valid ? carve_batch(nullptr, num_tables, p, sh.tile).bytes : 0;
    }
    size_t best = 0;
    for (uint32_t s : kSmallChoices)
        for (uint32_t t : kTileChoices) {
            const Shape sh{s, t};
            const HostPlan p = host_plan(h_offsets, num_tables, sh);
            if (!p.valid) return 0;
            best = std::max(best, carve_batch(nullptr, num_tables, p, t).bytes);
        }
    return best;
}

extern "C" wrs_status wrs_batched_build_f32(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                            int64_t num_tables, const wrs_build_opts* opts, wrs_alias_row* d_table,
                                            double* d_W, void* d_scratch, size_t scratch_bytes, void* stream_) {
    if (!d_w || !d_offsets || !h_offsets || !d_table || !d_scratch || num_tables < 1) return WRS_ERR_INVALID_ARGUMENT;
    Shape sh;
    if (!shape_of(opts, &sh)) return WRS_ERR_INVALID_ARGUMENT;
    if (opts && opts->method != WRS_METHOD_SPLIT) return WRS_ERR_UNSUPPORTED;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    BatchLayout L;
    const wrs_status st = batched_build(d_w, d_offsets, h_offsets, num_tables, sh, d_table, d_W, d_scratch,
                                        scratch_bytes, stream, &L);
    if (st != WRS_SUCCESS) return st;
    if (opts && (opts->flags & WRS_FLAG_SYNC)) return read_device_status(&L.hdr0->status, stream);
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_batched_sample(const wrs_alias_row* d_table, const int64_t* d_offsets, int64_t num_tables,
                                         const int64_t* d_sample_offsets, uint64_t total_samples, uint64_t seed,
                                         uint64_t counter_base, uint32_t* d_out, void* stream_) {
    if (!d_table || !d_offsets || !d_sample_offsets || !d_out || num_tables < 1) return WRS_ERR_INVALID_ARGUMENT;
    if (total_samples == 0) return WRS_SUCCESS;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const uint64_t per_cta = (uint64_t)kBatchSampleThreads * kBatchSamplePer;
    const uint64_t grid = (total_samples + per_cta - 1) / per_cta;
    if (grid > 0x7fffffffull) return WRS_ERR_INVALID_ARGUMENT;
    batch_sample_kernel<<<(uint32_t)grid, kBatchSampleThreads, 0, stream>>>(
        d_table, d_offsets, num_tables, d_sample_offsets, total_samples, seed, counter_base, d_out, nullptr, nullptr,
        nullptr, nullptr, nullptr, 0u);
    return launch_status();
}

extern "C" size_t wrs_batched_build_sample_scratch_bytes(const int64_t* h_offsets, int64_t num_tables,
                                                         const wrs_build_opts* opts) {
    auto bytes = [&](const Shape& sh) -> size_t {
        const HostPlan p = host_plan(h_offsets, num_tables, sh);
        return p.valid ? carve_batch(nullptr, num_tables, p, sh.tile, true).bytes : 0;
    };
    if (opts) {
        Shape sh;
        return shape_of(opts, &sh) ? bytes(sh) : 0;
    }
    size_t best = 0;
    for (uint32_t s : kSmallChoices)
        for (uint32_t t : kTileChoices) {
            const size_t b = bytes(Shape{s, t});
            if (b == 0) return 0;
            best = std::max(best, b);
        }
    return best;
}

extern "C" wrs_status wrs_batched_build_sample(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                               int64_t num_tables, const wrs_build_opts* opts, wrs_alias_row* d_table,
                                               double* d_W, const int64_t* d_sample_offsets, uint64_t total_samples,
                                               uint64_t seed, uint64_t counter_base, uint32_t* d_out, void* d_scratch,
                                               size_t scratch_bytes, void* stream_) {
    if (!d_w || !d_offsets || !h_offsets || !d_table || !d_scratch || !d_sample_offsets || num_tables < 1 ||
        (total_samples > 0 && !d_out))
        return WRS_ERR_INVALID_ARGUMENT;
    Shape sh;
    if (!shape_of(opts, &sh)) return WRS_ERR_INVALID_ARGUMENT;
    if (opts && opts->method != WRS_METHOD_SPLIT) return WRS_ERR_UNSUPPORTED;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const SampleArgs sa{d_sample_offsets, total_samples, seed, counter_base, d_out};
    BatchLayout L;
    const wrs_status st = batched_build(d_w, d_offsets, h_offsets, num_tables, sh, d_table, d_W, d_scratch,
                                        scratch_bytes, stream, &L, nullptr, nullptr, nullptr, &sa);
    if (st != WRS_SUCCESS) return st;
    if (opts && (opts->flags & WRS_FLAG_SYNC)) return read_device_status(&L.hdr0->status, stream);
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_batched_per_table(const float* d_w, const int64_t* h_offsets,
                                            const int64_t* h_sample_offsets, const int64_t* h_tables, int64_t num_ids,
                                            const wrs_build_opts* opts, wrs_alias_row* d_table, uint64_t seed,
                                            uint64_t counter_base, uint32_t* d_out, void* d_scratch,
                                            size_t scratch_bytes, void* stream) {
    if (!d_w || !h_offsets || !h_sample_offsets || !h_tables || num_ids < 0 || !d_table || !d_scratch)
        return WRS_ERR_INVALID_ARGUMENT;
    for (int64_t i = 0; i < num_ids; ++i) {
        const int64_t t = h_tables[i];
        const int64_t off = h_offsets[t], n = h_offsets[t + 1] - off;
        const int64_t s0 = h_sample_offsets[t], cnt = h_sample_offsets[t + 1] - s0;
        if (n < 0 || cnt < 0) return WRS_ERR_INVALID_ARGUMENT;
        if (n == 0) continue;
        wrs_status st = wrs_alias_build_f32(d_w + off, n, opts, d_table + off, nullptr, d_scratch, scratch_bytes, stream);
        if (st == WRS_SUCCESS && cnt > 0)
            st = wrs_alias_sample(d_table + off, n, (uint64_t)cnt, seed, counter_base + (uint64_t)s0, nullptr,
                                  d_out + s0, nullptr, stream);
        if (st != WRS_SUCCESS) return st;
    }
    return WRS_SUCCESS;
}

namespace wrs {
namespace {

// Times every launch shape of this batch's build (with `sa`, of its build and sample) and writes
// the fastest into *opts. Every shape is captured into a graph and its launches timed, so that
// the host's planning (a pass over the offsets per call) stays out of the device time.
wrs_status autotune_shapes(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets, int64_t num_tables,
                           wrs_alias_row* d_table, void* d_scratch, size_t scratch_bytes, wrs_build_opts* opts,
                           cudaStream_t stream, const SampleArgs* sa) {
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return WRS_ERR_CUDA;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return WRS_ERR_CUDA;
    }
    float best_ms = 1e30f;
    Shape best{kDefaultSmall, 2048};
    wrs_status result = WRS_SUCCESS;
    cudaStream_t cap = nullptr;  // the capture stream, ordered after the caller's stream
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess || cudaEventRecord(e0, stream) != cudaSuccess ||
        cudaStreamWaitEvent(cap, e0, 0) != cudaSuccess)
        result = WRS_ERR_CUDA;
    for (uint32_t s : kSmallChoices) {
        for (uint32_t t : kTileChoices) {
            if (result != WRS_SUCCESS) break;
            const Shape sh{s, t};
            BatchLayout L;
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            wrs_status st = WRS_SUCCESS;
            if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                result = WRS_ERR_CUDA;
                break;
            }
            st = batched_build(d_w, d_offsets, h_offsets, num_tables, sh, d_table, nullptr, d_scratch, scratch_bytes,
                               cap, &L, nullptr, nullptr, nullptr, sa);
            if (cudaStreamEndCapture(cap, &graph) != cudaSuccess && st == WRS_SUCCESS) st = WRS_ERR_CUDA;
            // with node priorities, as a caller should instantiate it: the tiled passes' side stream
            // keeps its higher priority in the replay
            if (st == WRS_SUCCESS &&
                cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess)
                st = WRS_ERR_CUDA;
            float ms_min = 1e30f;
            for (int rep = 0; st == WRS_SUCCESS && rep < 4; ++rep) {  // the first launch warms up
                cudaEventRecord(e0, cap);
                if (cudaGraphLaunch(exec, cap) != cudaSuccess) st = WRS_ERR_CUDA;
                cudaEventRecord(e1, cap);
                if (st == WRS_SUCCESS) st = read_device_status(&L.hdr0->status, cap);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) ms_min = std::min(ms_min, ms);
            }
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            if (st != WRS_SUCCESS) {
                result = st;
                break;
            }
            if (ms_min < best_ms) {
                best_ms = ms_min;
                best = sh;
            }
        }
    }
    if (cap) {
        cudaStreamSynchronize(cap);
        cudaStreamDestroy(cap);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (result != WRS_SUCCESS) return result;
    opts->small_table_items = best.small_max;
    opts->tile_items = best.tile;
    return WRS_SUCCESS;
}

}  // namespace
}  // namespace wrs

extern "C" wrs_status wrs_batched_autotune(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                           int64_t num_tables, wrs_alias_row* d_table, void* d_scratch,
                                           size_t scratch_bytes, wrs_build_opts* opts, void* stream_) {
    if (!opts || !d_w || !d_offsets || !h_offsets || !d_table || !d_scratch) return WRS_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < wrs_batched_build_scratch_bytes(h_offsets, num_tables, nullptr))
        return WRS_ERR_SCRATCH_TOO_SMALL;
    return autotune_shapes(d_w, d_offsets, h_offsets, num_tables, d_table, d_scratch, scratch_bytes, opts,
                           static_cast<cudaStream_t>(stream_), nullptr);
}

extern "C" wrs_status wrs_batched_autotune_build_sample(const float* d_w, const int64_t* d_offsets,
                                                        const int64_t* h_offsets, int64_t num_tables,
                                                        wrs_alias_row* d_table, const int64_t* d_sample_offsets,
                                                        uint64_t total_samples, uint32_t* d_out, void* d_scratch,
                                                        size_t scratch_bytes, wrs_build_opts* opts, void* stream_) {
    if (!opts || !d_w || !d_offsets || !h_offsets || !d_table || !d_scratch || !d_sample_offsets ||
        (total_samples > 0 && !d_out))
        return WRS_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < wrs_batched_build_sample_scratch_bytes(h_offsets, num_tables, nullptr))
        return WRS_ERR_SCRATCH_TOO_SMALL;
    const SampleArgs sa{d_sample_offsets, total_samples, 0, 0, d_out};
    return autotune_shapes(d_w, d_offsets, h_offsets, num_tables, d_table, d_scratch, scratch_bytes, opts,
                           static_cast<cudaStream_t>(stream_), &sa);
}

// ---------------------------------------------------------------- mixed batches
namespace wrs {
namespace {

size_t mixed_scratch_bytes(const int64_t* h_offsets, const uint8_t* h_kinds, int64_t num_tables,
                           const wrs_build_opts* opts) {
    if (opts) {
        Shape sh;
        if (!shape_of(opts, &sh)) return 0;
        const HostPlan p = host_plan(h_offsets, num_tables, sh, h_kinds);
        return p.valid ? carve_batch(nullptr, num_tables, p, sh.tile).bytes : 0;
    }
    size_t best = 0;
    for (uint32_t s : kSmallChoices)
        for (uint32_t t : kTileChoices) {
            const Shape sh{s, t};
            const HostPlan p = host_plan(h_offsets, num_tables, sh, h_kinds);
            if (!p.valid) return 0;
            best = std::max(best, carve_batch(nullptr, num_tables, p, t).bytes);
        }
    return best;
}

wrs_status launch_mixed_sample(const wrs_alias_row* d_table, const uint32_t* d_A, const float* d_frac,
                               const uint64_t* d_a_size, const int64_t* d_offsets, const uint8_t* d_kinds,
                               int64_t num_tables, const int64_t* d_sample_offsets, uint64_t total_samples,
                               uint64_t seed, uint64_t counter_base, uint32_t max_tries, uint32_t* d_out,
                               uint32_t* d_status, cudaStream_t stream) {
    if (total_samples == 0) return WRS_SUCCESS;
    const uint64_t per_cta = (uint64_t)kBatchSampleThreads * kBatchSamplePer;
    const uint64_t grid = (total_samples + per_cta - 1) / per_cta;
    if (grid > 0x7fffffffull) return WRS_ERR_INVALID_ARGUMENT;
    batch_sample_kernel<<<(uint32_t)grid, kBatchSampleThreads, 0, stream>>>(
        d_table, d_offsets, num_tables, d_sample_offsets, total_samples, seed, counter_base, d_out, d_status, d_kinds,
        d_A, d_frac, d_a_size, max_tries ? max_tries : 64u);
    return launch_status();
}

// Size class of a table of n >= 1 items: ceil(log2 n).
int size_class(int64_t n) { return n <= 1 ? 0 : 64 - __builtin_clzll((unsigned long long)(n - 1)); }

}  // namespace
}  // namespace wrs

extern "C" size_t wrs_batched_mixed_build_scratch_bytes(const int64_t* h_offsets, const uint8_t* h_kinds,
                                                        int64_t num_tables, const wrs_build_opts* opts) {
    return mixed_scratch_bytes(h_offsets, h_kinds, num_tables, opts);
}

extern "C" wrs_status wrs_batched_mixed_build_f32(const float* d_w, const int64_t* d_offsets,
                                                  const int64_t* h_offsets, const uint8_t* d_kinds,
                                                  const uint8_t* h_kinds, int64_t num_tables,
                                                  const wrs_build_opts* opts, wrs_alias_row* d_table, uint32_t* d_A,
                                                  float* d_frac, uint64_t* d_a_size, double* d_W, void* d_scratch,
                                                  size_t scratch_bytes, void* stream_) {
    if (!d_w || !d_offsets || !h_offsets || !d_scratch || num_tables < 1) return WRS_ERR_INVALID_ARGUMENT;
    if ((d_kinds == nullptr) != (h_kinds == nullptr)) return WRS_ERR_INVALID_ARGUMENT;
    Shape sh;
    if (!shape_of(opts, &sh)) return WRS_ERR_INVALID_ARGUMENT;
    if (opts && opts->method != WRS_METHOD_SPLIT) return WRS_ERR_UNSUPPORTED;
    const HostPlan p = host_plan(h_offsets, num_tables, sh, h_kinds);
    if (!p.valid) return WRS_ERR_INVALID_ARGUMENT;
    if ((p.listed_tables > 0 || p.big_tables > 0) && !d_table) return WRS_ERR_INVALID_ARGUMENT;
    if ((p.rej_warp_tables > 0 || p.rej_block_tables > 0) && (!d_A || !d_frac || !d_a_size))
        return WRS_ERR_INVALID_ARGUMENT;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    const RejOut r{d_A, d_frac, d_a_size};
    BatchLayout L;
    const wrs_status st = batched_build(d_w, d_offsets, h_offsets, num_tables, sh, d_table, d_W, d_scratch,
                                        scratch_bytes, stream, &L, d_kinds, h_kinds, &r);
    if (st != WRS_SUCCESS) return st;
    if (opts && (opts->flags & WRS_FLAG_SYNC)) return read_device_status(&L.hdr0->status, stream);
    return WRS_SUCCESS;
}

extern "C" wrs_status wrs_batched_mixed_sample(const wrs_alias_row* d_table, const uint32_t* d_A,
                                               const float* d_frac, const uint64_t* d_a_size,
                                               const int64_t* d_offsets, const uint8_t* d_kinds, int64_t num_tables,
                                               const int64_t* d_sample_offsets, uint64_t total_samples, uint64_t seed,
                                               uint64_t counter_base, uint32_t max_tries, uint32_t* d_out,
                                               uint32_t* d_status, void* stream_) {
    if (!d_offsets || !d_sample_offsets || !d_out || num_tables < 1) return WRS_ERR_INVALID_ARGUMENT;
    if (!d_kinds && !d_table) return WRS_ERR_INVALID_ARGUMENT;
    if (d_kinds && (!d_A || !d_frac || !d_a_size)) return WRS_ERR_INVALID_ARGUMENT;
    return launch_mixed_sample(d_table, d_A, d_frac, d_a_size, d_offsets, d_kinds, num_tables, d_sample_offsets,
                               total_samples, seed, counter_base, max_tries, d_out, d_status,
                               static_cast<cudaStream_t>(stream_));
}

extern "C" wrs_status wrs_batched_autotune_kinds(const float* d_w, const int64_t* d_offsets,
                                                 const int64_t* h_offsets, int64_t num_tables,
                                                 const int64_t* d_sample_offsets, const int64_t* h_sample_offsets,
                                                 const wrs_build_opts* opts, wrs_alias_row* d_table, uint32_t* d_A,
                                                 float* d_frac, uint64_t* d_a_size, uint8_t* d_kinds_tmp,
                                                 uint32_t* d_out, void* d_scratch, size_t scratch_bytes,
                                                 uint8_t* h_kinds_out, uint8_t* class_kinds, float* class_ms,
                                                 void* stream_) {
    if (!d_w || !d_offsets || !h_offsets || !d_sample_offsets || !h_sample_offsets || !d_table || !d_A || !d_frac ||
        !d_a_size || !d_kinds_tmp || !d_out || !d_scratch || !h_kinds_out || num_tables < 1)
        return WRS_ERR_INVALID_ARGUMENT;
    Shape sh;
    if (!shape_of(opts, &sh)) return WRS_ERR_INVALID_ARGUMENT;
    if (opts && opts->method != WRS_METHOD_SPLIT) return WRS_ERR_UNSUPPORTED;
    const HostPlan p_all = host_plan(h_offsets, num_tables, sh, nullptr);
    if (!p_all.valid) return WRS_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < mixed_scratch_bytes(h_offsets, nullptr, num_tables, opts)) return WRS_ERR_SCRATCH_TOO_SMALL;
    const int64_t total_i = h_sample_offsets[num_tables];
    if (h_sample_offsets[0] != 0 || total_i < 0) return WRS_ERR_INVALID_ARGUMENT;
    const uint64_t total = (uint64_t)total_i;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_);
    constexpr int kClasses = 33;
    constexpr float kRejectionWins = 0.95f;  // rejection's time over alias's below which it is chosen
    std::vector<int> cls((size_t)num_tables);
    bool present[kClasses] = {};
    for (int64_t t = 0; t < num_tables; ++t) {
        const int64_t n = h_offsets[t + 1] - h_offsets[t];
        cls[(size_t)t] = n > 0 ? size_class(n) : -1;
        if (n > 0) present[cls[(size_t)t]] = true;
    }
    uint8_t choice[kClasses];
    for (int c = 0; c < kClasses; ++c) choice[c] = WRS_TABLE_SKIP;
    if (class_ms)
        for (int c = 0; c < 2 * kClasses; ++c) class_ms[c] = 0.0f;
    std::vector<uint8_t> kinds((size_t)num_tables);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return WRS_ERR_CUDA;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return WRS_ERR_CUDA;
    }
    const RejOut r{d_A, d_frac, d_a_size};
    wrs_status result = WRS_SUCCESS;
    for (int c = 0; c < kClasses && result == WRS_SUCCESS; ++c) {
        if (!present[c]) continue;
        float ms_of[2] = {1e30f, 1e30f};
        for (int m = 0; m < 2 && result == WRS_SUCCESS; ++m) {
            const uint8_t kind = m == 0 ? (uint8_t)WRS_TABLE_ALIAS : (uint8_t)WRS_TABLE_REJECTION;
            for (int64_t t = 0; t < num_tables; ++t) kinds[(size_t)t] = cls[(size_t)t] == c ? kind : WRS_TABLE_SKIP;
            if (cudaMemcpyAsync(d_kinds_tmp, kinds.data(), (size_t)num_tables, cudaMemcpyHostToDevice, stream) !=
                cudaSuccess) {
                result = WRS_ERR_CUDA;
                break;
            }
            for (int rep = 0; rep < 3; ++rep) {  // the first run warms up
                BatchLayout L;
                cudaEventRecord(e0, stream);
                wrs_status st = batched_build(d_w, d_offsets, h_offsets, num_tables, sh, d_table, nullptr, d_scratch,
                                              scratch_bytes, stream, &L, d_kinds_tmp, kinds.data(), &r);
                if (st == WRS_SUCCESS)
                    st = launch_mixed_sample(d_table, d_A, d_frac, d_a_size, d_offsets, d_kinds_tmp, num_tables,
                                             d_sample_offsets, total, 0x5A5A5A5Aull, 0, 0, d_out, nullptr, stream);
                cudaEventRecord(e1, stream);
                if (st == WRS_SUCCESS) st = read_device_status(&L.hdr0->status, stream);
                if (st != WRS_SUCCESS) {
                    result = st;
                    break;
                }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0) ms_of[m] = std::min(ms_of[m], ms);
            }
        }
        // rejection only where it wins clearly: a class timed alone does not carry the rejection
        // kernels' cost to the rest of the batch (on 10^6 tables of 1..64 items, classes whose
        // two timings were within 1.2% chose rejection and the batch took 7.58 ms, 7.10 ms as
        // all alias)
        choice[c] = ms_of[1] < kRejectionWins * ms_of[0] ? (uint8_t)WRS_TABLE_REJECTION : (uint8_t)WRS_TABLE_ALIAS;
        if (class_ms) {
            class_ms[2 * c] = ms_of[0];
            class_ms[2 * c + 1] = ms_of[1];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (result != WRS_SUCCESS) return result;
    for (int64_t t = 0; t < num_tables; ++t)
        h_kinds_out[t] = cls[(size_t)t] < 0 ? (uint8_t)WRS_TABLE_SKIP : choice[cls[(size_t)t]];
    if (class_kinds)
        for (int c = 0; c < kClasses; ++c) class_kinds[c] = choice[c];
    return WRS_SUCCESS;
}
