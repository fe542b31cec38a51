// batched_kernels.cuh — the batched (CSR) alias build and sampler for sm_100a.
//
// The reference has no batched form: its experiment drivers build many tables by looping
// over AliasTableSplitGpu objects, one build() (several launches, device-to-host copies and
// allocations) per table (construction/aliasTable/buildMethod/AliasTableSplitGpu.cu:388-468).
// Here a whole CSR batch is built by a fixed sequence of launches that depends only on the
// batch's shape, so it can be captured in a CUDA graph:
//   * small tables (n <= small_max, at most 32 * SPL items) are built one per warp by a
//     persistent kernel, everything in registers and shared memory;
//   * larger tables go through the tiled passes of the single-table build, run once over
//     the tiles of all of them (tile_reduce, heavy_list, tile_link, split_pack with
//     BATCH = true), with per-table weight totals and tile prefixes from the kernels below.
// Both produce, for every table, exactly the rows a single-table build of its weights gives.
// The plan (which tables are large, their tiles) is computed on the device from the CSR
// offsets by three small kernels.
#pragma once

#include "build_kernels.cuh"

namespace wrs {

// ---------------------------------------------------------------- planning
// A table is "large" when small_max < n. Planning block pb covers tables
// [pb * kPlanBlock, (pb + 1) * kPlanBlock): plan_count counts its large tables, their tiles
// and their items, plan_scan turns the counts into offsets, plan_fill writes the TableDesc
// of every large table and the table of every global tile. Totals that differ from the
// host's plan (made from its copy of the offsets) are reported as WRS_ERR_INVALID_ARGUMENT
// in the plan status, and the batched passes then do nothing.
constexpr int kPlanBlock = 1024;

// Per-table method of a mixed batch (kinds[t]; a null kinds array means every table is an
// alias table). The alias passes build only WRS_TABLE_ALIAS tables, the rejection passes only
// WRS_TABLE_REJECTION ones; a table of any other kind is skipped by both.
__device__ __forceinline__ bool kind_is(const uint8_t* kinds, int64_t t, uint8_t k) {
    return kinds ? __ldg(kinds + t) == k : k == WRS_TABLE_ALIAS;
}

struct PlanCounts {
    uint32_t tables;
    uint32_t tiles;
    uint64_t items;
};
__device__ __forceinline__ PlanCounts pc_add(const PlanCounts& a, const PlanCounts& b) {
    return PlanCounts{a.tables + b.tables, a.tiles + b.tiles, a.items + b.items};
}
__device__ __forceinline__ PlanCounts pc_sub(const PlanCounts& a, const PlanCounts& b) {
    return PlanCounts{a.tables - b.tables, a.tiles - b.tiles, a.items - b.items};
}
__device__ __forceinline__ PlanCounts pc_shfl_up(const PlanCounts& v, int d) {
    return PlanCounts{__shfl_up_sync(0xffffffffu, v.tables, d), __shfl_up_sync(0xffffffffu, v.tiles, d),
                      __shfl_up_sync(0xffffffffu, v.items, d)};
}
__device__ __forceinline__ PlanCounts pc_shfl(const PlanCounts& v, int src) {
    return PlanCounts{__shfl_sync(0xffffffffu, v.tables, src), __shfl_sync(0xffffffffu, v.tiles, src),
                      __shfl_sync(0xffffffffu, v.items, src)};
}
static_assert(kPlanBlock == 32 * 32, "one scan slot per lane");
// Exclusive scan over a kPlanBlock-thread CTA; *total gets the CTA total. Ends with a barrier.
__device__ __forceinline__ PlanCounts pc_block_scan(const PlanCounts v, PlanCounts* s, PlanCounts* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PlanCounts inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const PlanCounts o = pc_shfl_up(inc, off);
        if (lane >= off) inc = pc_add(inc, o);
    }
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    PlanCounts t = s[lane];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const PlanCounts o = pc_shfl_up(t, off);
        if (lane >= off) t = pc_add(t, o);
    }
    *total = pc_shfl(t, 31);
    const PlanCounts zero{0u, 0u, 0ull};
    const PlanCounts base = pc_shfl(t, warp > 0 ? warp - 1 : 0);
    __syncthreads();
    return pc_sub(pc_add(warp ? base : zero, inc), v);
}

__device__ __forceinline__ PlanCounts plan_of(const int64_t* offsets, const uint8_t* kinds, int64_t num_tables,
                                             int64_t t, uint32_t small_max, uint32_t tile_items, int64_t* n_out) {
    PlanCounts c{0u, 0u, 0ull};
    int64_t n = 0;
    if (t < num_tables && kind_is(kinds, t, WRS_TABLE_ALIAS)) {
        n = offsets[t + 1] - offsets[t];
        if (n > (int64_t)small_max) c = PlanCounts{1u, (uint32_t)((n + tile_items - 1) / tile_items), (uint64_t)n};
    }
    *n_out = n;
    return c;
}

__global__ void __launch_bounds__(kPlanBlock) plan_count_kernel(const int64_t* __restrict__ offsets,
                                                               const uint8_t* kinds, int64_t num_tables,
                                                               uint32_t small_max,
                                                               uint32_t tile_items, PlanCounts* blk) {
    pdl_enter();
    __shared__ PlanCounts s[32];
    int64_t n;
    const PlanCounts c =
        plan_of(offsets, kinds, num_tables, (int64_t)blockIdx.x * kPlanBlock + threadIdx.x, small_max, tile_items, &n);
    PlanCounts tot;
    pc_block_scan(c, s, &tot);
    if (threadIdx.x == 0) blk[blockIdx.x] = tot;
}

// One CTA: exclusive scan of the block counts (in place), in chunks of kPlanBlock; checks
// the totals against the host's plan.
__global__ void __launch_bounds__(kPlanBlock) plan_scan_kernel(PlanCounts* blk, uint32_t num_blk, PlanCounts cap,
                                                              uint32_t* plan_status) {
    pdl_enter();
    __shared__ PlanCounts s[32];
    PlanCounts carry{0u, 0u, 0ull};
    for (uint32_t c = 0; c < num_blk; c += kPlanBlock) {
        const uint32_t i = c + threadIdx.x;
        const PlanCounts v = i < num_blk ? blk[i] : PlanCounts{0u, 0u, 0ull};
        PlanCounts tot;
        const PlanCounts ex = pc_block_scan(v, s, &tot);
        if (i < num_blk) blk[i] = pc_add(carry, ex);
        carry = pc_add(carry, tot);
    }
    if (threadIdx.x == 0 && (carry.tables != cap.tables || carry.tiles != cap.tiles || carry.items != cap.items))
        record_status(plan_status, WRS_ERR_INVALID_ARGUMENT);
}

__global__ void __launch_bounds__(kPlanBlock) plan_fill_kernel(const int64_t* __restrict__ offsets,
                                                              const uint8_t* kinds, int64_t num_tables,
                                                              uint32_t small_max,
                                                              uint32_t tile_items, const PlanCounts* blk,
                                                              PlanCounts cap, TableDesc* desc, uint32_t* tile_table) {
    pdl_enter();
    __shared__ PlanCounts s[32];
    const int64_t t = (int64_t)blockIdx.x * kPlanBlock + threadIdx.x;
    int64_t n;
    const PlanCounts c = plan_of(offsets, kinds, num_tables, t, small_max, tile_items, &n);
    PlanCounts tot;
    const PlanCounts ex = pc_add(blk[blockIdx.x], pc_block_scan(c, s, &tot));
    if (c.tables == 0) return;
    // a plan that does not fit the host's capacities is reported by plan_scan_kernel
    if (ex.tables >= cap.tables || ex.tiles + c.tiles > cap.tiles || ex.items + c.items > cap.items) return;
    TableDesc d;
    d.item_off = (uint64_t)offsets[t];
    d.n = (uint64_t)n;
    d.heavy_off = ex.items;
    d.tile0 = ex.tiles;
    d.ntiles = c.tiles;
    d.id = (uint32_t)t;
    d.pad = 0;
    desc[ex.tables] = d;
    for (uint32_t k = 0; k < c.tiles; ++k) tile_table[ex.tiles + k] = ex.tables;
}

// ---------------------------------------------------------------- large tables: W
// One CTA per global tile sums its items (double-double, the partial goes to partials[g]);
// the last CTA of each table (ticket in the table's header) combines the table's partials
// in tile order and fills the header as wsum_kernel does for a single table.
constexpr int kBatchWsumThreads = 256;

template <int T>
__global__ void __launch_bounds__(kBatchWsumThreads) batch_wsum_kernel(const float* __restrict__ w,
                                                                       BuildHeader* hdrs, double2* partials,
                                                                       TileMap map, double* W_out) {
    pdl_enter();
    constexpr int NT = kBatchWsumThreads;
    const uint32_t g = blockIdx.x;
    if (plan_failed<true>(map)) return;
    const TileRef tr = tile_ref<true>(map, g);
    BuildHeader* hdr = hdrs + tr.table;
    const float* wt = w + tr.item_off;
    const uint64_t i0 = (uint64_t)tr.local * T, i1 = min(tr.n, i0 + T);
    DD acc = {0.0, 0.0};
    bool bad = false;
    for (uint64_t i = i0 + threadIdx.x; i < i1; i += NT) {
        const float x = __ldg(wt + i);
        bad |= weight_invalid(x);
        acc = dd_add_d(acc, (double)x);
    }
    if (bad) record_status(&hdr->status, kErrInvalidWeight);
    __shared__ DD s_part[NT / 32];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    acc = dd_norm(acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        DD o;
        o.hi = __shfl_down_sync(0xffffffffu, acc.hi, off);
        o.lo = __shfl_down_sync(0xffffffffu, acc.lo, off);
        acc = dd_add(acc, o);
    }
    if (lane == 0) s_part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD t = s_part[0];
        for (int i = 1; i < NT / 32; ++i) t = dd_add(t, s_part[i]);
        partials[g] = make_double2(t.hi, t.lo);
        __threadfence();
        const uint32_t ticket = atomicAdd(&hdr->wsum_ticket, 1u);
        s_last = (ticket == tr.ntiles - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    DD t = {0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < tr.ntiles; i += NT) {
        const double2 p = __ldcg(partials + tr.tile0 + i);
        const DD pd = {p.x, p.y};
        t = dd_add(t, pd);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        DD o;
        o.hi = __shfl_down_sync(0xffffffffu, t.hi, off);
        o.lo = __shfl_down_sync(0xffffffffu, t.lo, off);
        t = dd_add(t, o);
    }
    __syncthreads();
    if (lane == 0) s_part[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD r = s_part[0];
        for (int i = 1; i < NT / 32; ++i) r = dd_add(r, s_part[i]);
        r = dd_norm(r);
        hdr->W_hi = r.hi;
        hdr->W_lo = r.lo;
        const double W_N = r.hi / (double)tr.n;
        hdr->W_N = W_N;
        hdr->R = 1.0 / W_N;
        const ClassParams cp = class_params(W_N, 1.0 / W_N);
        hdr->R32 = cp.R32;
        hdr->H1 = cp.H1;
        hdr->Hh = cp.Hh;
        if (W_out) W_out[map.desc[tr.table].id] = r.hi;
        if (!(r.hi > 0.0) || isinf(r.hi)) record_status(&hdr->status, isinf(r.hi) ? kErrInvalidWeight : kErrZeroTotal);
    }
}

// ---------------------------------------------------------------- large tables: tile prefixes
// One CTA per large table: inclusive prefixes of its tiles' aggregates (chunks of
// kPrefixTiles tiles with a carry), and the table's excess correction.
__global__ void __launch_bounds__(kPrefixThreads) batch_prefix_kernel(BuildHeader* hdrs, const TileVals* agg,
                                                                     TileVals* incl, const TableDesc* desc,
                                                                     const uint32_t* plan_status) {
    pdl_enter();
    __shared__ PVals s_warp[kPrefixThreads / 32];
    if (__ldg(plan_status) != 0) return;
    const TableDesc d = desc[blockIdx.x];
    BuildHeader* hdr = hdrs + blockIdx.x;
    if (load_relaxed(&hdr->status) != 0) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PVals carry = pv_zero();
    for (uint32_t c = 0; c < d.ntiles; c += kPrefixTiles) {
        const uint32_t t0 = c + threadIdx.x * kPrefixPerThread;
        PVals loc[kPrefixPerThread];
        PVals run = pv_zero();
#pragma unroll
        for (int k = 0; k < kPrefixPerThread; ++k) {
            const PVals v = (t0 + k < d.ntiles) ? pv_of(agg[d.tile0 + t0 + k]) : pv_zero();
            run = pv_add(run, v);
            loc[k] = run;
        }
        PVals inc = run;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const PVals o = pv_shfl_up(inc, off);
            if (lane >= off) inc = pv_add(inc, o);
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        PVals base = carry, tot = carry;
        for (int i = 0; i < kPrefixThreads / 32; ++i) {
            const PVals t = s_warp[i];
            if (i < warp) base = pv_add(base, t);
            tot = pv_add(tot, t);
        }
        base = pv_add(base, inc);
        base.nL -= run.nL;
        base.nH -= run.nH;
        base.S -= run.S;
        base.L -= run.L;
        base.E -= run.E;
#pragma unroll
        for (int k = 0; k < kPrefixPerThread; ++k) {
            if (t0 + k >= d.ntiles) break;
            const PVals v = pv_add(base, loc[k]);
            TileVals o;
            o.nL = v.nL;
            o.nH = v.nH;
            o.first_heavy = 0xffffffffu;
            o.last_heavy = 0xffffffffu;
            o.S = v.S;
            o.L = v.L;
            o.E = v.E;
            incl[d.tile0 + t0 + k] = o;
            if (t0 + k == d.ntiles - 1) hdr->nfix = excess_correction(v.S + q_round24(v.L), v.E);
        }
        carry = tot;
        __syncthreads();
    }
}

// The first error of any large table's build (or of the plan) goes to the batch status word.
__global__ void batch_status_kernel(const BuildHeader* hdrs, uint32_t num_tables, uint32_t* status) {
    pdl_enter();
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < num_tables; b += gridDim.x * blockDim.x) {
        const uint32_t st = hdrs[b].status;
        if (st != 0) record_status(status, st);
    }
}

// ---------------------------------------------------------------- small tables: a lane group each
// The whole build of a table of n <= GW * SPL items in one group of GW lanes (GW = 32: a warp
// per table; GW = 2 .. 16: 32 / GW tables per warp, for the tiny tables that dominate skewed
// batches). Lane l of the group holds the ipl = ceil(n / GW) consecutive items l * ipl ..; the
// quantities are those of the tiled passes for a one-tile table (A_before = 0, no dithering
// offset), so the rows equal a single-table build's. Shared memory per group: light keys from
// the front and heavy keys from the back of one u64 array, and the heavies' corrected excess
// ends and items.
//
// Size classes: n <= 4, 8, 16, 32 by groups of 2, 4, 8, 16 lanes with two items a lane; n <= 64
// by a warp with two items a lane; the rest (up to small_max) by a warp with small_max / 32
// items a lane. Tables above small_max and up to kMediumMax items are built by a CTA each in
// shared memory (medium_tables_kernel; lists 6 and 7 by CTA size), larger ones by the tiled passes.
// table_lists_kernel lists the batch's small and medium tables per class (appending with one
// atomic per CTA and class: the order within a list is arbitrary, the rows do not depend on it),
// and one launch per class builds its list.
constexpr int kSmallClasses = 6;
constexpr int kLists = 8;
constexpr int64_t kMediumSplit = 2048;  // medium tables up to this size: CTAs of 256 threads
constexpr int64_t kMediumMax = 8192;    // the rest: CTAs of 1024 threads
__host__ __device__ __forceinline__ int small_class(int64_t n) {
    return n <= 4 ? 0 : n <= 8 ? 1 : n <= 16 ? 2 : n <= 32 ? 3 : n <= 64 ? 4 : 5;
}
// List of an alias table of n >= 1 items, or -1 for the tiled passes.
__host__ __device__ __forceinline__ int table_list(int64_t n, uint32_t small_max) {
    if (n <= (int64_t)small_max) return small_class(n);
    if (n <= kMediumSplit) return 6;
    if (n <= kMediumMax) return 7;
    return -1;
}

// The batch header (the first header of the batch scratch, zeroed before every build) seen as
// the batch status word and the fill counters of the lists.
struct BatchCounters {
    uint32_t status;
    uint32_t list_fill[kLists];
    uint32_t spill_fill;                    // build and sample: tables left to the chunked sampler
    unsigned long long list_items[kLists];  // items of each list's tables
    unsigned long long table_sum;           // sum over listed tables of (t + 1) * n_t (mod 2^64)
    unsigned long long chunks;              // build and sample: chunks of the chunked sampler
};
static_assert(sizeof(BatchCounters) <= sizeof(BuildHeader) && offsetof(BatchCounters, status) == 0,
              "batch counters overlay the batch header");

struct TableLists {
    BatchCounters* cnt;        // fill counters and checks, zero at the start
    uint32_t* list;            // table ids; list c at [base[c], base[c] + cap[c])
    uint32_t base[kLists];
    uint32_t cap[kLists];      // the host's count of the list
    uint64_t items[kLists];    // the host's items of the list
    uint64_t table_sum;        // the host's sum of (t + 1) * n_t over listed tables
};

// One thread per table; positions come from a shared-memory counter per list and CTA, then one
// global atomic per list and CTA reserves the CTA's run of each list. The CTAs also add up the
// items of each list and a position-weighted table sum, which lists_check_kernel compares with
// the host's plan (offsets that differ from the host's copy are an error, as in the tiled passes).
constexpr int kListThreads = 1024;
__global__ void __launch_bounds__(kListThreads) table_lists_kernel(const int64_t* __restrict__ offsets,
                                                                  const uint8_t* kinds, int64_t num_tables,
                                                                  uint32_t small_max, TableLists L,
                                                                  uint32_t* status,
                                                                  const int64_t* __restrict__ sample_offsets,
                                                                  uint32_t* spill, uint32_t spill_cap) {
    __shared__ uint32_t s_cnt[kLists], s_base[kLists], s_items[kLists];
    __shared__ unsigned long long s_tsum;
    const int64_t t = (int64_t)blockIdx.x * kListThreads + threadIdx.x;
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < kLists) {
        s_cnt[threadIdx.x] = 0;
        s_items[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) s_tsum = 0;
    __syncthreads();
    int cls = -1;
    uint32_t n32 = 0;
    if (t < num_tables && kind_is(kinds, t, WRS_TABLE_ALIAS)) {
        const int64_t n = __ldg(offsets + t + 1) - __ldg(offsets + t);
        if (n >= 1) cls = table_list(n, small_max);
        if (cls >= 0) n32 = (uint32_t)n;  // <= kMediumMax
        // build and sample: an empty table with samples goes to the chunked sampler (which
        // reports it)
        if (n == 0 && sample_offsets && __ldg(sample_offsets + t + 1) != __ldg(sample_offsets + t)) {
            const uint32_t k = atomicAdd(&L.cnt->spill_fill, 1u);
            if (k < spill_cap) spill[k] = (uint32_t)t;
            else record_status(status, WRS_ERR_INVALID_ARGUMENT);
        }
    }
    uint32_t pos = 0;
#pragma unroll
    for (int c = 0; c < kLists; ++c) {
        const uint32_t m = __ballot_sync(0xffffffffu, cls == c);
        if (m == 0) continue;
        const uint32_t items = __reduce_add_sync(0xffffffffu, cls == c ? n32 : 0u);
        const int leader = __ffs(m) - 1;
        uint32_t b = 0;
        if (lane == leader) {
            b = atomicAdd(s_cnt + c, (uint32_t)__popc(m));
            atomicAdd(s_items + c, items);
        }
        b = __shfl_sync(0xffffffffu, b, leader);
        if (cls == c) pos = b + (uint32_t)__popc(m & ((1u << lane) - 1u));
    }
    unsigned long long ts = cls >= 0 ? (unsigned long long)(t + 1) * n32 : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ts += __shfl_down_sync(0xffffffffu, ts, o);
    if (lane == 0 && ts) atomicAdd(&s_tsum, ts);
    __syncthreads();
    if (threadIdx.x < kLists && s_cnt[threadIdx.x] > 0) {
        s_base[threadIdx.x] = atomicAdd(L.cnt->list_fill + threadIdx.x, s_cnt[threadIdx.x]);
        atomicAdd(L.cnt->list_items + threadIdx.x, (unsigned long long)s_items[threadIdx.x]);
    }
    if (threadIdx.x == 0 && s_tsum) atomicAdd(&L.cnt->table_sum, s_tsum);
    __syncthreads();
    if (cls >= 0) {
        pos += s_base[cls];
        // more tables of a list than the host counted: offsets differ from the host's
        if (pos < L.cap[cls]) L.list[L.base[cls] + pos] = (uint32_t)t;
        else record_status(status, WRS_ERR_INVALID_ARGUMENT);
    }
}

// After table_lists_kernel: the lists against the host's plan.
__global__ void lists_check_kernel(TableLists L, uint32_t* status) {
    const int c = threadIdx.x;
    bool bad = false;
    if (c < kLists) bad = L.cnt->list_fill[c] != L.cap[c] || L.cnt->list_items[c] != L.items[c];
    if (c == 0) bad |= L.cnt->table_sum != (unsigned long long)L.table_sum;
    if (__any_sync(0xffffffffu, bad) && c == 0) record_status(status, WRS_ERR_INVALID_ARGUMENT);
}

constexpr int kSmallWarps = 4;

template <int SPL, int GW = 32>
struct SmallSmem {
    static constexpr int CAP = GW * SPL;
    uint64_t key[CAP];
    uint64_t elo[CAP];
    uint32_t ehi[CAP];
    uint32_t item[CAP];
};

// Exclusive scans over a group of GW lanes (width GW shuffles); `total` gets the group's sum.
template <int GW>
__device__ __forceinline__ uint32_t group_excl_scan_u32(uint32_t v, uint32_t mask, uint32_t& total) {
    const int gl = threadIdx.x & (GW - 1);
    uint32_t inc = v;
#pragma unroll
    for (int off = 1; off < GW; off <<= 1) {
        const uint32_t o = __shfl_up_sync(mask, inc, off, GW);
        if (gl >= off) inc += o;
    }
    total = __shfl_sync(mask, inc, GW - 1, GW);
    return inc - v;
}
template <int GW>
__device__ __forceinline__ uint64_t group_excl_scan_u64(uint64_t v, uint32_t mask, uint64_t& total) {
    const int gl = threadIdx.x & (GW - 1);
    uint64_t inc = v;
#pragma unroll
    for (int off = 1; off < GW; off <<= 1) {
        const uint64_t o = __shfl_up_sync(mask, inc, off, GW);
        if (gl >= off) inc += o;
    }
    total = __shfl_sync(mask, inc, GW - 1, GW);
    return inc - v;
}

// One table of n items (1 <= n <= GW * SPL) by the group of GW lanes in `mask` (gl = the
// lane's index in the group), with the group's shared memory `sm`.
template <int SPL, int GW>
__device__ __forceinline__ void small_table_build(const float* __restrict__ w, int64_t off, uint32_t n, int64_t t,
                                                  uint32_t mask, int gl, SmallSmem<SPL, GW>& sm,
                                                  wrs_alias_row* __restrict__ table, double* W_out,
                                                  uint32_t* status) {
    constexpr int CAP = GW * SPL;
    const uint32_t ipl = (n + GW - 1) / GW;
    const float* wt = w + off;
    wrs_alias_row* rows = table + off;
    const uint32_t i0 = (uint32_t)gl * ipl;
    float x[SPL];
    DD acc = {0.0, 0.0};
    bool bad = false;
#pragma unroll
    for (int k = 0; k < SPL; ++k) {
        const uint32_t i = i0 + k;
        const bool in = (uint32_t)k < ipl && i < n;
        x[k] = in ? __ldg(wt + i) : -1.0f;
        if (in) {
            bad |= weight_invalid(x[k]);
            acc = dd_add_d(acc, (double)x[k]);
        }
    }
    acc = dd_norm(acc);
#pragma unroll
    for (int o = GW / 2; o > 0; o >>= 1) {
        DD v;
        v.hi = __shfl_down_sync(mask, acc.hi, o, GW);
        v.lo = __shfl_down_sync(mask, acc.lo, o, GW);
        acc = dd_add(acc, v);
    }
    acc = dd_norm(acc);
    const double W = __shfl_sync(mask, acc.hi, 0, GW);
    const bool any_bad = __any_sync(mask, bad);
    if (any_bad || !(W > 0.0) || isinf(W)) {
        if (gl == 0) record_status(status, (any_bad || isinf(W)) ? kErrInvalidWeight : kErrZeroTotal);
        return;
    }
    if (gl == 0 && W_out) W_out[t] = W;
    const double W_N = W / (double)n;
    const ClassParams cp = class_params(W_N, 1.0 / W_N);
    // classification and per-lane sums
    float pk[SPL];
    uint32_t lbits = 0, hbits = 0, gbits = 0;
    uint64_t S = 0, L = 0, E = 0;
#pragma unroll
    for (int k = 0; k < SPL; ++k) {
        const float wk = x[k];
        const bool heavy = wk > cp.H1;
        const bool small = wk >= 0.0f && wk < cp.Hh;
        const bool large = wk >= cp.Hh && !heavy;
        const float p = __fmul_rn(wk, cp.R32);
        pk[k] = p;
        lbits |= (uint32_t)(small || large) << k;
        hbits |= (uint32_t)heavy << k;
        gbits |= (uint32_t)large << k;
        if (small) S += small_deficit(p);
        if (large) L += rare_q(wk, false, cp);
        if (heavy) E += rare_q(wk, true, cp);
    }
    uint32_t nl_tot, nh_tot;
    const uint32_t l0 = group_excl_scan_u32<GW>((uint32_t)__popc(lbits), mask, nl_tot);
    const uint32_t h0 = group_excl_scan_u32<GW>((uint32_t)__popc(hbits), mask, nh_tot);
    uint64_t S_tot, L_tot, E_tot;
    const uint64_t s0 = group_excl_scan_u64<GW>(S, mask, S_tot);
    const uint64_t lq0 = group_excl_scan_u64<GW>(L, mask, L_tot);
    const uint64_t e0 = group_excl_scan_u64<GW>(E, mask, E_tot);
    const u128 A_tot = ((u128)S_tot << 16) + q_round24((u128)L_tot << 16);
    const int64_t nfix = excess_correction(A_tot, (u128)E_tot << 40);
    Dither dth;
    dth.c0 = 1ull << 23;
    dth.c0h = 0;
    // keys: lights from the front, heavies from the back (CAP - nh_tot + j)
    {
        uint64_t sr = s0, lr = lq0, er = e0;
        uint64_t D = dither_at(dth, lr);
        uint32_t li = l0, hj = h0;
#pragma unroll
        for (int k = 0; k < SPL; ++k) {
            const float wk = x[k];
            if ((lbits >> k) & 1u) {
                sm.key[li++] = sr + D;
                if ((gbits >> k) & 1u) {
                    lr += rare_q(wk, false, cp);
                    const uint64_t D1 = dither_at(dth, lr);
                    pk[k] = dithered_prob(D1 - D);
                    D = D1;
                } else {
                    sr += small_deficit(pk[k]);
                }
            } else if ((hbits >> k) & 1u) {
                er += rare_q(wk, true, cp);
                const u128 Et = q_scale_excess((u128)er << 40, nfix);
                const u128 d = Et + 0xffff;
                sm.key[CAP - nh_tot + hj] = (q_hi(d) >> 16) ? ~0ull : (uint64_t)(d >> 16);
                sm.elo[hj] = q_lo(Et);
                sm.ehi[hj] = (uint32_t)q_hi(Et);
                sm.item[hj] = i0 + k;
                ++hj;
            }
        }
    }
    __syncwarp(mask);
    const uint64_t* hkey = sm.key + (CAP - nh_tot);
    // heavy rows
    for (uint32_t j = gl; j < nh_tot; j += GW) {
        const uint64_t kh = hkey[j];
        uint32_t lo = 0, hi = nl_tot;  // rank: the first light whose key is not below kh
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sm.key[mid] < kh) lo = mid + 1; else hi = mid;
        }
        const u128 Et = q_make(sm.ehi[j], sm.elo[j]);
        const u128 A_next = (lo < nl_tot) ? ((u128)sm.key[lo] << 16) : A_tot;
        wrs_alias_row r;
        r.prob = heavy_row_prob(q_one() + Et - A_next);
        r.alias = (j + 1 < nh_tot) ? sm.item[j + 1] : sm.item[j];
        rows[sm.item[j]] = r;
    }
    // light rows: alias = the first heavy whose key exceeds the light's (else the last heavy)
    {
        uint32_t li = l0;
#pragma unroll
        for (int k = 0; k < SPL; ++k) {
            if (!((lbits >> k) & 1u)) continue;
            uint32_t al;
            if (nh_tot == 0) {
                al = i0 + k;
            } else {
                const uint64_t kl = sm.key[li];
                uint32_t lo = 0, hi = nh_tot;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (hkey[mid] > kl) hi = mid; else lo = mid + 1;
                }
                al = sm.item[lo < nh_tot ? lo : nh_tot - 1];
            }
            wrs_alias_row r;
            r.prob = pk[k];
            r.alias = al;
            rows[i0 + k] = r;
            ++li;
        }
    }
    __syncwarp(mask);  // the next table reuses this group's shared memory
}

// The tables of list[0 .. min(cap, *fill)), a group of GW lanes each.
template <int SPL, int GW = 32>
__global__ void __launch_bounds__(32 * kSmallWarps) small_tables_kernel(const float* __restrict__ w,
                                                                       const int64_t* __restrict__ offsets,
                                                                       const uint32_t* __restrict__ list,
                                                                       const uint32_t* fill, uint32_t cap,
                                                                       wrs_alias_row* __restrict__ table,
                                                                       double* W_out, uint32_t* status) {
    static_assert(GW == 32 || GW == 16 || GW == 8 || GW == 4 || GW == 2, "lane group width");
    constexpr int CAP = GW * SPL;
    constexpr int GPW = 32 / GW;  // groups per warp
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane / GW, gl = lane & (GW - 1);
    const uint32_t mask = GW == 32 ? 0xffffffffu : (((1u << GW) - 1u) << (grp * GW));
    SmallSmem<SPL, GW>& sm = reinterpret_cast<SmallSmem<SPL, GW>*>(smem_raw)[warp * GPW + grp];
    const uint32_t count = min(cap, *fill);
    const uint32_t ngroups = gridDim.x * (uint32_t)(kSmallWarps * GPW);
    for (uint32_t e = (blockIdx.x * kSmallWarps + warp) * GPW + grp; e < count; e += ngroups) {
        const int64_t t = __ldg(list + e);
        const int64_t off = __ldg(offsets + t);
        const int64_t n = __ldg(offsets + t + 1) - off;
        if (n < 1 || n > CAP) continue;  // uniform over the group; never for a listed table
        small_table_build<SPL, GW>(w, off, (uint32_t)n, t, mask, gl, sm, table, W_out, status);
    }
}

// ---------------------------------------------------------------- medium tables: a CTA each
// A table of small_max < n <= NS items by one CTA of MT threads with the whole table in shared
// memory (NS = 8 MT): the weights, then the light and heavy keys (lights from the front and
// heavies from the back of one array, like the lane-group build), the heavies' inclusive excess
// prefixes, the light and heavy items (one array, the same way round), the rows' probabilities
// (over the weights) and aliases. Thread k holds the items [k * ipt, (k + 1) * ipt), ipt =
// ceil(n / MT). The quantities are those of a one-tile table over the whole table (A_before = 0,
// no dithering offset), so the rows equal a single-table build's:
//   1. the weights are copied in (coalesced) and summed in double-double, W over the CTA;
//   2. per-thread sums of small-light deficits (Q16.48), large-light deficits (Q16.48), heavy
//      excess (Q40.24) and the light and heavy counts, scanned over the CTA;
//   3. every thread walks its items again from its prefixes: light keys, heavy keys and excess
//      prefixes, items, and the light probabilities;
//   4. the merge of the light keys with the heavy keys (a heavy precedes a light of equal key),
//      cut into equal runs of the merged order by a binary search per thread (merge path): a
//      light's alias is the next heavy in that order (the last heavy when none follows); a
//      heavy's probability is 1 + its corrected excess end - the next light's key (the total
//      deficit when none follows), its alias the next heavy (itself for the last one);
//   5. the rows are written out (coalesced).
constexpr int kMediumItemsPerThread = 8;

template <int MT>
struct MediumRed {
    DD dd[MT / 32];
    uint64_t sc[4][MT / 32];
    double W;
};
// dynamic shared memory of a CTA for tables of up to NS items
template <int MT>
constexpr size_t medium_smem_bytes() {
    constexpr size_t NS = (size_t)MT * kMediumItemsPerThread;
    return sizeof(MediumRed<MT>) + NS * (8 + 8 + 4 + 4 + 4);
}

// Exclusive scan of four u64 values per thread over the CTA; tot gets the CTA's totals.
// Starts and ends with a barrier.
template <int MT>
__device__ __forceinline__ void cta_scan4(uint64_t (&v)[4], uint64_t (&tot)[4], uint64_t (&sc)[4][MT / 32]) {
    constexpr int NW = MT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t inc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        inc[q] = v[q];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t x = __shfl_up_sync(0xffffffffu, inc[q], o);
            if (lane >= o) inc[q] += x;
        }
    }
    __syncthreads();
    if (lane == 31)
#pragma unroll
        for (int q = 0; q < 4; ++q) sc[q][warp] = inc[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint64_t wv = lane < NW ? sc[q][lane] : 0ull;
        uint64_t wi = wv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t x = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += x;
        }
        tot[q] = __shfl_sync(0xffffffffu, wi, 31);
        const uint64_t wbase = __shfl_sync(0xffffffffu, wi - wv, warp);
        v[q] = wbase + inc[q] - v[q];
    }
    __syncthreads();
}

template <int MT>
__device__ __forceinline__ void medium_table_build(const float* __restrict__ w, int64_t off, uint32_t n, int64_t t,
                                                   wrs_alias_row* __restrict__ table, double* W_out,
                                                   uint32_t* status, unsigned char* smem) {
    constexpr int NW = MT / 32;
    constexpr uint32_t NS = (uint32_t)MT * kMediumItemsPerThread;
    MediumRed<MT>& red = *reinterpret_cast<MediumRed<MT>*>(smem);
    uint64_t* key = reinterpret_cast<uint64_t*>(smem + sizeof(MediumRed<MT>));  // lights front, heavies back
    uint64_t* hE = key + NS;                                                    // heavy j: inclusive excess
    float* wp = reinterpret_cast<float*>(hE + NS);                               // weight, then probability
    uint32_t* item = reinterpret_cast<uint32_t*>(wp + NS);                       // lights front, heavies back
    uint32_t* alias = item + NS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float* wt = w + off;
    // 1. weights in, weight total
    DD acc = {0.0, 0.0};
    bool bad = false;
    for (uint32_t i = tid; i < n; i += MT) {
        const float x = __ldg(wt + i);
        wp[i] = x;
        bad |= weight_invalid(x);
        acc = dd_add_d(acc, (double)x);
    }
    acc = dd_norm(acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        DD u;
        u.hi = __shfl_down_sync(0xffffffffu, acc.hi, o);
        u.lo = __shfl_down_sync(0xffffffffu, acc.lo, o);
        acc = dd_add(acc, u);
    }
    if (lane == 0) red.dd[warp] = acc;
    const int any_bad = __syncthreads_or(bad);
    if (warp == 0) {
        DD v = lane < NW ? red.dd[lane] : DD{0.0, 0.0};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            DD u;
            u.hi = __shfl_down_sync(0xffffffffu, v.hi, o);
            u.lo = __shfl_down_sync(0xffffffffu, v.lo, o);
            v = dd_add(v, u);
        }
        if (lane == 0) red.W = dd_norm(v).hi;
    }
    __syncthreads();
    const double W = red.W;
    if (any_bad || !(W > 0.0) || isinf(W)) {  // uniform over the CTA
        if (tid == 0) record_status(status, (any_bad || isinf(W)) ? kErrInvalidWeight : kErrZeroTotal);
        return;
    }
    if (tid == 0 && W_out) W_out[t] = W;
    const double W_N = W / (double)n;
    const ClassParams cp = class_params(W_N, 1.0 / W_N);
    const uint32_t ipt = (n + MT - 1) / MT;
    const uint32_t i0 = min(n, (uint32_t)tid * ipt), i1 = min(n, i0 + ipt);
    // 2. per-thread sums, scanned: S, L, E, lights | heavies << 32
    uint64_t v[4] = {0ull, 0ull, 0ull, 0ull};
    for (uint32_t i = i0; i < i1; ++i) {
        const float x = wp[i];
        if (x > cp.H1) {
            v[2] += rare_q(x, true, cp);
            v[3] += 1ull << 32;
        } else {
            v[3] += 1ull;
            if (x < cp.Hh) v[0] += small_deficit(__fmul_rn(x, cp.R32));
            else v[1] += rare_q(x, false, cp);
        }
    }
    uint64_t tot[4];
    cta_scan4<MT>(v, tot, red.sc);
    const uint32_t nl = (uint32_t)tot[3], nh = (uint32_t)(tot[3] >> 32);
    const u128 A_tot = ((u128)tot[0] << 16) + q_round24((u128)tot[1] << 16);
    const int64_t nfix = excess_correction(A_tot, (u128)tot[2] << 40);
    Dither dth;
    dth.c0 = 1ull << 23;
    dth.c0h = 0;
    uint64_t* hkey = key + (NS - nh);
    uint32_t* hitem = item + (NS - nh);
    // 3. keys, heavy excess prefixes, items, light probabilities
    {
        uint64_t sr = v[0], lr = v[1], er = v[2];
        uint32_t li = (uint32_t)v[3], hj = (uint32_t)(v[3] >> 32);
        uint64_t D = dither_at(dth, lr);
        for (uint32_t i = i0; i < i1; ++i) {
            const float x = wp[i];
            if (x > cp.H1) {
                er += rare_q(x, true, cp);
                const u128 d = q_scale_excess((u128)er << 40, nfix) + 0xffff;
                hkey[hj] = (q_hi(d) >> 16) ? ~0ull : (uint64_t)(d >> 16);
                hE[hj] = er;
                hitem[hj] = i;
                ++hj;
            } else {
                key[li] = sr + D;
                item[li] = i;
                ++li;
                float pk;
                if (x >= cp.Hh) {
                    lr += rare_q(x, false, cp);
                    const uint64_t D1 = dither_at(dth, lr);
                    pk = dithered_prob(D1 - D);
                    D = D1;
                } else {
                    pk = __fmul_rn(x, cp.R32);
                    sr += small_deficit(pk);
                }
                wp[i] = pk;
            }
        }
    }
    __syncthreads();
    // 4. merge path
    {
        const uint32_t M = nl + nh;
        const uint32_t mpt = (M + MT - 1) / MT;
        const uint32_t d0 = min(M, (uint32_t)tid * mpt), d1 = min(M, d0 + mpt);
        uint32_t lo = d0 > nh ? d0 - nh : 0u, hi = min(d0, nl);
        while (lo < hi) {  // lights among the first d0 of the merged order
            const uint32_t mid = (lo + hi) >> 1;
            if (key[mid] < hkey[d0 - 1 - mid]) lo = mid + 1; else hi = mid;
        }
        uint32_t a = lo, b = d0 - lo;
        for (uint32_t k = d0; k < d1; ++k) {
            if (b < nh && (a >= nl || hkey[b] <= key[a])) {
                const u128 Et = q_scale_excess((u128)hE[b] << 40, nfix);
                const u128 A_next = a < nl ? ((u128)key[a] << 16) : A_tot;
                const uint32_t it = hitem[b];
                wp[it] = heavy_row_prob(q_one() + Et - A_next);
                alias[it] = b + 1 < nh ? hitem[b + 1] : it;
                ++b;
            } else {
                const uint32_t it = item[a];
                alias[it] = nh == 0 ? it : hitem[b < nh ? b : nh - 1];
                ++a;
            }
        }
    }
    __syncthreads();
    // 5. rows out
    uint2* rows = reinterpret_cast<uint2*>(table + off);
    for (uint32_t i = tid; i < n; i += MT) rows[i] = make_uint2(__float_as_uint(wp[i]), alias[i]);
}

// The tables of list[0 .. min(cap, *fill)), a CTA each (persistent CTAs over the list).
template <int MT>
__global__ void __launch_bounds__(MT) medium_tables_kernel(const float* __restrict__ w,
                                                         const int64_t* __restrict__ offsets,
                                                         const uint32_t* __restrict__ list, const uint32_t* fill,
                                                         uint32_t cap, wrs_alias_row* __restrict__ table,
                                                         double* W_out, uint32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int64_t NS = (int64_t)MT * kMediumItemsPerThread;
    const uint32_t count = min(cap, *fill);
    for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
        const int64_t t = __ldg(list + e);
        const int64_t off = __ldg(offsets + t);
        const int64_t n = __ldg(offsets + t + 1) - off;
        if (n < 1 || n > NS) continue;  // uniform over the CTA; never for a listed table
        medium_table_build<MT>(w, off, (uint32_t)n, t, table, W_out, status, smem_raw);
        __syncthreads();  // shared memory is reused by the next table
    }
}

// ---------------------------------------------------------------- batched plain sampling
// Output position s of the batch belongs to table t with sample_offsets[t] <= s <
// sample_offsets[t + 1] and follows the plain contract over the global position s:
// Philox counter counter_base + s, row = floor((x1:x0) * n_t / 2^64) (table-local),
// coin = (x2 >> 8) * 2^-24, result = coin < prob[row] ? row : alias[row]. A warp takes
// 32 * kBatchSamplePer consecutive positions, lane l the positions base + 32 k + l, so that every
// store of the warp is one coalesced line. The warp finds the table of its first position by a
// 32-way search of the sample offsets (one load per lane and level); every lane moves forward
// from there (a few single steps, then a binary search over the rest). In an all-alias batch
// the lane first resolves the tables of all its positions, then draws and reads all its rows,
// so that its row reads are in flight together.
// In a mixed batch (kinds not null) a rejection table's positions follow the rejection
// contract instead (rejection_sample_kernel: b = counter_base + s, one try per Philox block,
// a 64-bit slot uniform and the acceptance from the table's own slot range), and the positions of a
// skipped table are left as they are.
constexpr int kBatchSampleThreads = 256;
constexpr int kBatchSamplePer = 8;

// The last table whose sample range starts at or before s, over tables [lo, hi].
__device__ __forceinline__ int64_t batch_table_of(const int64_t* __restrict__ sample_offsets, uint64_t s, int64_t lo,
                                                  int64_t hi) {
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if ((uint64_t)__ldg(sample_offsets + mid) <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The same over all tables, by the whole warp for one position s (uniform over the warp): each
// level splits the range into 32 parts and a ballot picks the last part that starts at or before s.
__device__ __forceinline__ int64_t warp_table_of(const int64_t* __restrict__ sample_offsets, uint64_t s,
                                                 int64_t num_tables, uint32_t lane) {
    int64_t lo = 0, hi = num_tables - 1;
    for (;;) {
        const int64_t step = hi - lo >= 32 ? (hi - lo + 32) >> 5 : 1;
        const int64_t idx = lo + (int64_t)lane * step;
        const bool le = idx <= hi && (uint64_t)__ldg(sample_offsets + idx) <= s;
        const uint32_t m = __ballot_sync(0xffffffffu, le);
        const int j = m ? 31 - __clz(m) : 0;
        lo += (int64_t)j * step;
        if (step == 1) return lo;
        hi = min(hi, lo + step - 1);
    }
}

// Moves lane state (t, s_end_t) forward to the table of position s >= the previous position.
__device__ __forceinline__ void batch_advance(const int64_t* __restrict__ sample_offsets, int64_t num_tables,
                                              uint64_t s, int64_t& t, uint64_t& s_end_t) {
    int steps = 0;
    do {
        ++t;
        s_end_t = (uint64_t)__ldg(sample_offsets + t + 1);
    } while (s >= s_end_t && t + 1 < num_tables && ++steps < 4);
    if (s >= s_end_t && t + 1 < num_tables) {
        t = batch_table_of(sample_offsets, s, t + 1, num_tables - 1);
        s_end_t = (uint64_t)__ldg(sample_offsets + t + 1);
    }
}

__global__ void __launch_bounds__(kBatchSampleThreads) batch_sample_kernel(
    const wrs_alias_row* __restrict__ table, const int64_t* __restrict__ offsets, int64_t num_tables,
    const int64_t* __restrict__ sample_offsets, uint64_t total, uint64_t seed, uint64_t counter_base,
    uint32_t* __restrict__ out, uint32_t* status, const uint8_t* kinds, const uint32_t* __restrict__ A,
    const float* __restrict__ frac, const uint64_t* __restrict__ a_size, uint32_t max_tries) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t wbase = (((uint64_t)blockIdx.x * kBatchSampleThreads + threadIdx.x) >> 5) *
                           (32ull * kBatchSamplePer);
    if (wbase >= total) return;  // uniform over the warp
    int64_t t = warp_table_of(sample_offsets, wbase, num_tables, lane);
    uint64_t s_end_t = (uint64_t)__ldg(sample_offsets + t + 1);
    const uint64_t base = wbase + lane;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    if (!kinds) {
        int64_t offk[kBatchSamplePer];
        uint32_t nk[kBatchSamplePer];
        int64_t off = __ldg(offsets + t);
        uint64_t n = (uint64_t)(__ldg(offsets + t + 1) - off);
#pragma unroll
        for (int k = 0; k < kBatchSamplePer; ++k) {
            const uint64_t s = base + 32ull * k;
            offk[k] = 0;
            nk[k] = 0;  // 0: no sample at s (past the end) or an invalid one
            if (s >= total) continue;
            if (s >= s_end_t && t + 1 < num_tables) {
                batch_advance(sample_offsets, num_tables, s, t, s_end_t);
                off = __ldg(offsets + t);
                n = (uint64_t)(__ldg(offsets + t + 1) - off);
            }
            if (n == 0 || n > 0xffffffffull || s >= s_end_t) {
                out[s] = 0xffffffffu;
                if (status) record_status(status, WRS_ERR_INVALID_ARGUMENT);
                continue;
            }
            offk[k] = off;
            nk[k] = (uint32_t)n;
        }
        uint32_t rowk[kBatchSamplePer];
        float coink[kBatchSamplePer];
        uint2 ek[kBatchSamplePer];
#pragma unroll
        for (int k = 0; k < kBatchSamplePer; ++k) {
            const uint64_t b = counter_base + base + 32ull * k;
            const Philox4 x = philox4x32_10((uint32_t)b, (uint32_t)(b >> 32), 0u, 0u, k0, k1);
            rowk[k] = scale_u64(x.x[0], x.x[1], nk[k]);
            coink[k] = coin24(x.x[2]);
            if (nk[k]) ek[k] = __ldg(reinterpret_cast<const uint2*>(table + offk[k]) + rowk[k]);
        }
#pragma unroll
        for (int k = 0; k < kBatchSamplePer; ++k)
            if (nk[k]) out[base + 32ull * k] = coink[k] < __uint_as_float(ek[k].x) ? rowk[k] : ek[k].y;
        return;
    }
    int64_t off = __ldg(offsets + t);
    uint64_t n = (uint64_t)(__ldg(offsets + t + 1) - off);
    uint8_t kind = __ldg(kinds + t);
    for (int k = 0; k < kBatchSamplePer; ++k) {
        const uint64_t s = base + 32ull * k;
        if (s >= total) break;
        if (s >= s_end_t && t + 1 < num_tables) {
            batch_advance(sample_offsets, num_tables, s, t, s_end_t);
            off = __ldg(offsets + t);
            n = (uint64_t)(__ldg(offsets + t + 1) - off);
            kind = __ldg(kinds + t);
        }
        if (kind != WRS_TABLE_ALIAS && s < s_end_t) {
            if (kind != WRS_TABLE_REJECTION) continue;  // a skipped table
            const uint64_t asz = __ldg(a_size + t);
            if (asz == 0 || asz > 0xffffffffull) {
                out[s] = 0xffffffffu;
                if (status) record_status(status, WRS_ERR_INVALID_ARGUMENT);
                continue;
            }
            const uint32_t* At = A + 2 * off;
            const uint64_t b = counter_base + s;
            uint32_t res = 0xffffffffu;
            for (uint32_t tr = 0; tr < max_tries; ++tr) {
                const Philox4 r = philox4x32_10((uint32_t)b, (uint32_t)(b >> 32), tr, 0x52454a00u, k0, k1);
                const uint32_t xc = r.x[2];
                const uint32_t e = __ldg(At + scale_u64(r.x[0], r.x[1], (uint32_t)asz));
                const uint32_t item = e & 0x7fffffffu;
                if ((e >> 31) == 0u || coin24(xc) < __ldg(frac + off + item)) {
                    res = item;
                    break;
                }
            }
            if (res == 0xffffffffu && status) record_status(status, kErrTooManyTries);
            out[s] = res;
            continue;
        }
        if (n == 0 || n > 0xffffffffull || s >= s_end_t) {
            out[s] = 0xffffffffu;
            if (status) record_status(status, WRS_ERR_INVALID_ARGUMENT);
            continue;
        }
        const uint64_t b = counter_base + s;
        const Philox4 x = philox4x32_10((uint32_t)b, (uint32_t)(b >> 32), 0u, 0u, k0, k1);
        const uint32_t row = scale_u64(x.x[0], x.x[1], (uint32_t)n);
        const uint2 e = __ldg(reinterpret_cast<const uint2*>(table + off) + row);
        out[s] = coin24(x.x[2]) < __uint_as_float(e.x) ? row : e.y;
    }
}

// ---------------------------------------------------------------- build and sample
// wrs_batched_build_sample draws the samples of each list's tables right after the list is
// built, on the list's stream, while the tiled passes still run: list_sample_kernel gives a
// warp to each table of a list (positions so[t] + lane + 32 j, the plain contract over the
// global position, exactly as batch_sample_kernel). A table with more than kListSampleMax
// samples is put on the spill list instead; after all builds, chunks_plan_kernel cuts the
// tiled tables and the spilled ones into chunks of kChunkSamples positions and
// chunk_sample_kernel draws them.
constexpr uint32_t kListSampleMax = 2048;
constexpr uint32_t kChunkSamples = 2048;
constexpr int kChunkThreads = 256;
constexpr int kListSampleWarps = 8;

__device__ __forceinline__ uint32_t alias_sample_at(const uint2* __restrict__ rows, uint32_t n, uint64_t b,
                                                    uint32_t k0, uint32_t k1) {
    const Philox4 x = philox4x32_10((uint32_t)b, (uint32_t)(b >> 32), 0u, 0u, k0, k1);
    const uint32_t row = scale_u64(x.x[0], x.x[1], n);
    const uint2 e = __ldg(rows + row);
    return coin24(x.x[2]) < __uint_as_float(e.x) ? row : e.y;
}

__global__ void __launch_bounds__(32 * kListSampleWarps) list_sample_kernel(
    const wrs_alias_row* __restrict__ table, const int64_t* __restrict__ offsets,
    const int64_t* __restrict__ sample_offsets, const uint32_t* __restrict__ list, const uint32_t* fill,
    uint32_t cap, uint64_t seed, uint64_t counter_base, uint32_t* __restrict__ out, uint32_t* spill,
    uint32_t* spill_fill, uint32_t spill_cap, uint32_t* status) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t count = min(cap, *fill);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const uint32_t nwarps = gridDim.x * kListSampleWarps;
    for (uint32_t e = blockIdx.x * kListSampleWarps + (threadIdx.x >> 5); e < count; e += nwarps) {
        const int64_t t = __ldg(list + e);
        const int64_t s0 = __ldg(sample_offsets + t), s1 = __ldg(sample_offsets + t + 1);
        if (s1 <= s0) {
            if (s1 < s0 && lane == 0) record_status(status, WRS_ERR_INVALID_ARGUMENT);
            continue;
        }
        if (s1 - s0 > (int64_t)kListSampleMax) {  // uniform over the warp
            if (lane == 0) {
                const uint32_t k = atomicAdd(spill_fill, 1u);
                if (k < spill_cap) spill[k] = (uint32_t)t;
                else record_status(status, WRS_ERR_INVALID_ARGUMENT);
            }
            continue;
        }
        const int64_t off = __ldg(offsets + t);
        const uint32_t n = (uint32_t)(__ldg(offsets + t + 1) - off);  // 1 <= n <= kMediumMax: a listed table
        const uint2* rows = reinterpret_cast<const uint2*>(table + off);
        for (int64_t s = s0 + lane; s < s1; s += 32) out[s] = alias_sample_at(rows, n, counter_base + (uint64_t)s, k0, k1);
    }
}

// One CTA: the tiled tables (desc[0 .. num_big)) and the spilled ones (spill[0 .. *spill_fill))
// as one list gen[] with the exclusive prefix of their chunk counts; the total in *chunks. Also
// checks sample_offsets[num_tables] == total.
__global__ void __launch_bounds__(1024) chunks_plan_kernel(const TableDesc* desc, uint32_t num_big,
                                                          const uint32_t* plan_status, const uint32_t* spill,
                                                          const uint32_t* spill_fill, uint32_t spill_cap,
                                                          const int64_t* __restrict__ sample_offsets,
                                                          int64_t num_tables, uint64_t total, uint32_t* gen,
                                                          uint64_t* gen_prefix, unsigned long long* chunks,
                                                          uint32_t* status) {
    __shared__ uint64_t s_warp[32];
    __shared__ uint64_t s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the tiled tables are listed only if their plan held
    const uint32_t nbig = (plan_status && *plan_status) ? 0u : num_big;
    const uint32_t nsp = min(spill_cap, *spill_fill);
    const uint32_t m = nbig + nsp;
    if (threadIdx.x == 0) {
        s_carry = 0;
        if ((uint64_t)__ldg(sample_offsets + num_tables) != total || __ldg(sample_offsets) != 0)
            record_status(status, WRS_ERR_INVALID_ARGUMENT);
    }
    __syncthreads();
    for (uint32_t c0 = 0; c0 < m; c0 += 1024) {
        const uint32_t j = c0 + threadIdx.x;
        uint64_t v = 0;
        if (j < m) {
            const uint32_t t = j < nbig ? desc[j].id : spill[j - nbig];
            gen[j] = t;
            const int64_t cnt = __ldg(sample_offsets + t + 1) - __ldg(sample_offsets + t);
            v = cnt > 0 ? ((uint64_t)cnt + kChunkSamples - 1) / kChunkSamples : 0ull;
        }
        uint64_t inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t x = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += x;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            uint64_t wv = s_warp[lane], wi = wv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t x = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += x;
            }
            s_warp[lane] = wi - wv;
        }
        __syncthreads();
        if (j < m) gen_prefix[j] = s_carry + s_warp[warp] + inc - v;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry += s_warp[31] + inc;  // the last thread's inclusive value
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        gen_prefix[m] = s_carry;
        *chunks = s_carry;
    }
}

// Persistent CTAs over the chunks: chunk c belongs to gen entry j (the last with gen_prefix[j]
// <= c) and covers its positions so[t] + (c - gen_prefix[j]) * kChunkSamples + [0, kChunkSamples).
__global__ void __launch_bounds__(kChunkThreads) chunk_sample_kernel(
    const wrs_alias_row* __restrict__ table, const int64_t* __restrict__ offsets,
    const int64_t* __restrict__ sample_offsets, const uint32_t* __restrict__ gen,
    const uint64_t* __restrict__ gen_prefix, const uint32_t* spill_fill, uint32_t spill_cap,
    const uint32_t* plan_status, uint32_t num_big, const unsigned long long* chunks, uint64_t seed,
    uint64_t counter_base, uint32_t* __restrict__ out, uint32_t* status) {
    const uint32_t nbig = (plan_status && *plan_status) ? 0u : num_big;
    const uint32_t m = nbig + min(spill_cap, *spill_fill);
    const uint64_t nchunks = *chunks;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (uint64_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        uint32_t lo = 0, hi = m - 1;  // m >= 1 when there are chunks
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(gen_prefix + mid) <= c) lo = mid; else hi = mid - 1;
        }
        const int64_t t = __ldg(gen + lo);
        const int64_t s1 = __ldg(sample_offsets + t + 1);
        const int64_t sb = __ldg(sample_offsets + t) + (int64_t)(c - __ldg(gen_prefix + lo)) * kChunkSamples;
        const int64_t se = min(s1, sb + (int64_t)kChunkSamples);
        const int64_t off = __ldg(offsets + t);
        const int64_t n = __ldg(offsets + t + 1) - off;
        if (n <= 0 || n > 0xffffffffll) {  // an empty table with samples
            for (int64_t s = sb + threadIdx.x; s < se; s += kChunkThreads) out[s] = 0xffffffffu;
            if (threadIdx.x == 0) record_status(status, WRS_ERR_INVALID_ARGUMENT);
            continue;
        }
        const uint2* rows = reinterpret_cast<const uint2*>(table + off);
        for (int64_t s = sb + threadIdx.x; s < se; s += kChunkThreads)
            out[s] = alias_sample_at(rows, (uint32_t)n, counter_base + (uint64_t)s, k0, k1);
    }
}

}  // namespace wrs
