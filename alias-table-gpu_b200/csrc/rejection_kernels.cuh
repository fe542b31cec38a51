// rejection_kernels.cuh — rejection-sampling structure build for sm_100a.
//
// Replaces RejectionSampling::build (construction/rejectionSampling/RejectionSampling.cu:26-56)
// and its fillA variants (RejectionSamplingBinarySearch.cu:12-37, RejectionSamplingDirect.cu:12-32).
// Item i owns c_i = floor(n w_i / W) + 1 consecutive slots of A (the reference's
// CalcNumOccurrencesOperator, RejectionSampling.cu:26-33, with the same FP64 expression), so
// |A| <= 2n. The reference sums W on the CPU, runs a CUB inclusive scan, copies |A| to the
// host and fills A by one binary search per slot. Here W comes from the shared compensated
// pass, the slot offsets from a decoupled look-back scan over tiles, and each tile fills its
// own slot range with coalesced stores; items with more than kRejBig slots are deferred to
// a list that a second kernel fills with the whole grid.
#pragma once

#include <cstdint>

#include "build_kernels.cuh"

namespace wrs {

constexpr uint32_t kRejBig = 256;           // items with more slots go to the deferred list
constexpr uint32_t kRejHugeSlots = 1u << 16;  // deferred items above this are filled by the whole grid

struct RejBigEntry {
    uint64_t start;
    uint32_t count;
    uint32_t item;
};

__device__ __forceinline__ uint64_t load_acquire_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void store_release_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Tile look-back words: (flag << 62) | value, flag 1 = aggregate, 2 = inclusive.
template <int IPT>
__global__ void __launch_bounds__(kBuildThreads) rejection_tile_kernel(
    const float* __restrict__ w, uint64_t n, BuildHeader* hdr, uint64_t* tile_words, uint32_t num_tiles,
    uint32_t* __restrict__ A, uint64_t a_capacity, float* __restrict__ frac, RejBigEntry* big_list,
    uint64_t big_capacity, uint64_t* a_size_out, WaitCfg wc) {
    pdl_enter();
    constexpr int T = kBuildThreads * IPT;
    __shared__ uint32_t s_tile;
    __shared__ int s_abort;
    // inclusive prefix of small-item slot counts | exclusive prefix of all slot counts (tile-
    // local); in the staged form the tile's slots themselves
    __shared__ uint32_t s_buf[2 * T];
    uint32_t* s_small_incl = s_buf;
    uint32_t* s_off = s_buf + T;
    __shared__ uint64_t s_warp64[kBuildThreads / 32 + 1];
    __shared__ uint32_t s_warp32[kBuildThreads / 32 + 1];
    __shared__ uint64_t s_base;

    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&hdr->tile_ticket, 1u);
        s_abort = (load_relaxed(&hdr->status) != 0);
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= num_tiles) return;
    const bool publish = tile != wc.hold;  // a held tile (failure-detection tests) publishes nothing
    if (s_abort) {
        if (threadIdx.x == 0 && publish) store_release_u64(&tile_words[tile], (2ull << 62));
        return;
    }
    const double W = hdr->W_hi;
    const double nd = (double)n;
    float x[IPT];
    load_tile_items<IPT>(w, n, tile, threadIdx.x, x);
    const uint64_t item0 = (uint64_t)tile * T + (uint64_t)threadIdx.x * IPT;
    uint32_t cs[IPT];
    uint64_t tsum = 0;
    uint32_t tsmall = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        cs[k] = 0;
        if (x[k] < 0.0f) continue;
        uint32_t c;
        float fr;
        rej_item(x[k], nd, W, c, fr);
        frac[item0 + k] = fr;
        cs[k] = c;
        tsum += c;
        if (c <= kRejBig) tsmall += c;
    }
    // CTA exclusive scans: all slots (u64), small slots (u32)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t inc64 = tsum;
    uint32_t inc32 = tsmall;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint64_t o64 = __shfl_up_sync(0xffffffffu, inc64, off);
        const uint32_t o32 = __shfl_up_sync(0xffffffffu, inc32, off);
        if (lane >= off) {
            inc64 += o64;
            inc32 += o32;
        }
    }
    if (lane == 31) {
        s_warp64[warp] = inc64;
        s_warp32[warp] = inc32;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t a64 = 0;
        uint32_t a32 = 0;
        for (int i = 0; i < kBuildThreads / 32; ++i) {
            const uint64_t t64 = s_warp64[i];
            const uint32_t t32 = s_warp32[i];
            s_warp64[i] = a64;
            s_warp32[i] = a32;
            a64 += t64;
            a32 += t32;
        }
        s_warp64[kBuildThreads / 32] = a64;
        s_warp32[kBuildThreads / 32] = a32;
    }
    __syncthreads();
    const uint64_t ex64 = s_warp64[warp] + inc64 - tsum;
    const uint32_t ex32 = s_warp32[warp] + inc32 - tsmall;
    const uint64_t tile_total = s_warp64[kBuildThreads / 32];
    const uint32_t small_total = s_warp32[kBuildThreads / 32];

    // decoupled look-back on the tile slot totals (single 64-bit words)
    if (threadIdx.x < 32) {
        uint64_t excl = 0;
        if (tile == 0) {
            if (lane == 0 && publish) store_release_u64(&tile_words[0], (2ull << 62) | tile_total);
        } else {
            if (lane == 0 && publish) store_release_u64(&tile_words[tile], (1ull << 62) | tile_total);
            int64_t pred = (int64_t)tile - 1;
            bool timed_out = false;
            const uint64_t t_start = global_ns();
            while (true) {
                const int64_t p = pred - lane;
                uint64_t word = (2ull << 62);
                if (p >= 0) {
                    uint32_t spins = 0;
                    while (((word = load_acquire_u64(&tile_words[p])) >> 62) == 0u) {
                        __nanosleep(32);
                        if ((++spins & 255u) == 0u) {
                            if (wait_expired(t_start, wc) || load_relaxed(&hdr->status) != 0) {
                                timed_out = true;
                                break;
                            }
                        }
                    }
                }
                if (__any_sync(0xffffffffu, timed_out)) {
                    if (lane == 0) record_status(&hdr->status, kErrTimeout);
                    break;
                }
                const bool is_incl = (word >> 62) == 2u;
                const uint32_t mask = __ballot_sync(0xffffffffu, is_incl);
                const int stop = mask ? (__ffs(mask) - 1) : 31;
                uint64_t val = (lane <= stop) ? (word & ((1ull << 62) - 1)) : 0ull;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) val += __shfl_xor_sync(0xffffffffu, val, off);
                excl += val;
                if (mask) break;
                pred -= 32;
            }
            if (lane == 0 && publish) store_release_u64(&tile_words[tile], (2ull << 62) | (excl + tile_total));
        }
        if (lane == 0) {
            s_base = excl;
            if (tile == num_tiles - 1) {
                const uint64_t asz = excl + tile_total;
                hdr->a_size = asz;
                // an array that does not fit reports size 0, so that no sampler reads past it
                if (a_size_out) *a_size_out = (asz > a_capacity) ? 0ull : asz;
                if (asz > a_capacity) record_status(&hdr->status, kErrCapacity);
            }
        }
    }
    // a tile without deferred items and with at most 2T slots is staged: each thread writes its
    // items' slots at their tile offsets, then the tile's slots go out with coalesced stores
    const bool staged = tile_total <= (uint64_t)(2 * T) && (uint64_t)small_total == tile_total;
    if (staged) {
        uint32_t o = (uint32_t)ex64;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint32_t item = (uint32_t)(item0 + k);
            for (uint32_t j = 0; j < cs[k]; ++j) s_buf[o + j] = item | (j == 0 ? 0x80000000u : 0u);
            o += cs[k];
        }
        __syncthreads();
        const uint64_t base = s_base;
        for (uint32_t q = threadIdx.x; q < (uint32_t)tile_total; q += kBuildThreads)
            if (base + q < a_capacity) A[base + q] = s_buf[q];
        return;
    }
    // per-item offsets and the small-slot prefix into shared memory
    {
        uint64_t o = ex64;
        uint32_t so = ex32;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const int li = threadIdx.x * IPT + k;
            s_off[li] = (uint32_t)o;  // tile-local: < 2^32 unless a single tile holds a huge item
            const uint32_t c = cs[k];
            if (c <= kRejBig) so += c;
            s_small_incl[li] = so;
            o += c;
        }
    }
    __syncthreads();
    const uint64_t base = s_base;
    // deferred items
    {
        uint64_t o = ex64;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint32_t c = cs[k];
            if (c > kRejBig) {
                const uint64_t idx = atomicAdd((unsigned long long*)&hdr->big_count, 1ull);
                if (idx < big_capacity) {
                    RejBigEntry e;
                    e.start = base + o;
                    e.count = c;
                    e.item = (uint32_t)(item0 + k);
                    big_list[idx] = e;
                }
            }
            o += c;
        }
    }
    // small items: coalesced fill of their slots; slot q of the tile's small slots belongs to
    // the first item whose inclusive small prefix exceeds q
    for (uint32_t q = threadIdx.x; q < small_total; q += kBuildThreads) {
        uint32_t lo = 0, hi = T - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_small_incl[mid] > q) hi = mid; else lo = mid + 1;
        }
        const uint32_t k = lo;
        const uint32_t first = (k ? s_small_incl[k - 1] : 0u);
        const uint64_t slot = base + s_off[k] + (q - first);
        if (slot < a_capacity) A[slot] = (uint32_t)((uint64_t)tile * T + k) | (q == first ? 0x80000000u : 0u);
    }
}

// Deferred items: a warp per item up to kRejHugeSlots slots; larger ones go to the huge list
// (their index in the deferred list) for rejection_huge_kernel.
__global__ void __launch_bounds__(256) rejection_big_kernel(BuildHeader* hdr, const RejBigEntry* big_list,
                                                            uint64_t big_capacity, uint32_t* __restrict__ A,
                                                            uint64_t a_capacity, uint32_t* huge_idx,
                                                            uint64_t huge_capacity) {
    pdl_enter();
    const uint64_t cnt_raw = hdr->big_count;
    const uint64_t cnt = cnt_raw < big_capacity ? cnt_raw : big_capacity;
    if (cnt == 0) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp_g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t e = warp_g; e < cnt; e += nwarps) {
        const RejBigEntry be = big_list[e];
        if (be.count > kRejHugeSlots) {
            if (lane == 0) {
                const uint64_t h = atomicAdd((unsigned long long*)&hdr->huge_count, 1ull);
                if (h < huge_capacity) huge_idx[h] = (uint32_t)e;
            }
            continue;
        }
        for (uint32_t i = lane; i < be.count; i += 32) {
            const uint64_t slot = be.start + i;
            if (slot < a_capacity) A[slot] = be.item | (i == 0 ? 0x80000000u : 0u);
        }
    }
}

// The huge deferred items (more than kRejHugeSlots slots each, at most 2n / kRejHugeSlots of
// them): each item's slots in chunks of kRejChunk, block b taking chunks b, b + gridDim.x, ...
constexpr uint32_t kRejChunk = 4096;
__global__ void __launch_bounds__(256) rejection_huge_kernel(const BuildHeader* hdr, const RejBigEntry* big_list,
                                                             const uint32_t* huge_idx, uint64_t huge_capacity,
                                                             uint32_t* __restrict__ A, uint64_t a_capacity) {
    pdl_enter();
    const uint64_t cnt_raw = hdr->huge_count;
    const uint64_t cnt = cnt_raw < huge_capacity ? cnt_raw : huge_capacity;
    for (uint64_t h = 0; h < cnt; ++h) {
        const RejBigEntry be = big_list[huge_idx[h]];
        const uint32_t chunks = (be.count + kRejChunk - 1) / kRejChunk;
        for (uint32_t c = blockIdx.x; c < chunks; c += gridDim.x) {
            const uint32_t j1 = min(be.count, (c + 1) * kRejChunk);
            for (uint32_t j = c * kRejChunk + threadIdx.x; j < j1; j += blockDim.x) {
                const uint64_t slot = be.start + j;
                if (slot < a_capacity) A[slot] = be.item | (j == 0 ? 0x80000000u : 0u);
            }
        }
    }
}

}  // namespace wrs
