// batched_rejection_kernels.cuh — rejection structures of the rejection tables of a mixed
// batch (sm_100a).
//
// Each rejection table t gets what wrs_rejection_build_f32 builds for its weights alone
// (RejectionSampling::build + fillA, construction/rejectionSampling/RejectionSampling.cu:26-56):
// W = the correctly rounded sum of its weights, c_i = floor(n w_i / W) + 1 slots for item i
// (the same FP64 expression, rej_item in wrs_common.cuh), the slots in item order, a slot
// holding its table-local item with bit 31 set on the item's first slot, and frac_i = the
// first slot's acceptance. Table t's slots start at A[2 * offsets[t]] (|A_t| <= 2 n_t), its
// acceptances at frac[offsets[t]], and |A_t| goes to a_size[t].
// Tables of up to kRejWarpMax items are built one per warp, larger ones one per CTA; both
// walk the table in rounds (one item per lane, or IPT per thread), scan the slot counts of
// the round and write each item's slots, items with many slots cooperatively.
#pragma once

#include "batched_kernels.cuh"

namespace wrs {

constexpr uint32_t kRejWarpMax = 4096;  // tables up to this many items: one warp each
constexpr int kRejWarps = 4;            // warps per CTA of the warp form
constexpr int kRejBlockThreads = 512;   // CTA form
constexpr int kRejBlockIpt = 4;
constexpr uint32_t kRejLaneSlots = 8;   // items with more slots are written by the whole group

__device__ __forceinline__ uint32_t rej_slot(uint32_t item, uint32_t j) { return item | (j ? 0u : 0x80000000u); }

__global__ void __launch_bounds__(32 * kRejWarps) rej_warp_tables_kernel(const float* __restrict__ w,
                                                                        const int64_t* __restrict__ offsets,
                                                                        const uint8_t* kinds, int64_t num_tables,
                                                                        uint32_t* __restrict__ A,
                                                                        float* __restrict__ frac, uint64_t* a_size,
                                                                        double* W_out, uint32_t* status) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * kRejWarps;
    for (int64_t t = (int64_t)blockIdx.x * kRejWarps + warp; t < num_tables; t += nwarps) {
        const int64_t off = offsets[t];
        const int64_t nn = offsets[t + 1] - off;
        if (nn < 1 || nn > (int64_t)kRejWarpMax || !kind_is(kinds, t, WRS_TABLE_REJECTION)) continue;
        const uint32_t n = (uint32_t)nn;
        const float* wt = w + off;
        DD acc = {0.0, 0.0};
        bool bad = false;
        for (uint32_t i = lane; i < n; i += 32) {
            const float x = __ldg(wt + i);
            bad |= weight_invalid(x);
            acc = dd_add_d(acc, (double)x);
        }
        acc = dd_norm(acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            DD v;
            v.hi = __shfl_down_sync(0xffffffffu, acc.hi, o);
            v.lo = __shfl_down_sync(0xffffffffu, acc.lo, o);
            acc = dd_add(acc, v);
        }
        acc = dd_norm(acc);
        const double W = __shfl_sync(0xffffffffu, acc.hi, 0);
        const bool any_bad = __any_sync(0xffffffffu, bad);
        if (any_bad || !(W > 0.0) || isinf(W)) {
            if (lane == 0) {
                record_status(status, (any_bad || isinf(W)) ? kErrInvalidWeight : kErrZeroTotal);
                a_size[t] = 0;
            }
            continue;
        }
        if (lane == 0 && W_out) W_out[t] = W;
        const double nd = (double)n;
        uint32_t* At = A + 2 * off;
        float* ft = frac + off;
        const uint32_t cap = 2u * n;
        uint32_t base = 0;
        for (uint32_t r = 0; r < n; r += 32) {
            const uint32_t i = r + lane;
            uint32_t c = 0;
            if (i < n) {
                float fr;
                rej_item(__ldg(wt + i), nd, W, c, fr);
                ft[i] = fr;
            }
            uint32_t tot;
            const uint32_t ex = base + warp_excl_scan_u32(c, tot);
            if (c <= kRejLaneSlots)
                for (uint32_t j = 0; j < c; ++j)
                    if (ex + j < cap) At[ex + j] = rej_slot(i, j);
            for (uint32_t big = __ballot_sync(0xffffffffu, c > kRejLaneSlots); big; big &= big - 1) {
                const int src = __ffs(big) - 1;
                const uint32_t cb = __shfl_sync(0xffffffffu, c, src), eb = __shfl_sync(0xffffffffu, ex, src);
                for (uint32_t j = lane; j < cb; j += 32)
                    if (eb + j < cap) At[eb + j] = rej_slot(r + (uint32_t)src, j);
            }
            base += tot;
        }
        if (lane == 0) {
            if (base > cap) record_status(status, kErrCapacity);
            a_size[t] = base > cap ? 0ull : base;
        }
    }
}

// One CTA per rejection table of more than warp_max items (CTAs stride over the tables).
__global__ void __launch_bounds__(kRejBlockThreads) rej_block_tables_kernel(const float* __restrict__ w,
                                                                           const int64_t* __restrict__ offsets,
                                                                           const uint8_t* kinds, int64_t num_tables,
                                                                           uint32_t warp_max, uint32_t* __restrict__ A,
                                                                           float* __restrict__ frac,
                                                                           uint64_t* a_size, double* W_out,
                                                                           uint32_t* status) {
    constexpr int NT = kRejBlockThreads, IPT = kRejBlockIpt, R = NT * IPT;
    __shared__ DD s_dd[NT / 32];
    __shared__ uint32_t s_scan[NT / 32];
    __shared__ double s_W;
    __shared__ int s_bad;
    __shared__ uint32_t s_big_cnt;
    __shared__ uint32_t s_big_pos[R], s_big_c[R], s_big_item[R];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t t = blockIdx.x; t < num_tables; t += gridDim.x) {
        const int64_t off = offsets[t];
        const int64_t nn = offsets[t + 1] - off;
        if (nn <= (int64_t)warp_max || !kind_is(kinds, t, WRS_TABLE_REJECTION)) continue;  // uniform in the CTA
        const uint32_t n = (uint32_t)nn;
        const float* wt = w + off;
        DD acc = {0.0, 0.0};
        bool bad = false;
        for (uint32_t i = tid; i < n; i += NT) {
            const float x = __ldg(wt + i);
            bad |= weight_invalid(x);
            acc = dd_add_d(acc, (double)x);
        }
        acc = dd_norm(acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            DD v;
            v.hi = __shfl_down_sync(0xffffffffu, acc.hi, o);
            v.lo = __shfl_down_sync(0xffffffffu, acc.lo, o);
            acc = dd_add(acc, v);
        }
        const bool wbad = __any_sync(0xffffffffu, bad);
        if (lane == 0) s_dd[warp] = acc;
        if (tid == 0) s_bad = 0;
        __syncthreads();
        if (wbad && lane == 0) s_bad = 1;
        if (tid == 0) {
            DD r = s_dd[0];
            for (int i = 1; i < NT / 32; ++i) r = dd_add(r, s_dd[i]);
            r = dd_norm(r);
            s_W = r.hi;
        }
        __syncthreads();
        const double W = s_W;
        if (s_bad || !(W > 0.0) || isinf(W)) {
            if (tid == 0) {
                record_status(status, (s_bad || isinf(W)) ? kErrInvalidWeight : kErrZeroTotal);
                a_size[t] = 0;
            }
            __syncthreads();
            continue;
        }
        if (tid == 0 && W_out) W_out[t] = W;
        const double nd = (double)n;
        uint32_t* At = A + 2 * off;
        float* ft = frac + off;
        const uint32_t cap = 2u * n;
        uint32_t base = 0;
        for (uint32_t r = 0; r < n; r += R) {
            const uint32_t i0 = r + (uint32_t)tid * IPT;
            uint32_t c[IPT];
            uint32_t cs = 0;
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                c[k] = 0;
                if (i0 + k < n) {
                    float fr;
                    rej_item(__ldg(wt + i0 + k), nd, W, c[k], fr);
                    ft[i0 + k] = fr;
                }
                cs += c[k];
            }
            if (tid == 0) s_big_cnt = 0;
            uint32_t tot;
            uint32_t pos = base + block_scan1<NT, uint32_t>(cs, s_scan, tot);  // barrier inside
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                if (c[k] <= kRejLaneSlots) {
                    for (uint32_t j = 0; j < c[k]; ++j)
                        if (pos + j < cap) At[pos + j] = rej_slot(i0 + k, j);
                } else {
                    const uint32_t b = atomicAdd(&s_big_cnt, 1u);
                    s_big_pos[b] = pos;
                    s_big_c[b] = c[k];
                    s_big_item[b] = i0 + k;
                }
                pos += c[k];
            }
            __syncthreads();
            const uint32_t nb = s_big_cnt;
            for (uint32_t b = 0; b < nb; ++b) {
                const uint32_t p0 = s_big_pos[b], cb = s_big_c[b], item = s_big_item[b];
                for (uint32_t j = tid; j < cb; j += NT)
                    if (p0 + j < cap) At[p0 + j] = rej_slot(item, j);
            }
            __syncthreads();  // the next round rewrites the big list and the scan slots
            base += tot;
        }
        if (tid == 0) {
            if (base > cap) record_status(status, kErrCapacity);
            a_size[t] = base > cap ? 0ull : base;
        }
    }
}

}  // namespace wrs
