// precision_kernels.cuh — the all-FP64 and all-FP32 comparison builds (WRS_PRECISION_FP64,
// WRS_PRECISION_FP32).
//
// The default build (build_kernels.cuh, split_kernels.cuh) keeps the deficit and excess lines
// in exact fixed point and only the stored probabilities in FP32. These builds run the same
// merge of the two lines with every quantity in one floating-point type R, as the reference's
// build does in FP64 (TableStorage.cuh:8-11, AliasTableSplitGpu.cu:406-432): the weight total
// W, W/N, each light's deficit W/N - w and each heavy's excess w - W/N, and their prefix sums,
// are R values rounded at every operation. Light i (w <= W/N) aliases the first heavy whose
// excess end E_j exceeds its deficit start A_i; heavy j keeps r_j = W/N + E_j - A_next (A_next:
// the deficit start of the first light with A > ... >= E_j, or the line's total) and aliases
// heavy j + 1. Stored probabilities are w / (W/N) and r_j / (W/N) in R, rounded to FP32 and
// clamped to [0, 1]. The rounding of the lines is what the precision comparison measures.
//
// Summation order (deterministic, restated by the CPU oracle). The weight total: a tile is 256
// threads x 8 consecutive items; a thread sums its items in order, each warp's 32 thread sums
// in lane order, the 8 warp sums in order; over tiles, thread c of one 1024-thread CTA sums tiles
// [c K, (c + 1) K) in order (K = ceil(tiles / 1024)) and thread 0 sums the 1024 chunk sums in
// order. The two lines: each tile's deficits (excesses) are summed in item order by one thread,
// the tiles' bases by one thread in tile order (b_{t+1} = b_t + total_t), and an item's line
// position is b_t + (its tile-local prefix). Since rounding is monotone, the lines never
// decrease, which the merge's partition relies on.
#pragma once

#include <cstdint>

#include "build_kernels.cuh"

namespace wrs {

constexpr int kPrecThreads = 256;
constexpr int kPrecIpt = 8;
constexpr int kPrecTile = kPrecThreads * kPrecIpt;
constexpr int kPrecScanThreads = 1024;

// Per-tile sums of the comparison builds.
template <typename R>
struct PrecTile {
    uint32_t nL, nH;
    R sL;  // light deficits (or, in the weight pass, the weights)
    R sH;  // heavy excesses
};

// Exclusive prefix of one value per thread of a 256-thread CTA in the order above; returns
// the thread's exclusive prefix, `total` gets the CTA's sum. s needs 8 x 33 entries.
template <typename R>
__device__ __forceinline__ R prec_block_scan(R v, R* s, R& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s[warp * 33 + lane] = v;
    __syncthreads();
    if (lane == 0) {
        R acc = (R)0;
        for (int l = 0; l < 32; ++l) {
            const R t = s[warp * 33 + l];
            s[warp * 33 + l] = acc;
            acc = acc + t;
        }
        s[warp * 33 + 32] = acc;  // the warp's total
    }
    __syncthreads();
    __shared__ R s_wbase[kPrecThreads / 32 + 1];
    if (threadIdx.x == 0) {
        R acc = (R)0;
        for (int w = 0; w < kPrecThreads / 32; ++w) {
            s_wbase[w] = acc;
            acc = acc + s[w * 33 + 32];
        }
        s_wbase[kPrecThreads / 32] = acc;
    }
    __syncthreads();
    const R ex = s_wbase[warp] + s[warp * 33 + lane];
    total = s_wbase[kPrecThreads / 32];
    __syncthreads();  // s is reused by the caller's next scan
    return ex;
}
// The items of thread `tid` in tile `tile` (items past n read as -1).
__device__ __forceinline__ void prec_load(const float* __restrict__ w, uint64_t n, uint32_t tile, float (&x)[kPrecIpt]) {
    load_items<kPrecThreads, kPrecIpt>(w, n, tile, threadIdx.x, x);
}

// Pass 1: per tile, the sum of its weights in R (and the invalid-weight check).
template <typename R>
__global__ void __launch_bounds__(kPrecThreads) prec_weight_tiles_kernel(const float* __restrict__ w, uint64_t n,
                                                                         BuildHeader* hdr, PrecTile<R>* tiles) {
    __shared__ R s[8 * 33];
    float x[kPrecIpt];
    prec_load(w, n, blockIdx.x, x);
    R acc = (R)0;
    bool bad = false;
#pragma unroll
    for (int k = 0; k < kPrecIpt; ++k) {
        const uint64_t i = (uint64_t)blockIdx.x * kPrecTile + (uint64_t)threadIdx.x * kPrecIpt + k;
        if (i < n) {
            bad |= weight_invalid(x[k]);
            acc = acc + (R)x[k];
        }
    }
    if (bad) record_status(&hdr->status, kErrInvalidWeight);
    R total;
    prec_block_scan<R>(acc, s, total);
    if (threadIdx.x == 0) {
        PrecTile<R> t;
        t.nL = 0;
        t.nH = 0;
        t.sL = total;
        t.sH = (R)0;
        tiles[blockIdx.x] = t;
    }
}

// One CTA: the weight total W from the tiles' weight sums, in the order above; W and
// W/N = W / n into the header (W_hi, W_N as doubles; exact for R = float) and d_W.
template <typename R>
__global__ void __launch_bounds__(kPrecScanThreads) prec_weight_total_kernel(BuildHeader* hdr,
                                                                             const PrecTile<R>* tiles,
                                                                             uint32_t num_tiles, uint64_t n,
                                                                             double* W_out) {
    __shared__ R s_l[kPrecScanThreads];
    const uint32_t K = (num_tiles + kPrecScanThreads - 1) / kPrecScanThreads;
    const uint32_t t0 = threadIdx.x * K, t1 = min(num_tiles, t0 + K);
    R al = (R)0;
    for (uint32_t t = t0; t < t1; ++t) al = al + tiles[t].sL;
    s_l[threadIdx.x] = al;
    __syncthreads();
    if (threadIdx.x != 0) return;
    R W = (R)0;
    for (int c = 0; c < kPrecScanThreads; ++c) W = W + s_l[c];
    const R W_N = W / (R)(double)n;
    hdr->W_hi = (double)W;
    hdr->W_lo = 0.0;
    hdr->W_N = (double)W_N;
    if (W_out) *W_out = (double)W;
    if (!(W > (R)0) || isinf((double)W)) record_status(&hdr->status, isinf((double)W) ? kErrInvalidWeight : kErrZeroTotal);
}

// The classification against W/N (in R): light w <= W/N, deficit W/N - w; heavy w > W/N,
// excess w - W/N.
template <typename R>
struct PrecItem {
    bool valid, heavy;
    R q;  // deficit (light) or excess (heavy)
};
template <typename R>
__device__ __forceinline__ PrecItem<R> prec_item(float wf, R W_N) {
    PrecItem<R> it;
    const R wr = (R)wf;
    it.valid = wf >= 0.0f;
    it.heavy = it.valid && wr > W_N;
    it.q = it.heavy ? wr - W_N : W_N - wr;
    return it;
}

// Pass 2 (SCATTER false) / pass 4 (SCATTER true): one thread per tile of kPrecTile items, in item
// order. Pass 2 writes the tile's light and heavy counts and its deficit and excess sums; pass 4
// writes each light's deficit start b + (local prefix, exclusive) and probability, and each
// heavy's excess end b + (local prefix, inclusive), at its global light / heavy index.
template <typename R, bool SCATTER>
__global__ void __launch_bounds__(128) prec_lines_kernel(const float* __restrict__ w, uint64_t n,
                                                         const BuildHeader* hdr, PrecTile<R>* tiles,
                                                         const PrecTile<R>* prefix, uint32_t num_tiles,
                                                         R* __restrict__ Lkey, uint32_t* __restrict__ Litem,
                                                         float* __restrict__ Lprob, R* __restrict__ Hkey,
                                                         uint32_t* __restrict__ Hitem) {
    const uint32_t tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= num_tiles) return;
    if (earlier_status(hdr) != 0) return;
    const R W_N = (R)__ldg(&hdr->W_N);
    const uint64_t i0 = (uint64_t)tile * kPrecTile;
    const uint64_t i1 = min(n, i0 + kPrecTile);
    R sl = (R)0, sh = (R)0;
    uint64_t gl = 0, gh = 0;
    R bl = (R)0, bh = (R)0;
    if (SCATTER) {
        const PrecTile<R> b = prefix[tile];
        bl = b.sL;
        bh = b.sH;
        gl = b.nL;
        gh = b.nH;
    }
    uint32_t cl = 0, ch = 0;
    for (uint64_t i = i0; i < i1; ++i) {
        const float wf = __ldg(w + i);
        const PrecItem<R> it = prec_item<R>(wf, W_N);
        if (!it.valid) continue;
        if (it.heavy) {
            sh = sh + it.q;
            if (SCATTER) {
                if (gh < n) {
                    Hkey[gh] = bh + sh;
                    Hitem[gh] = (uint32_t)i;
                }
                ++gh;
            }
            ++ch;
        } else {
            if (SCATTER) {
                if (gl < n) {
                    Lkey[gl] = bl + sl;
                    Litem[gl] = (uint32_t)i;
                    Lprob[gl] = (float)min((R)1, (R)wf / W_N);
                }
                ++gl;
            }
            sl = sl + it.q;
            ++cl;
        }
    }
    if (!SCATTER) {
        PrecTile<R> t;
        t.nL = cl;
        t.nH = ch;
        t.sL = sl;
        t.sH = sh;
        tiles[tile] = t;
    }
}

// One thread: the tiles' bases of the two lines in tile order (b_{t+1} = b_t + total_t) and the
// light / heavy counts before each tile; prefix[num_tiles] gets the totals.
template <typename R>
__global__ void prec_line_bases_kernel(BuildHeader* hdr, const PrecTile<R>* tiles, PrecTile<R>* prefix,
                                       uint32_t num_tiles) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (earlier_status(hdr) != 0) return;
    PrecTile<R> b;
    b.nL = 0;
    b.nH = 0;
    b.sL = (R)0;
    b.sH = (R)0;
    for (uint32_t t = 0; t < num_tiles; ++t) {
        const PrecTile<R> v = tiles[t];
        prefix[t] = b;
        b.nL += v.nL;
        b.nH += v.nH;
        b.sL = b.sL + v.sL;
        b.sH = b.sH + v.sH;
    }
    prefix[num_tiles] = b;
    hdr->nH_total = b.nH;
}

// Pass 5: the merge. Merged order: heavy j comes before light i iff E_j <= A_i. Thread t takes
// merged positions [t C, t C + C): a binary search for the number of lights among the first
// t C positions (the merge-path co-rank), then C merge steps. A light's row: its probability
// and the first heavy not before it (the last heavy past the end); a heavy's row: r = W/N +
// E_j - A_next over W/N (A_next: the first light after it, or the deficit line's total) and
// the next heavy (itself for the last).
constexpr int kPrecMergeChunk = 16;
template <typename R>
__global__ void __launch_bounds__(256) prec_merge_kernel(const BuildHeader* hdr, const PrecTile<R>* totals,
                                                         const R* __restrict__ Lkey,
                                                         const uint32_t* __restrict__ Litem,
                                                         const float* __restrict__ Lprob,
                                                         const R* __restrict__ Hkey,
                                                         const uint32_t* __restrict__ Hitem, uint64_t n,
                                                         wrs_alias_row* __restrict__ table) {
    if (earlier_status(hdr) != 0) return;
    const PrecTile<R> tot = *totals;
    const uint64_t nL = tot.nL, nH = tot.nH;
    const uint64_t M = nL + nH;
    const uint64_t d0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * kPrecMergeChunk;
    if (d0 >= M || nL > n || nH > n) return;
    const R W_N = (R)__ldg(&hdr->W_N);
    const R A_total = tot.sL;
    // co-rank: i lights and d0 - i heavies before position d0; heavy j before light i iff
    // Hkey[j] <= Lkey[i]
    uint64_t lo = d0 > nH ? d0 - nH : 0, hi = min(d0, nL);
    while (lo < hi) {
        const uint64_t i = (lo + hi) >> 1;  // candidate: i lights taken, j = d0 - i heavies
        const uint64_t j = d0 - i;
        // too few lights taken if light i comes before heavy j - 1
        if (j > 0 && Lkey[i] < Hkey[j - 1]) lo = i + 1; else hi = i;
    }
    uint64_t i = lo, j = d0 - lo;
    const uint64_t d1 = min(M, d0 + kPrecMergeChunk);
    for (uint64_t d = d0; d < d1; ++d) {
        const bool take_heavy = j < nH && (i >= nL || Hkey[j] <= Lkey[i]);
        wrs_alias_row r;
        if (take_heavy) {
            const R A_next = i < nL ? Lkey[i] : A_total;
            const R rr = (W_N + Hkey[j] - A_next) / W_N;
            r.prob = (float)max((R)0, min((R)1, rr));
            r.alias = Hitem[j + 1 < nH ? j + 1 : j];
            const uint32_t item = Hitem[j];
            if (item < n) table[item] = r;
            ++j;
        } else {
            r.prob = Lprob[i];
            const uint32_t item = Litem[i];
            r.alias = nH ? Hitem[j < nH ? j : nH - 1] : item;
            if (item < n) table[item] = r;
            ++i;
        }
    }
}

}  // namespace wrs
