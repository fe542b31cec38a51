// build_kernels.cuh — the alias-table build ("split/pack", PSA) for sm_100a.
//
// The reference builds an alias table with the sequential greedy sweep of
// construction/aliasTable/packMethod/PackMethodBasic.cuh:59-126 over light items
// (w <= W/N) and heavy items (w > W/N), both in index order, cut into p independent
// segments by the split search of splitMethod/SplitMethodBasic.cu:14-50 over FP64 prefix
// sums of the light and heavy weights (AliasTableSplitGpu.cu:406-432).
//
// The same sweep, written as a merge. Measure weights in rows (W/N = 1). Light i has
// deficit d_i = 1 - p_i (p_i = its stored probability); heavy j has excess e_j = h_j - 1.
// With A_i = sum_{t<i} d_t (start of light i's deficit interval) and
// E_j = sum_{t<=j} e_t (end of heavy j's excess interval), the sweep's state after i lights
// and j heavies holds residual 1 + E_j - A_i on heavy j, so
//   * light i takes heavy J(i) = #{j : E_j <= A_i} as its alias, and
//   * heavy j becomes a row when the lights run past E_j: with I(j) = #{i : A_i < E_j},
//     its row keeps r_j = 1 + E_j - A_{I(j)} (in (0, 1]) and aliases heavy j + 1.
// The split search of the reference (sigma = prefixL[i] + prefixH[j] <= W*n'/N) is this
// merge's diagonal search; segments here are tiles of the light side.
//
// Exactness. A and E are kept in Q64.64 fixed point (unsigned __int128), so all
// comparisons are exact and agree across CTAs. A heavy's reconstructed probability is
// r_j + sum of its donees' deficits + (1 - r_{j-1}) = 1 + E_j - E_{j-1} = h_j whatever the
// light deficits are, as long as A is built from the deficits actually stored. Two global
// effects remain and are handled explicitly:
//   * Stored light probabilities are FP32. Lights with p >= 1/2 ("large") are dithered:
//     with L_i = exact prefix of their true deficits, the stored deficit is
//     round24(L_i + d_i) - round24(L_i), a multiple of 2^-24 (exact in FP32) within 2^-24 of
//     the true value, and the sum over all large lights stays within 2^-25 of exact.
//     Lights with p < 1/2 ("small") store the nearest FP32.
//   * The remaining mismatch D = A_total - E_total is spread over all heavies in
//     proportion to their excess by the monotone map E -> E + floor(E * N / 2^64),
//     N = round(2^64 * D / E_total) (q_scale_excess), so no single heavy absorbs it.
// Per-item relative error is then below ~2^-23 + |D| / E_total for every input.
//
// Passes: (1) wsum: compensated W; (2) tile_reduce: per-tile counts and sums of the three
// streams (small-light deficits S, large-light true deficits L, heavy excess E);
// (3) tile_prefix: inclusive Q64.64 tile prefixes (block scans chained by a short
// decoupled look-back); (4) tile_link: per light tile, the heavy tiles whose excess range
// covers the tile's deficit range (the split); (5) split_pack: pair the tile's lights with
// those heavies (the pack) and write rows. Tile t owns (writes the row of) every heavy whose corrected
// excess end lies in (A_before(t), A_after(t)]; tile 0's interval is open to the left and
// the last tile's to the right, so every heavy is written exactly once.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "wrs_common.cuh"

namespace wrs {

constexpr int kBuildThreads = 256;

// Per-tile values (aggregate or prefix) of the three Q64.64 streams and the counts.
struct __align__(16) TileVals {
    uint32_t nL;
    uint32_t nH;
    uint32_t first_heavy;  // aggregate only: smallest heavy item of the tile (or ~0)
    uint32_t last_heavy;   // aggregate only: largest heavy item of the tile (or ~0)
    u128 S;  // sum of stored deficits of small lights (p < 1/2)
    u128 L;  // sum of true deficits of large lights (p >= 1/2)
    u128 E;  // sum of heavy excess
};
static_assert(sizeof(TileVals) == 64, "TileVals layout");

__host__ __device__ __forceinline__ TileVals tv_zero() {
    TileVals v;
    v.nL = 0;
    v.nH = 0;
    v.first_heavy = 0xffffffffu;
    v.last_heavy = 0xffffffffu;
    v.S = 0;
    v.L = 0;
    v.E = 0;
    return v;
}
__host__ __device__ __forceinline__ TileVals tv_add(const TileVals& a, const TileVals& b) {
    TileVals r;
    r.nL = a.nL + b.nL;
    r.nH = a.nH + b.nH;
    r.first_heavy = 0xffffffffu;
    r.last_heavy = 0xffffffffu;
    r.S = a.S + b.S;
    r.L = a.L + b.L;
    r.E = a.E + b.E;
    return r;
}

// Header at the start of every build scratch buffer; zeroed before every build.
struct __align__(16) BuildHeader {
    uint32_t status;
    uint32_t wsum_ticket;
    uint32_t tile_ticket;
    uint32_t aux_ticket;
    double W_hi;
    double W_lo;
    double W_N;
    double R;           // 1 / W_N
    uint64_t a_size;    // rejection: |A|
    uint64_t big_count; // rejection: number of deferred large items
    float R32;          // class thresholds (ClassParams), set with W
    float H1;
    float Hh;
    uint32_t nH_total;  // split build: number of heavy items, set by the scan pass
    int64_t nfix;       // excess correction, set with the tile prefixes
    uint64_t huge_count; // rejection: number of deferred items filled by the whole grid
    uint32_t chunk_count; // split build: tiles pack_walk_kernel left to the chunked form
    uint32_t pad1;
    uint32_t pad2;
    uint64_t pad[2];
};
static_assert(sizeof(BuildHeader) == 128, "header layout");

// ---------------------------------------------------------------- classification
// The per-item quantities; every pass that needs them computes them the same way, and the
// CPU oracle restates them operation by operation. Within a tile, light deficits are
// summed as u64 in Q16.48 and heavy excess in Q40.24 (each rounded to nearest, ties to
// even, by one hardware conversion of an exactly scaled value); tile aggregates and
// prefixes are Q64.64. A light's merge key is exact on the 2^-48 grid, so comparisons
// against the (full-resolution) corrected excess line stay exact; the per-item rounding
// only moves a heavy's reconstructed probability by at most (number of donees) x 2^-49 rows.
//
// Classes, with thresholds computed once per build from W/N (ClassParams):
//   heavy        w > H1 (H1 = largest float <= W/N, so exactly w > W/N): excess h - 1,
//                h = w * (N/W) in FP64;
//   large light  Hh <= w <= H1 (Hh = smallest float >= W/(2N)): true deficit 1 - w*(N/W)
//                in FP64, stored probability dithered (see the pack pass);
//   small light  w < Hh: stored probability p = w * fl32(N/W) in FP32 (within 2 ulp of
//                w/(W/N)), deficit 1 - p.
// Large lights and heavies are the "rare" classes: the passes handle them in a second,
// per-thread loop over their bits, so the FP64 path costs work only where it is needed.
struct ClassParams {
    double R;   // N / W
    float R32;  // fl32(R)
    float H1;   // largest float <= W/N
    float Hh;   // smallest float >= W/(2N)
};

__device__ __forceinline__ ClassParams class_params(const double W_N, const double R) {
    ClassParams c;
    c.R = R;
    c.R32 = __double2float_rn(R);
    c.H1 = __double2float_rd(W_N);
    c.Hh = __double2float_ru(__dmul_rn(0.5, W_N));
    return c;
}

// The class thresholds of this build, as the weight-total pass stored them in the header.
// Passes after that one read header fields through the read-only (L1) path: every warp of
// every CTA reads them, and an L2-only load would send all of those reads to one L2 line.
__device__ __forceinline__ ClassParams load_class_params(const BuildHeader* hdr) {
    ClassParams c;
    c.R = __ldg(&hdr->R);
    c.R32 = __ldg(&hdr->R32);
    c.H1 = __ldg(&hdr->H1);
    c.Hh = __ldg(&hdr->Hh);
    return c;
}
// Status left by the earlier passes of this build (set only before this kernel started).
__device__ __forceinline__ uint32_t earlier_status(const BuildHeader* hdr) { return __ldg(&hdr->status); }

constexpr uint64_t kOneQ48 = 1ull << 48;

// Q16.48 deficit of a small light with stored probability p: 2^48 - rne(p * 2^48)
// (p * 2^48 is exact in FP32).
__device__ __forceinline__ uint64_t small_deficit(float p) {
    return kOneQ48 - __float2ull_rn(__fmul_rn(p, 281474976710656.0f));
}

// A rare item's quantity: heavy excess max(h, 1) - 1 in Q40.24, or a large light's true
// deficit 1 - min(h, 1) in Q16.48, with h = w * (N/W) in FP64.
__device__ __forceinline__ uint64_t rare_q(float wf, bool heavy, const ClassParams& cp) {
    const double hd = __dmul_rn((double)wf, cp.R);
    const double v = heavy ? __dsub_rn(fmax(hd, 1.0), 1.0) : __dsub_rn(1.0, fmin(hd, 1.0));
    return __double2ull_rn(__dmul_rn(v, heavy ? 16777216.0 : 281474976710656.0));
}

// Dithering of large lights, in the tile frame. Globally, A_i = S_i + round24(L_i) with S_i,
// L_i the Q64.64 prefixes of small-light deficits and large-light true deficits; a large
// light stores the deficit round24(L_i + d) - round24(L_i), a multiple of 2^-24 (exact in
// FP32). Inside a tile with L_i = L_before + x (x in Q16.48), only the low 40 bits of
// L_before matter: with c0 = ((L_before mod 2^40) >> 16) + 2^23,
//   round24(L_before + x) - round24(L_before) = (((c0 + x) >> 24) - (c0 >> 24)) << 24
// in Q16.48 units, which needs only 64-bit arithmetic.
struct Dither {
    uint64_t c0;
    uint64_t c0h;
};
__device__ __forceinline__ Dither make_dither(u128 L_before) {
    Dither d;
    d.c0 = ((q_lo(L_before) & ((1ull << 40) - 1)) >> 16) + (1ull << 23);
    d.c0h = d.c0 >> 24;
    return d;
}
__device__ __forceinline__ uint64_t dither_at(const Dither& d, uint64_t x) { return (((d.c0 + x) >> 24) - d.c0h) << 24; }
// Stored probability of a large light from the dithered deficit (a multiple of 2^-24).
__device__ __forceinline__ float dithered_prob(uint64_t dd48) {
    const uint32_t units = (uint32_t)(dd48 >> 24);
    return (float)(16777216u - units) * 5.9604644775390625e-8f;
}

// A heavy's row probability from r in Q64.64 (clamped to [0, 1]).
__device__ __forceinline__ float heavy_row_prob(u128 r) {
    if (q_is_negative(r)) return 0.0f;
    if (r >= q_one()) return 1.0f;
    return __double2float_rn(__dmul_rn((double)(q_lo(r) >> 11), 1.1102230246251565404e-16));
}

// Start of the deficit line of everything before a tile prefix.
__device__ __forceinline__ u128 deficit_line(const TileVals& v) { return v.S + q_round24(v.L); }

// ---------------------------------------------------------------- double-double sums
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_add_d(DD a, double x) {
    double s, e;
    two_sum(a.hi, x, s, e);
    a.hi = s;
    a.lo += e;
    return a;
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    e += a.lo + b.lo;
    DD r;
    two_sum(s, e, r.hi, r.lo);
    return r;
}
__device__ __forceinline__ DD dd_norm(DD a) {
    DD r;
    two_sum(a.hi, a.lo, r.hi, r.lo);
    return r;
}

__device__ __forceinline__ bool weight_invalid(float w) {
    return !(w >= 0.0f) || isinf(w);  // NaN, negative, +inf
}

// ---------------------------------------------------------------- pass 1: W
// Every thread accumulates a double-double over a reverse grid-stride walk: the walk
// ends at the front of the array, which the next pass (tiles in ascending ticket order)
// reads first while it is still in L2. The last CTA combines the per-CTA partials in index
// order, so the result does not depend on scheduling. Also zeroes `zero_words` (the
// look-back flags of the next pass).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) wsum_kernel(const float* __restrict__ w, uint64_t n,
                                                     BuildHeader* hdr, double2* partials,
                                                     uint32_t* zero_words, uint64_t num_zero_words,
                                                     double* W_out) {
    pdl_enter();
    const uint64_t gtid = (uint64_t)blockIdx.x * BLOCK + threadIdx.x;
    const uint64_t gsize = (uint64_t)gridDim.x * BLOCK;
    for (uint64_t i = gtid; i < num_zero_words; i += gsize) zero_words[i] = 0u;

    DD acc = {0.0, 0.0};
    bool bad = false;
    const bool aligned = ((uintptr_t)w & 15u) == 0;
    if (aligned) {
        const int64_t n4 = (int64_t)(n >> 2);
        const float4* w4 = reinterpret_cast<const float4*>(w);
        const int64_t gs = (int64_t)gsize;
        int64_t q = n4 - 1 - (int64_t)gtid;
        // four independent 16-byte loads in flight per thread, summed into two accumulators
        DD acc2 = {0.0, 0.0};
        for (; q - 3 * gs >= 0; q -= 4 * gs) {
            float4 v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = __ldg(w4 + q - j * gs);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                bad |= weight_invalid(v[j].x) | weight_invalid(v[j].y) | weight_invalid(v[j].z) |
                       weight_invalid(v[j].w);
                DD& a = (j & 1) ? acc2 : acc;
                a = dd_add_d(a, (double)v[j].x);
                a = dd_add_d(a, (double)v[j].y);
                a = dd_add_d(a, (double)v[j].z);
                a = dd_add_d(a, (double)v[j].w);
            }
        }
        acc = dd_add(acc, acc2);
        for (; q - gs >= 0; q -= 2 * gs) {
            const float4 a = __ldg(w4 + q);
            const float4 b = __ldg(w4 + q - gs);
            bad |= weight_invalid(a.x) | weight_invalid(a.y) | weight_invalid(a.z) | weight_invalid(a.w);
            bad |= weight_invalid(b.x) | weight_invalid(b.y) | weight_invalid(b.z) | weight_invalid(b.w);
            acc = dd_add_d(acc, (double)a.x);
            acc = dd_add_d(acc, (double)a.y);
            acc = dd_add_d(acc, (double)a.z);
            acc = dd_add_d(acc, (double)a.w);
            acc = dd_add_d(acc, (double)b.x);
            acc = dd_add_d(acc, (double)b.y);
            acc = dd_add_d(acc, (double)b.z);
            acc = dd_add_d(acc, (double)b.w);
        }
        if (q >= 0) {
            const float4 a = __ldg(w4 + q);
            bad |= weight_invalid(a.x) | weight_invalid(a.y) | weight_invalid(a.z) | weight_invalid(a.w);
            acc = dd_add_d(acc, (double)a.x);
            acc = dd_add_d(acc, (double)a.y);
            acc = dd_add_d(acc, (double)a.z);
            acc = dd_add_d(acc, (double)a.w);
        }
        for (uint64_t i = ((uint64_t)n4 << 2) + gtid; i < n; i += gsize) {
            const float x = w[i];
            bad |= weight_invalid(x);
            acc = dd_add_d(acc, (double)x);
        }
    } else {
        for (int64_t i = (int64_t)n - 1 - (int64_t)gtid; i >= 0; i -= (int64_t)gsize) {
            const float x = w[i];
            bad |= weight_invalid(x);
            acc = dd_add_d(acc, (double)x);
        }
    }
    if (bad) record_status(&hdr->status, kErrInvalidWeight);

    __shared__ DD s_part[BLOCK / 32];
    __shared__ bool s_last;
    acc = dd_norm(acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        DD o;
        o.hi = __shfl_down_sync(0xffffffffu, acc.hi, off);
        o.lo = __shfl_down_sync(0xffffffffu, acc.lo, off);
        acc = dd_add(acc, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) s_part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD t = s_part[0];
        for (int i = 1; i < BLOCK / 32; ++i) t = dd_add(t, s_part[i]);
        partials[blockIdx.x] = make_double2(t.hi, t.lo);
        __threadfence();
        const uint32_t ticket = atomicAdd(&hdr->wsum_ticket, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    DD t = {0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += BLOCK) {
        const double2 p = __ldcg(partials + i);
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
        for (int i = 1; i < BLOCK / 32; ++i) r = dd_add(r, s_part[i]);
        r = dd_norm(r);
        hdr->W_hi = r.hi;
        hdr->W_lo = r.lo;
        const double W_N = r.hi / (double)n;
        hdr->W_N = W_N;
        hdr->R = 1.0 / W_N;
        const ClassParams cp = class_params(W_N, 1.0 / W_N);
        hdr->R32 = cp.R32;
        hdr->H1 = cp.H1;
        hdr->Hh = cp.Hh;
        if (W_out) *W_out = r.hi;
        if (!(r.hi > 0.0) || isinf(r.hi)) record_status(&hdr->status, isinf(r.hi) ? kErrInvalidWeight : kErrZeroTotal);
        hdr->wsum_ticket = 0u;
    }
}

// ---------------------------------------------------------------- CTA scan helpers
// Exclusive CTA-wide scans. Each warp scans with shuffles, the last lane of every warp
// publishes its total in s[warp], and after one barrier every warp scans the NT/32 totals
// itself (no serial step). The caller must not rewrite s before a barrier that follows all
// reads of it (each scan below gets its own slots).
struct Scan3 {  // a count and two u64 sums
    uint32_t c;
    uint64_t a;
    uint64_t b;
};
__device__ __forceinline__ Scan3 s3_add(const Scan3& x, const Scan3& y) {
    Scan3 r;
    r.c = x.c + y.c;
    r.a = x.a + y.a;
    r.b = x.b + y.b;
    return r;
}
__device__ __forceinline__ Scan3 s3_shfl_up(const Scan3& v, int d) {
    Scan3 o;
    o.c = __shfl_up_sync(0xffffffffu, v.c, d);
    o.a = __shfl_up_sync(0xffffffffu, v.a, d);
    o.b = __shfl_up_sync(0xffffffffu, v.b, d);
    return o;
}
__device__ __forceinline__ Scan3 s3_shfl(const Scan3& v, int src) {
    Scan3 o;
    o.c = __shfl_sync(0xffffffffu, v.c, src);
    o.a = __shfl_sync(0xffffffffu, v.a, src);
    o.b = __shfl_sync(0xffffffffu, v.b, src);
    return o;
}

template <int NT>
__device__ __forceinline__ Scan3 block_scan3(const Scan3 v, Scan3* s, Scan3& total) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Scan3 inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Scan3 o = s3_shfl_up(inc, off);
        if (lane >= off) inc = s3_add(inc, o);
    }
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    Scan3 t = {0u, 0ull, 0ull};
    if (lane < NW) t = s[lane];
#pragma unroll
    for (int off = 1; off < NW; off <<= 1) {
        const Scan3 o = s3_shfl_up(t, off);
        if (lane >= off) t = s3_add(t, o);
    }
    total = s3_shfl(t, NW - 1);
    const Scan3 base = s3_shfl(t, warp > 0 ? warp - 1 : 0);
    Scan3 ex;
    ex.c = (warp ? base.c : 0u) + inc.c - v.c;
    ex.a = (warp ? base.a : 0ull) + inc.a - v.a;
    ex.b = (warp ? base.b : 0ull) + inc.b - v.b;
    return ex;
}

template <int NT, typename U>
__device__ __forceinline__ U block_scan1(const U v, U* s, U& total) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    U inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const U o = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += o;
    }
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    U t = (lane < NW) ? s[lane] : (U)0;
#pragma unroll
    for (int off = 1; off < NW; off <<= 1) {
        const U o = __shfl_up_sync(0xffffffffu, t, off);
        if (lane >= off) t += o;
    }
    total = __shfl_sync(0xffffffffu, t, NW - 1);
    const U base = __shfl_sync(0xffffffffu, t, warp > 0 ? warp - 1 : 0);
    return (warp ? base : (U)0) + inc - v;
}

// The IPT consecutive weights of thread `tid` of an NT-thread CTA in tile `tile`
// (T = NT * IPT items); items past n read as -1.
template <int NT, int IPT>
__device__ __forceinline__ void load_items(const float* __restrict__ w, uint64_t n, uint64_t tile, int tid,
                                           float (&x)[IPT]) {
    constexpr uint64_t T = (uint64_t)NT * IPT;
    const uint64_t base = tile * T + (uint64_t)tid * IPT;
    const bool aligned = ((uintptr_t)w & 15u) == 0;
    if (aligned && base + IPT <= n) {
        const float4* p = reinterpret_cast<const float4*>(w + base);
#pragma unroll
        for (int k = 0; k < IPT / 4; ++k) {
            const float4 v = __ldg(p + k);
            x[4 * k + 0] = v.x;
            x[4 * k + 1] = v.y;
            x[4 * k + 2] = v.z;
            x[4 * k + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < IPT; ++k) x[k] = (base + k < n) ? __ldg(w + base + k) : -1.0f;
    }
}

// The IPT weights of thread `tid` in tile `tile`; items past n read as -1.
template <int IPT>
__device__ __forceinline__ void load_tile_items(const float* __restrict__ w, uint64_t n, uint64_t tile, int tid,
                                                float (&x)[IPT]) {
    constexpr uint64_t T = (uint64_t)kBuildThreads * IPT;
    const uint64_t base = tile * T + (uint64_t)tid * IPT;
    const bool aligned = ((uintptr_t)w & 15u) == 0;
    if (aligned && base + IPT <= n) {
        const float4* p = reinterpret_cast<const float4*>(w + base);
#pragma unroll
        for (int k = 0; k < IPT / 4; ++k) {
            const float4 v = __ldg(p + k);
            x[4 * k + 0] = v.x;
            x[4 * k + 1] = v.y;
            x[4 * k + 2] = v.z;
            x[4 * k + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < IPT; ++k) x[k] = (base + k < n) ? __ldg(w + base + k) : -1.0f;
    }
}

__device__ __forceinline__ TileVals ldcg_tilevals(const TileVals* src) {
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    const uint4 w0 = __ldcg(s4 + 0), w1 = __ldcg(s4 + 1), w2 = __ldcg(s4 + 2), w3 = __ldcg(s4 + 3);
    TileVals v;
    v.nL = w0.x;
    v.nH = w0.y;
    v.first_heavy = w0.z;
    v.last_heavy = w0.w;
    v.S = q_make(((uint64_t)w1.w << 32) | w1.z, ((uint64_t)w1.y << 32) | w1.x);
    v.L = q_make(((uint64_t)w2.w << 32) | w2.z, ((uint64_t)w2.y << 32) | w2.x);
    v.E = q_make(((uint64_t)w3.w << 32) | w3.z, ((uint64_t)w3.y << 32) | w3.x);
    return v;
}

__device__ __forceinline__ u128 ldcg_E(const TileVals* src) {
    const uint4 w3 = __ldcg(reinterpret_cast<const uint4*>(src) + 3);
    return q_make(((uint64_t)w3.w << 32) | w3.z, ((uint64_t)w3.y << 32) | w3.x);
}

// ---------------------------------------------------------------- tile spaces
// The passes work on tiles of T items. A single-table build numbers the tiles of its table
// 0..num_tiles-1. A batched build (many CSR tables) lays the tiles of its multi-tile tables
// end to end: tile_table[g] names the table (its index in the batch's list of such tables)
// of global tile g, and TableDesc places that table in the CSR arrays. Rows, heavy items and
// aliases are table-local; per-table arrays (weights, rows, heavy list) are addressed from
// the table's offsets, per-tile arrays (aggregates, prefixes, masks) by global tile, and the
// tile starts of table b from tile0 + b (a table of k tiles has k + 1 starts).
struct TableDesc {
    uint64_t item_off;   // first item of the table in the CSR arrays
    uint64_t n;          // items
    uint64_t heavy_off;  // first entry of the table's heavy list (the listed tables' items, packed)
    uint32_t tile0;      // first global tile
    uint32_t ntiles;
    uint32_t id;         // the table's index in the CSR offsets
    uint32_t pad;
};
static_assert(sizeof(TableDesc) == 40, "TableDesc layout");
struct TileMap {
    const uint32_t* tile_table;   // batched: list index of every global tile's table
    const TableDesc* desc;        // batched: per listed table
    const uint32_t* plan_status;  // batched: nonzero if the plan does not match the launch
    uint64_t n;                   // single table: items
    uint32_t ntiles;              // single table: tiles
};
struct TileRef {
    uint32_t table;  // list index (0 for a single table)
    uint32_t local;  // tile index within the table
    uint32_t tile0;
    uint32_t ntiles;
    uint64_t item_off;
    uint64_t n;
    uint64_t heavy_off;
};
__device__ __forceinline__ TileRef table_ref(const TableDesc& d, uint32_t table, uint32_t local) {
    TileRef r;
    r.table = table;
    r.local = local;
    r.tile0 = d.tile0;
    r.ntiles = d.ntiles;
    r.item_off = d.item_off;
    r.n = d.n;
    r.heavy_off = d.heavy_off;
    return r;
}
// Batched kernels return at once when the plan is unusable (then tile_table and desc may be
// incomplete); a single table has no plan.
template <bool BATCH>
__device__ __forceinline__ bool plan_failed(const TileMap& map) {
    return BATCH && __ldg(map.plan_status) != 0;
}
template <bool BATCH>
__device__ __forceinline__ TileRef tile_ref(const TileMap& map, uint32_t g) {
    if (BATCH) {
        const uint32_t t = __ldg(map.tile_table + g);
        const TableDesc d = map.desc[t];
        return table_ref(d, t, g - d.tile0);
    }
    TileRef r;
    r.table = 0;
    r.local = g;
    r.tile0 = 0;
    r.ntiles = map.ntiles;
    r.item_off = 0;
    r.n = map.n;
    r.heavy_off = 0;
    return r;
}

// ---------------------------------------------------------------- pass 2: tile reduce
// One tile per CTA: counts and sums of the three streams, the tile's first and last heavy
// item, and its heavy mask (bit i of word i/32 <=> tile item i is heavy). No inter-CTA waits.
constexpr int kReduceThreads = 128;

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

template <int T, bool BATCH>
__global__ void __launch_bounds__(kReduceThreads) tile_reduce_kernel(const float* __restrict__ w,
                                                                     const BuildHeader* hdr, TileVals* agg,
                                                                     uint32_t* __restrict__ hmask, TileMap map) {
    pdl_enter();
    constexpr int IPT = T / kReduceThreads;
    constexpr int NW = kReduceThreads / 32;
    static_assert(IPT >= 4 && IPT <= 32 && (IPT & (IPT - 1)) == 0, "items per thread");
    __shared__ uint32_t s_nl[NW], s_nh[NW], s_fh[NW], s_lh[NW];
    __shared__ uint64_t s_s[NW], s_l[NW], s_e[NW];
    const uint32_t tile = blockIdx.x;  // global tile
    if (plan_failed<BATCH>(map)) return;
    const TileRef tr = tile_ref<BATCH>(map, tile);
    const float* wt = w + tr.item_off;
    float x[IPT];
    load_items<kReduceThreads, IPT>(wt, tr.n, tr.local, threadIdx.x, x);  // first: independent of the header
    hdr += tr.table;
    if (earlier_status(hdr) != 0) return;
    const ClassParams cp = load_class_params(hdr);
    const uint64_t item0 = (uint64_t)tr.local * T + (uint64_t)threadIdx.x * IPT;  // table-local
    uint32_t lbits = 0, sbits = 0, hbits = 0;
    uint64_t S = 0;
    // p * 2^48 = w * (fl32(N/W) * 2^48) exactly while the scaled factor is finite (a power-of-two
    // scaling commutes with rounding); small_deficit(p) = 2^48 - rne(p * 2^48).
    const float R48 = cp.R32 * 281474976710656.0f;
    if ((uint64_t)(tr.local + 1) * T <= tr.n && R48 < __int_as_float(0x7f800000)) {
        // a full tile: every item is present
        uint64_t qsum = 0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const float wk = x[k];
            const bool heavy = wk > cp.H1;
            const bool rare = wk >= cp.Hh;
            const uint64_t qs = __float2ull_rn(__fmul_rn(wk, R48));
            if (!rare) qsum += qs;
            hbits |= (uint32_t)heavy << k;
            sbits |= (uint32_t)!rare << k;
        }
        lbits = ~hbits & (IPT == 32 ? 0xffffffffu : ((1u << IPT) - 1u));
        S = (uint64_t)__popc(sbits) * kOneQ48 - qsum;
    } else {
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const float wk = x[k];
            const bool heavy = wk > cp.H1;
            const bool light = wk >= 0.0f && !heavy;
            const bool small = wk >= 0.0f && wk < cp.Hh;
            const uint64_t d = small_deficit(__fmul_rn(wk, cp.R32));
            S += small ? d : 0ull;
            lbits |= (uint32_t)light << k;
            sbits |= (uint32_t)small << k;
            hbits |= (uint32_t)heavy << k;
        }
    }
    // rare items (large lights and heavies): from the weights in registers when a thread has
    // many (all items predicated), else gathered again from L1 one by one
    uint64_t L = 0, E = 0;
    const uint32_t rbits = (lbits & ~sbits) | hbits;
    if ((uint32_t)__popc(rbits) * 4u > (uint32_t)IPT) {
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if ((rbits >> k) & 1u) {
                const bool heavy = (hbits >> k) & 1u;
                const uint64_t q = rare_q(x[k], heavy, cp);
                E += heavy ? q : 0ull;
                L += heavy ? 0ull : q;
            }
        }
    } else {
        for (uint32_t bits = rbits; bits; bits &= bits - 1) {
            const int k = __ffs(bits) - 1;
            const bool heavy = (hbits >> k) & 1u;
            const uint64_t q = rare_q(__ldg(wt + item0 + k), heavy, cp);
            E += heavy ? q : 0ull;
            L += heavy ? 0ull : q;
        }
    }
    // heavy mask words (32 / IPT lanes per word)
    {
        constexpr int LPW = 32 / IPT;
        uint32_t word = (IPT == 32) ? hbits : (hbits << ((threadIdx.x % LPW) * IPT));
#pragma unroll
        for (int d = 1; d < LPW; d <<= 1) word |= __shfl_xor_sync(0xffffffffu, word, d);
        if (threadIdx.x % LPW == 0) hmask[(uint64_t)tile * (T / 32) + threadIdx.x / LPW] = word;
    }
    const uint32_t nL = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(lbits));
    const uint32_t nH = __reduce_add_sync(0xffffffffu, (uint32_t)__popc(hbits));
    const uint32_t fh = __reduce_min_sync(0xffffffffu, hbits ? (uint32_t)item0 + (uint32_t)(__ffs(hbits) - 1) : 0xffffffffu);
    const uint32_t lh = __reduce_max_sync(0xffffffffu, hbits ? (uint32_t)item0 + 31u - (uint32_t)__clz(hbits) : 0u);
    S = warp_sum_u64(S);
    L = warp_sum_u64(L);
    E = warp_sum_u64(E);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_nl[warp] = nL;
        s_nh[warp] = nH;
        s_fh[warp] = fh;
        s_lh[warp] = lh;
        s_s[warp] = S;
        s_l[warp] = L;
        s_e[warp] = E;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    TileVals a;
    uint32_t tl = 0, th = 0, mf = 0xffffffffu, ml = 0;
    uint64_t ts = 0, tlv = 0, te = 0;
#pragma unroll
    for (int i = 0; i < NW; ++i) {
        tl += s_nl[i];
        th += s_nh[i];
        mf = min(mf, s_fh[i]);
        ml = max(ml, s_lh[i]);
        ts += s_s[i];
        tlv += s_l[i];
        te += s_e[i];
    }
    a.nL = tl;
    a.nH = th;
    a.first_heavy = mf;
    a.last_heavy = th ? ml : 0xffffffffu;
    a.S = (u128)ts << 16;
    a.L = (u128)tlv << 16;
    a.E = (u128)te << 40;
    agg[tile] = a;
}

// ---------------------------------------------------------------- pass 3: tile prefix
// Inclusive prefixes of the tile aggregates: each CTA scans kPrefixTiles consecutive tiles,
// and CTAs chain their totals with a decoupled look-back (at most num_tiles / kPrefixTiles
// CTAs, taken in ticket order; every wait is bounded).
constexpr int kPrefixThreads = 256;
constexpr int kPrefixPerThread = 4;
constexpr int kPrefixTiles = kPrefixThreads * kPrefixPerThread;

struct PVals {
    uint32_t nL, nH;
    u128 S, L, E;
};
__device__ __forceinline__ PVals pv_zero() {
    PVals v;
    v.nL = 0;
    v.nH = 0;
    v.S = 0;
    v.L = 0;
    v.E = 0;
    return v;
}
__device__ __forceinline__ PVals pv_add(const PVals& a, const PVals& b) {
    PVals r;
    r.nL = a.nL + b.nL;
    r.nH = a.nH + b.nH;
    r.S = a.S + b.S;
    r.L = a.L + b.L;
    r.E = a.E + b.E;
    return r;
}
__device__ __forceinline__ PVals pv_of(const TileVals& t) {
    PVals v;
    v.nL = t.nL;
    v.nH = t.nH;
    v.S = t.S;
    v.L = t.L;
    v.E = t.E;
    return v;
}
__device__ __forceinline__ PVals pv_shfl_up(const PVals& v, int d) {
    PVals o;
    o.nL = __shfl_up_sync(0xffffffffu, v.nL, d);
    o.nH = __shfl_up_sync(0xffffffffu, v.nH, d);
    o.S = shfl_up_u128(v.S, d);
    o.L = shfl_up_u128(v.L, d);
    o.E = shfl_up_u128(v.E, d);
    return o;
}
__device__ __forceinline__ PVals pv_shfl_xor(const PVals& v, int d) {
    PVals o;
    o.nL = __shfl_xor_sync(0xffffffffu, v.nL, d);
    o.nH = __shfl_xor_sync(0xffffffffu, v.nH, d);
    o.S = shfl_xor_u128(v.S, d);
    o.L = shfl_xor_u128(v.L, d);
    o.E = shfl_xor_u128(v.E, d);
    return o;
}

struct __align__(16) BlockWord {  // look-back record of one prefix CTA
    uint32_t flag;  // 0 = not ready, 1 = aggregate, 2 = inclusive
    uint32_t pad[3];
    PVals agg;
    PVals incl;
};

static __global__ void __launch_bounds__(kPrefixThreads) tile_prefix_kernel(BuildHeader* hdr, const TileVals* agg,
                                                                     TileVals* incl, BlockWord* blocks,
                                                                     uint32_t num_tiles, WaitCfg wc) {
    pdl_enter();
    __shared__ uint32_t s_blk;
    __shared__ PVals s_warp[kPrefixThreads / 32 + 1];
    __shared__ PVals s_base;
    __shared__ int s_abort;
    if (threadIdx.x == 0) {
        s_blk = atomicAdd(&hdr->aux_ticket, 1u);
        s_abort = load_relaxed(&hdr->status) != 0;
    }
    __syncthreads();
    const uint32_t blk = s_blk;
    const bool publish = blk != wc.hold;  // a held block (failure-detection tests) publishes nothing
    if (s_abort) {
        if (threadIdx.x == 0 && publish) store_release(&blocks[blk].flag, 2u);
        return;
    }
    const uint32_t t0 = blk * kPrefixTiles + threadIdx.x * kPrefixPerThread;
    PVals loc[kPrefixPerThread];
    PVals run = pv_zero();
#pragma unroll
    for (int k = 0; k < kPrefixPerThread; ++k) {
        const PVals v = (t0 + k < num_tiles) ? pv_of(agg[t0 + k]) : pv_zero();
        run = pv_add(run, v);
        loc[k] = run;  // thread-local inclusive
    }
    // CTA exclusive scan of the thread totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PVals inc = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const PVals o = pv_shfl_up(inc, d);
        if (lane >= d) inc = pv_add(inc, o);
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        PVals acc = pv_zero();
        for (int i = 0; i < kPrefixThreads / 32; ++i) {
            const PVals t = s_warp[i];
            s_warp[i] = acc;
            acc = pv_add(acc, t);
        }
        s_warp[kPrefixThreads / 32] = acc;
    }
    __syncthreads();
    PVals texcl = pv_add(s_warp[warp], inc);
    texcl.nL -= run.nL;
    texcl.nH -= run.nH;
    texcl.S -= run.S;
    texcl.L -= run.L;
    texcl.E -= run.E;
    const PVals btot = s_warp[kPrefixThreads / 32];
    // look-back over the preceding prefix CTAs (warp 0)
    if (warp == 0) {
        PVals excl = pv_zero();
        if (blk == 0) {
            if (lane == 0 && publish) {
                blocks[0].agg = btot;
                blocks[0].incl = btot;
                store_release(&blocks[0].flag, 2u);
            }
        } else {
            if (lane == 0 && publish) {
                blocks[blk].agg = btot;
                store_release(&blocks[blk].flag, 1u);
            }
            int64_t pred = (int64_t)blk - 1;
            bool timed_out = false;
            const uint64_t t_start = global_ns();
            while (true) {
                const int64_t p = pred - lane;
                uint32_t fl = 2u;
                PVals pv = pv_zero();
                if (p >= 0) {
                    uint32_t spins = 0;
                    while ((fl = load_acquire(&blocks[p].flag)) == 0u) {
                        __nanosleep(20);
                        if ((++spins & 255u) == 0u) {
                            if (wait_expired(t_start, wc) || load_relaxed(&hdr->status) != 0) {
                                timed_out = true;
                                break;
                            }
                        }
                    }
                    if (!timed_out) {
                        const PVals* src = (fl == 2u) ? &blocks[p].incl : &blocks[p].agg;
                        pv.nL = __ldcg(&src->nL);
                        pv.nH = __ldcg(&src->nH);
                        const uint4* q4 = reinterpret_cast<const uint4*>(&src->S);
                        for (int i = 0; i < 3; ++i) {
                            const uint4 v = __ldcg(q4 + i);
                            const u128 x = q_make(((uint64_t)v.w << 32) | v.z, ((uint64_t)v.y << 32) | v.x);
                            if (i == 0) pv.S = x; else if (i == 1) pv.L = x; else pv.E = x;
                        }
                    }
                }
                if (__any_sync(0xffffffffu, timed_out)) {
                    if (lane == 0) record_status(&hdr->status, kErrTimeout);
                    break;
                }
                const uint32_t incl_mask = __ballot_sync(0xffffffffu, fl == 2u);
                const int stop = incl_mask ? (__ffs(incl_mask) - 1) : 31;
                if (lane > stop) pv = pv_zero();
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) pv = pv_add(pv, pv_shfl_xor(pv, d));
                excl = pv_add(excl, pv);
                if (incl_mask) break;
                pred -= 32;
            }
            if (lane == 0 && publish) {
                blocks[blk].incl = pv_add(excl, btot);
                store_release(&blocks[blk].flag, 2u);
            }
        }
        if (lane == 0) s_base = excl;
    }
    __syncthreads();
    const PVals base = pv_add(s_base, texcl);
#pragma unroll
    for (int k = 0; k < kPrefixPerThread; ++k) {
        if (t0 + k >= num_tiles) break;
        const PVals v = pv_add(base, loc[k]);
        TileVals o;
        o.nL = v.nL;
        o.nH = v.nH;
        o.first_heavy = 0xffffffffu;
        o.last_heavy = 0xffffffffu;
        o.S = v.S;
        o.L = v.L;
        o.E = v.E;
        incl[t0 + k] = o;
        if (t0 + k == num_tiles - 1) hdr->nfix = excess_correction(v.S + q_round24(v.L), v.E);
    }
}

// Slot of entry i of a shared array that each thread fills at consecutive indices from a
// scanned start (the light keys of a pack tile, a heavy-list segment): the low four index
// bits XOR the next four. The threads of a warp start about a thread's item count apart, so
// without the XOR every lane's store would fall into the same bank (pair).
__device__ __forceinline__ uint32_t lkey_slot(uint32_t i) { return i ^ ((i >> 4) & 15u); }

// ---------------------------------------------------------------- pass 4: heavy list
// One tile per warp: the tile's heavies in item order (expanded from its heavy mask), their
// excess (weights gathered again), and their corrected excess ends E~ (Q64.64), written at
// their global heavy index g: heavy_item[g], heavy_E[g]. The list is sorted by E~.
__device__ __forceinline__ void store_u128(uint4* p, u128 v) {
    const uint64_t lo = q_lo(v), hi = q_hi(v);
    *p = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
}
__device__ __forceinline__ u128 load_u128(const uint4* p) {
    const uint4 v = __ldcg(p);
    return q_make(((uint64_t)v.w << 32) | v.z, ((uint64_t)v.y << 32) | v.x);
}

// Tiles (warps) per CTA of the heavy-list pass.
__host__ __device__ constexpr int heavy_warps(int) { return 4; }

// Items per segment of the heavy-list pass (16 per lane).
constexpr int kHeavySeg = 512;
// Heavies in a lane's 16 items from which it loads all of their weights at once.
constexpr int kDenseLane = 4;

// A warp's staging of one segment's heavies in heavy order: the within-tile inclusive excess
// prefix (Q40.24) and the item's offset in the segment, at swizzled slots (lkey_slot).
struct HeavyStage {
    uint64_t er[kHeavySeg];
    uint16_t off[kHeavySeg];
};

__device__ __forceinline__ uint32_t warp_excl_scan_u32(uint32_t v, uint32_t& total) {
    const int lane = threadIdx.x & 31;
    uint32_t inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += o;
    }
    total = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
}
__device__ __forceinline__ uint64_t warp_excl_scan_u64(uint64_t v, uint64_t& total) {
    const int lane = threadIdx.x & 31;
    uint64_t inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint64_t o = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += o;
    }
    total = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
}

template <int T, bool BATCH>
__global__ void __launch_bounds__(32 * heavy_warps(T)) heavy_list_kernel(const float* __restrict__ w,
                                                                      const BuildHeader* hdr, const TileVals* agg,
                                                                      const TileVals* incl,
                                                                      const uint32_t* __restrict__ hmask,
                                                                      uint32_t num_tiles, uint32_t* heavy_item,
                                                                      uint4* heavy_E, TileMap map) {
    pdl_enter();
    constexpr int WPT = T / 32;    // mask words per tile
    constexpr int WPL = WPT / 32;  // sparse form: lane l owns tile items [l*32*WPL, (l+1)*32*WPL)
    static_assert(WPL >= 1 && WPL <= 4, "mask words per lane");
    constexpr int NSEG = T / kHeavySeg;
    constexpr int NWARP = heavy_warps(T);
    __shared__ HeavyStage stage[NWARP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t u = blockIdx.x * NWARP + warp;  // global tile
    if (u >= num_tiles || plan_failed<BATCH>(map)) return;
    const TileRef tr = tile_ref<BATCH>(map, u);
    hdr += tr.table;
    if (earlier_status(hdr) != 0) return;
    const uint32_t m = __ldcg(&agg[u].nH);
    if (m == 0) return;
    const float* wt = w + tr.item_off;
    heavy_item += tr.heavy_off;
    heavy_E += tr.heavy_off;
    const ClassParams cp = load_class_params(hdr);
    const int64_t nfix = __ldg(&hdr->nfix);
    const uint32_t g0 = tr.local ? __ldcg(&incl[u - 1].nH) : 0u;
    const u128 Eb = tr.local ? ldcg_E(incl + u - 1) : (u128)0;
    if (m * 8u <= (uint32_t)T) {
        // sparse tile: each lane walks its own items twice around the warp's prefixes and
        // writes its heavies directly
        uint32_t wd[WPL];
#pragma unroll
        for (int i = 0; i < WPL; ++i) wd[i] = __ldg(hmask + (uint64_t)u * WPT + lane * WPL + i);
        const uint32_t ibase = tr.local * (uint32_t)T + (uint32_t)lane * WPL * 32u;
        uint32_t c = 0;
        uint64_t hs = 0;
#pragma unroll
        for (int i = 0; i < WPL; ++i) {
            c += (uint32_t)__popc(wd[i]);
            for (uint32_t b = wd[i]; b; b &= b - 1) hs += rare_q(__ldg(wt + ibase + i * 32 + __ffs(b) - 1), true, cp);
        }
        uint32_t ctot;
        uint32_t j = g0 + warp_excl_scan_u32(c, ctot);
        uint64_t htot;
        uint64_t er = warp_excl_scan_u64(hs, htot);
#pragma unroll
        for (int i = 0; i < WPL; ++i) {
            for (uint32_t b = wd[i]; b; b &= b - 1) {
                const uint32_t item = ibase + i * 32 + (uint32_t)(__ffs(b) - 1);
                er += rare_q(__ldg(wt + item), true, cp);  // the weight again, from L1
                heavy_item[j] = item;
                store_u128(heavy_E + j, q_scale_excess(Eb + ((u128)er << 40), nfix));
                ++j;
            }
        }
        return;
    }
    // dense tile: segment by segment, staged in heavy order and written with coalesced stores
    HeavyStage& sg = stage[warp];
    uint32_t j0 = g0;  // global heavy index of the segment's first heavy
    uint64_t e0 = 0;   // excess of the tile's heavies before the segment (Q40.24)
#pragma unroll 1
    for (int s = 0; s < NSEG; ++s) {
        // lane l: the 16 items [16 l, 16 l + 16) of the segment
        const uint32_t word = __ldg(hmask + (uint64_t)u * WPT + s * (kHeavySeg / 32) + (lane >> 1));
        const uint32_t bits = (word >> ((lane & 1) * 16)) & 0xffffu;
        const uint32_t sbase = tr.local * (uint32_t)T + (uint32_t)s * kHeavySeg;
        const float* wl = wt + sbase + lane * 16;
        // with many heavies a lane loads all 16 weights at once (independent loads); with few
        // it gathers its heavies' weights one by one
        const bool dense = __popc(bits) >= kDenseLane;
        float xv[16];
        uint64_t hs = 0;
        if (dense) {
            if (((uintptr_t)wl & 15u) == 0) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float4 v = __ldg(reinterpret_cast<const float4*>(wl) + k);
                    xv[4 * k] = v.x;
                    xv[4 * k + 1] = v.y;
                    xv[4 * k + 2] = v.z;
                    xv[4 * k + 3] = v.w;
                }
            } else {
#pragma unroll
                for (int k = 0; k < 16; ++k) xv[k] = __ldg(wl + k);
            }
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if ((bits >> k) & 1u) hs += rare_q(xv[k], true, cp);
        } else {
            for (uint32_t b = bits; b; b &= b - 1) hs += rare_q(__ldg(wl + __ffs(b) - 1), true, cp);
        }
        uint32_t ctot;
        uint64_t htot;
        uint32_t pos = warp_excl_scan_u32((uint32_t)__popc(bits), ctot);
        uint64_t er = e0 + warp_excl_scan_u64(hs, htot);
        if (dense) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                if ((bits >> k) & 1u) {
                    er += rare_q(xv[k], true, cp);
                    const uint32_t slot = lkey_slot(pos++);
                    sg.er[slot] = er;
                    sg.off[slot] = (uint16_t)(lane * 16 + k);
                }
            }
        } else {
            for (uint32_t b = bits; b; b &= b - 1) {
                const uint32_t k = (uint32_t)(__ffs(b) - 1);
                er += rare_q(__ldg(wl + k), true, cp);  // the weight again, from L1
                const uint32_t slot = lkey_slot(pos++);
                sg.er[slot] = er;
                sg.off[slot] = (uint16_t)(lane * 16 + k);
            }
        }
        __syncwarp();
        for (uint32_t p = lane; p < ctot; p += 32) {
            const uint32_t slot = lkey_slot(p);
            heavy_item[j0 + p] = sbase + sg.off[slot];
            store_u128(heavy_E + j0 + p, q_scale_excess(Eb + ((u128)sg.er[slot] << 40), nfix));
        }
        __syncwarp();  // the next segment reuses the stage
        j0 += ctot;
        e0 += htot;
    }
}

// ---------------------------------------------------------------- pass 5: split
// Per tile boundary b (0..num_tiles): the start of the deficit line A_before(b), the base of
// its dithering (Dither::c0), and bound = #{heavies with E~ <= A_before(b)} by a binary
// search of the heavy list (the reference's split search, at tile granularity), with
// bound = 0 at b = 0 and nH at b = num_tiles, so light tile t owns heavies
// [start[t].bound, start[t+1].bound).
struct __align__(16) TileStart {
    uint64_t A_lo;
    uint64_t A_hi;
    uint64_t c0;
    uint32_t bound;
    uint32_t pad;
};
static_assert(sizeof(TileStart) == 32, "TileStart layout");

// A group of kTileLinkLanes lanes per start: the starts of the global tiles, then (batched) the
// end of each table. The bound by a (kTileLinkLanes + 1)-ary search: each step tests
// kTileLinkLanes pivots at once (one L2 round trip), and the interval shrinks at every step
// whatever the list holds, so the loop ends on any input.
constexpr int kTileLinkLanes = 8;
template <bool BATCH>
__global__ void __launch_bounds__(256) tile_link_kernel(const BuildHeader* hdr, const TileVals* incl,
                                                        uint32_t num_tiles, uint32_t num_tables,
                                                        const uint4* heavy_E, TileStart* starts, TileMap map) {
    pdl_enter();
    constexpr uint32_t G = kTileLinkLanes;
    static_assert(32 % G == 0, "lane groups");
    if (plan_failed<BATCH>(map)) return;  // the same for every thread
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint32_t j = threadIdx.x % G;
    const uint32_t gfirst = (threadIdx.x & 31u) & ~(G - 1);  // the group's first lane in the warp
    bool active = true;
    TileRef tr;
    if (!BATCH) {
        if (i > num_tiles) {
            active = false;
        } else {
            tr = tile_ref<false>(map, 0);
            tr.local = i;  // the boundary: i == num_tiles is the table's end
        }
    } else if (i < num_tiles) {
        tr = tile_ref<true>(map, i);
    } else if (i < num_tiles + num_tables) {
        const uint32_t t = i - num_tiles;
        tr = table_ref(map.desc[t], t, map.desc[t].ntiles);
    } else {
        active = false;
    }
    if (active && earlier_status(hdr + tr.table) != 0) active = false;
    uint32_t b = 0, nH = 0;
    TileVals pv = tv_zero();
    if (active) {
        heavy_E += tr.heavy_off;
        b = tr.local;
        nH = __ldg(&incl[tr.tile0 + tr.ntiles - 1].nH);
        if (b) pv = ldcg_tilevals(incl + tr.tile0 + b - 1);
    }
    const u128 X = deficit_line(pv);
    // the bound lies in [lo, hi]: every heavy before lo ends at or below X, every one from hi on above
    uint32_t lo = 0, hi = 0;
    if (active && b == tr.ntiles) lo = hi = nH;
    else if (active && b > 0) hi = nH;
    while (__any_sync(0xffffffffu, lo < hi)) {
        const uint32_t len = hi - lo;
        bool pred = false;
        if (lo < hi) {
            const bool small = len <= G;
            const uint32_t p = small ? lo + j : lo + (uint32_t)(((uint64_t)(j + 1) * len) / (G + 1));
            if (!small || j < len) pred = load_u128(heavy_E + p) <= X;
        }
        const uint32_t m = (__ballot_sync(0xffffffffu, pred) >> gfirst) & ((1u << G) - 1u);
        if (lo < hi) {
            const uint32_t c = (uint32_t)__popc(m);  // the ends ascend: the first c pivots are at or below X
            if (len <= G) {
                lo = hi = lo + c;
            } else {
                const uint32_t lo0 = lo;
                if (c > 0) lo = lo0 + (uint32_t)(((uint64_t)c * len) / (G + 1)) + 1;
                if (c < G) hi = lo0 + (uint32_t)(((uint64_t)(c + 1) * len) / (G + 1));
            }
        }
    }
    if (!active || j != 0) return;
    TileStart ts;
    ts.A_lo = q_lo(X);
    ts.A_hi = q_hi(X);
    ts.c0 = make_dither(pv.L).c0;
    ts.bound = lo;
    ts.pad = 0;
    starts[tr.tile0 + tr.table + b] = ts;
}

// ---------------------------------------------------------------- pass 6: pack
// A leftover of the PSA+ local pass (psa_kernels.cuh), which split_pack reads in its leftover
// mode. Light: deficit in Q16.48 in `lo`, its row probability in prob_bits. Heavy: excess in
// Q64.64 in (hi, lo).
struct __align__(8) LeftSlot {
    uint32_t item;
    uint32_t prob_bits;
    uint64_t lo;
    uint64_t hi;
};
static_assert(sizeof(LeftSlot) == 24, "LeftSlot layout");

// Pack CTA shape per tile size: threads x items per thread.
template <int T>
struct PackShape;
template <>
struct PackShape<1024> {
    static constexpr int NT = 128, IPT = 8;
};
template <>
struct PackShape<2048> {
    static constexpr int NT = 256, IPT = 8;
};
template <>
struct PackShape<4096> {
    static constexpr int NT = 256, IPT = 16;
};

// Heavies per chunk for T items per tile: the own-tile phase keeps a u64 per tile item in
// the chunk arrays (16 * C >= 8 * T bytes).
__host__ __device__ constexpr int pack_chunk(int T) { return T / 2 > 1024 ? T / 2 : 1024; }

// Heavies that the merge-walk form of the pack kernel holds at once (a u64 key and a u32 item
// each, in the bytes of the chunk arrays).
__host__ __device__ constexpr int pack_walk_cap(int T) { return (pack_chunk(T) * 16 / 12) & ~31; }

// A heavy's key in a pack tile's frame: ceil((E~ - A_before) / 2^-48), clamped to
// [0, 2^64 - 1].
__device__ __forceinline__ uint64_t pack_heavy_key(u128 Et, u128 A_before) {
    if (Et <= A_before) return 0;
    const u128 d = Et - A_before + 0xffff;
    return (q_hi(d) >> 16) ? ~0ull : (uint64_t)(d >> 16);
}

// A heavy's corrected excess end (Q64.64) from its stored end E (Q40.24): the compact heavy
// list of the split build's scan pass keeps E uncorrected.
__device__ __forceinline__ u128 corrected_end(uint64_t E, int64_t nfix) { return q_scale_excess((u128)E << 40, nfix); }

// The pack kernel's view of the heavy list's excess ends: corrected Q64.64 ends (uint4 each;
// the reduce/prefix/heavy-list passes) or compact Q40.24 ends corrected on load (u64 each;
// the split build's scan pass).
template <bool E64>
struct HeavyEnds;
template <>
struct HeavyEnds<false> {
    const uint4* p;
    __device__ __forceinline__ u128 at(uint32_t g) const { return load_u128(p + g); }
};
template <>
struct HeavyEnds<true> {
    const uint64_t* p;
    int64_t nfix;
    __device__ __forceinline__ u128 at(uint32_t g) const { return corrected_end(__ldg(p + g), nfix); }
};

// Heavies that the split build's walk-form pack kernel (pack_walk_kernel) holds at once for T
// items per tile (a light tile of uniform weights owns about T/2 heavies, with a wide spread);
// tiles with more take split_pack_kernel's chunked form.
__host__ __device__ constexpr int walk_cap(int T) { return T; }

// Shared memory of the pack kernel, in this order: light keys (u64 x T; the staged rows at
// the end), heavy keys (u64 x C), heavy items (u32 x C), heavy ranks (u32 x C).
__host__ __device__ constexpr size_t pack_smem_bytes(int T) {
    return (size_t)T * sizeof(uint64_t) + (size_t)pack_chunk(T) * (sizeof(uint64_t) + 2 * sizeof(uint32_t));
}

// Staged row position of tile item i: an XOR swizzle inside each thread's IPT items, keyed by
// i / max(IPT, 16), so that a warp's 8-byte stores of its threads' k-th items cover all 16
// bank pairs twice (two wavefronts; keyed by the thread index alone, IPT = 8 would hit 8 bank
// pairs four times) and its reads of 32 consecutive rows stay a permutation (two wavefronts).
template <int IPT>
__device__ __forceinline__ uint32_t stage_pos(uint32_t i) {
    constexpr uint32_t kKey = IPT > 16 ? IPT : 16;
    return (i & ~(uint32_t)(IPT - 1)) | ((i ^ (i / kKey)) & (uint32_t)(IPT - 1));
}

// One light tile per CTA of NT threads, IPT consecutive items per thread.
//  (1) Own tile: every light's deficit-interval start goes to shared memory as a key in
//      the tile's frame, key = (A - A_before(t)) / 2^-48 (exact), with large lights dithered.
//  (2) Heavies [start[t].bound, start[t+1].bound] of the heavy list (the owned ones and the
//      next one), in chunks of at most C. A heavy's key in the same frame is
//      ceil((E~ - A_before) / 2^-48) clamped to [0, 2^64 - 1], so key(light) < key(heavy)
//      exactly when A < E~. A heavy's rank is the index of the first light whose key is not
//      below its own (I(j) = #{A < E~_j}, a binary search of the light keys); an owned heavy's
//      row keeps r = 1 + E~ - A_rank and aliases the next heavy. A light's alias is the first
//      heavy whose key exceeds its own (J(i) = #{E~ <= A_i}), i.e. the first heavy whose rank
//      exceeds the light's index: each thread finds it for its first light and then only
//      compares indices with ranks.
//  (3) Light rows, staged in shared memory and written out coalesced (the heavies' rows of
//      this tile belong to the tiles that own them).
// When the heavies of (2) fit in shared memory at once (at most pack_walk_cap(T), the common
// case), (1) and (2) are one merge instead: thread t takes the heavies whose keys lie in
// [b_t, b_t+1), b_t = its first light's key (a lower bound search), and walks its lights in
// order: heavies with key <= the light's key rank at that light (their A_next is its key),
// and the light's alias is the first heavy left. The heavies left after its last light rank
// at the next thread's first light. No light key goes to shared memory and no heavy searches
// the lights.
// In the leftover mode (LEFT, the PSA+ build's second pass) a tile's lights are its leftover
// lights from the slots (deficits and row probabilities given), and their rows are written
// at their items.
// E64 (the split build's compact heavy list): the heavy count comes from the header, and the
// kernel builds only the tiles that pack_walk_kernel listed (their heavies exceed walk_cap(T);
// the list's length in the header's chunk_count), CTA b taking entries b, b + gridDim.x, ...
template <int NT, int IPT, bool BATCH, bool LEFT, bool E64>
__device__ __forceinline__ void split_pack_tile(const float* __restrict__ w, const BuildHeader* hdr,
                                                const TileVals* incl, const TileStart* __restrict__ starts,
                                                const uint32_t* __restrict__ heavy_item,
                                                const void* __restrict__ heavy_E_raw, uint32_t gtile,
                                                wrs_alias_row* __restrict__ table, TileMap map,
                                                const LeftSlot* __restrict__ left) {
    constexpr int T = NT * IPT;
    constexpr int C = pack_chunk(T);
    constexpr int CW = pack_walk_cap(T);
    static_assert(16 * C >= 8 * T, "own-tile slots live in the chunk arrays");
    static_assert(12 * CW <= 16 * C, "walk arrays live in the chunk arrays");
    static_assert(IPT >= 4 && IPT <= 32 && (IPT & (IPT - 1)) == 0, "items per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* sLkey = reinterpret_cast<uint64_t*>(smem_raw);
    uint64_t* sHkey = sLkey + T;
    uint32_t* sHitem = reinterpret_cast<uint32_t*>(sHkey + C);
    uint32_t* sHrank = sHitem + C;
    uint64_t* sStage = sLkey;                                // row phase: staged rows
    uint64_t* sWk = sHkey;                                   // walk: heavy keys, then A_next keys
    uint32_t* sWi = reinterpret_cast<uint32_t*>(sWk + CW);   // walk: heavy items
    __shared__ Scan3 s_scan3[NT / 32];
    __shared__ uint32_t s_wa[NT];
    __shared__ uint32_t s_r0, s_pend_item;
    __shared__ float s_pend_prob;

    const int tid = threadIdx.x;
    if (plan_failed<BATCH>(map)) return;
    const TileRef tr = tile_ref<BATCH>(map, gtile);
    if constexpr (E64) {
        // only the tiles whose heavies exceed walk_cap(T), decided before any weight is read
        if (earlier_status(hdr) != 0) return;
        const uint32_t nH0 = __ldg(&hdr->nH_total);
        const uint32_t lo = starts[tr.local].bound, hi = starts[tr.local + 1].bound;
        if (hi < lo || hi > nH0) return;  // bounds out of order: an earlier pass failed
        if (nH0 == 0 || min(hi + 1u, nH0) - lo <= (uint32_t)walk_cap(NT * IPT)) return;
    }
    const uint32_t tile = tr.local;
    const uint64_t n = tr.n;
    w += tr.item_off;
    table += tr.item_off;
    heavy_item += tr.heavy_off;
    // ---- (1) own tile (the weights' loads go out first: they do not depend on the header)
    float x[IPT];
    if (!LEFT) load_items<NT, IPT>(w, n, tile, tid, x);
    hdr += tr.table;
    if (earlier_status(hdr) != 0) return;
    HeavyEnds<E64> he;
    if constexpr (E64) {
        he.p = static_cast<const uint64_t*>(heavy_E_raw) + tr.heavy_off;
        he.nfix = __ldg(&hdr->nfix);
    } else {
        he.p = static_cast<const uint4*>(heavy_E_raw) + tr.heavy_off;
    }
    const LeftSlot* ls = LEFT ? left + (uint64_t)tile * T : nullptr;
    const uint32_t nvalid = LEFT ? __ldcg(&incl[tile].nL) - (tile ? __ldcg(&incl[tile - 1].nL) : 0u) : 0u;
    const ClassParams cp = load_class_params(hdr);
    const uint32_t nH = E64 ? __ldg(&hdr->nH_total) : __ldg(&incl[tr.tile0 + tr.ntiles - 1].nH);
    const TileStart st0 = starts[tr.tile0 + tr.table + tile], st1 = starts[tr.tile0 + tr.table + tile + 1];
    const u128 A_before = q_make(st0.A_hi, st0.A_lo);
    const u128 A_after = q_make(st1.A_hi, st1.A_lo);
    const uint32_t g_lo = st0.bound, g_hi = st1.bound;
    const uint32_t g_end = min(g_hi + 1u, nH);  // the owned heavies and the next one
    const bool walk = nH != 0 && g_end - g_lo <= (uint32_t)CW;
    const uint32_t m_w = walk ? g_end - g_lo : 0u;
    if (walk) {
#pragma unroll 4
        for (uint32_t j = tid; j < m_w; j += NT) {
            sWk[j] = pack_heavy_key(he.at(g_lo + j), A_before);
            sWi[j] = __ldg(heavy_item + g_lo + j);
        }
    }
    // own-tile phase: a large light's slot (per item), in whichever array is free
    uint64_t* sSlotQ = walk ? sStage : sHkey;
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)tid * IPT);
    float pk[IPT];
    uint32_t lbits = 0, gbits = 0;  // bit k: item k is a light / a large light
    uint64_t asum = 0, lsum = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if constexpr (LEFT) {
            const uint32_t slot = (uint32_t)(tid * IPT + k);
            const bool valid = slot < nvalid;
            pk[k] = valid ? __uint_as_float(ls[slot].prob_bits) : 0.0f;
            asum += valid ? ls[slot].lo : 0ull;
            lbits |= (uint32_t)valid << k;
            continue;
        }
        const float wk = x[k];
        const bool small = wk >= 0.0f && wk < cp.Hh;
        const float p = __fmul_rn(wk, cp.R32);
        pk[k] = p;
        asum += small ? small_deficit(p) : 0ull;
        lbits |= (uint32_t)(wk >= 0.0f && !(wk > cp.H1)) << k;
        gbits |= (uint32_t)(wk >= cp.Hh && !(wk > cp.H1)) << k;
    }
    // large lights' true deficits (weights gathered again from L1), kept in their slots for
    // the dithering
    for (uint32_t bits = gbits; bits; bits &= bits - 1) {
        const int k = __ffs(bits) - 1;
        const uint64_t q = rare_q(__ldg(w + item0 + k), false, cp);
        sSlotQ[tid * IPT + k] = q;
        lsum += q;
    }
    const uint32_t nl = (uint32_t)__popc(lbits);
    Scan3 tot_l;
    const Scan3 ex = block_scan3<NT>(Scan3{nl, asum, lsum}, s_scan3, tot_l);
    const uint32_t nLt = tot_l.c;
    const uint32_t l0 = ex.c;  // this thread's lights are l0 .. l0 + nl - 1 in tile light order
    Dither dth;
    dth.c0 = st0.c0;
    dth.c0h = st0.c0 >> 24;
    const uint64_t D0 = dither_at(dth, ex.b);
    if (!walk) {
        uint64_t sr = ex.a, D = D0, lr = ex.b;
        uint32_t li = l0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const bool light = (lbits >> k) & 1u;
            if (light) sLkey[lkey_slot(li)] = sr + D;
            li += light ? 1u : 0u;
            if (LEFT) {
                sr += light ? ls[tid * IPT + k].lo : 0ull;
                continue;
            }
            sr += (light && !((gbits >> k) & 1u)) ? small_deficit(pk[k]) : 0ull;
            if ((gbits >> k) & 1u) {  // the dithering after a large light
                lr += sSlotQ[tid * IPT + k];
                const uint64_t D1 = dither_at(dth, lr);
                pk[k] = dithered_prob(D1 - D);
                D = D1;
            }
        }
    }
    if (tid == 0) {
        s_r0 = 0;
        s_pend_item = 0xffffffffu;
    }
    __syncthreads();  // keys complete; the slot arrays are free again

    uint32_t al[IPT];
    if (nH == 0) {
        // no heavy item anywhere: every row keeps itself
#pragma unroll
        for (int k = 0; k < IPT; ++k) al[k] = LEFT ? (((lbits >> k) & 1u) ? ls[tid * IPT + k].item : 0u) : item0 + k;
    } else if (walk) {
        // ---- (1)+(2) as one merge of this thread's lights with the heavies of its key range
        const uint32_t last_heavy = __ldg(heavy_item + nH - 1);
        uint32_t a = 0;
        {
            const uint64_t b_t = ex.a + D0;  // this thread's first light's key
            uint32_t hi = m_w;
            while (a < hi) {
                const uint32_t mid = (a + hi) >> 1;
                if (sWk[mid] < b_t) a = mid + 1; else hi = mid;
            }
        }
        s_wa[tid] = a;
        __syncthreads();  // every range known; from here a thread touches only its own keys
        const uint32_t a_end = (tid + 1 < NT) ? s_wa[tid + 1] : m_w;
        uint64_t hk = a < a_end ? sWk[a] : ~0ull;
        uint32_t cur = a < m_w ? sWi[a] : last_heavy;  // the first heavy left: the lights' alias
        uint64_t sr = ex.a, D = D0, lr = ex.b;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const bool light = (lbits >> k) & 1u;
            if (light) {
                const uint64_t key = sr + D;
                if (hk <= key) {
                    do {  // heavy a ranks at this light (a < a_end bounds the loop whatever the keys)
                        sWk[a] = key;
                        ++a;
                        hk = a < a_end ? sWk[a] : ~0ull;
                    } while (a < a_end && hk <= key);
                    cur = a < m_w ? sWi[a] : last_heavy;
                }
                al[k] = cur;
            }
            if (LEFT) {
                sr += light ? ls[tid * IPT + k].lo : 0ull;
                continue;
            }
            sr += (light && !((gbits >> k) & 1u)) ? small_deficit(pk[k]) : 0ull;
            if ((gbits >> k) & 1u) {  // the dithering after a large light
                lr += sSlotQ[tid * IPT + k];
                const uint64_t D1 = dither_at(dth, lr);
                pk[k] = dithered_prob(D1 - D);
                D = D1;
            }
        }
        // the heavies left rank at the next thread's first light (or past the tile's lights)
        const uint64_t nxt = (l0 + nl < nLt) ? sr + D : ~0ull;
        for (; a < a_end; ++a) sWk[a] = nxt;
    } else {
        // ---- (2) owned heavies and the next one, chunk by chunk
        const uint32_t last_heavy = __ldg(heavy_item + nH - 1);
#pragma unroll
        for (int k = 0; k < IPT; ++k) al[k] = last_heavy;  // lights past every heavy's excess
                                                            // (rounding residue only)
        for (uint32_t cs = g_lo; cs < g_end; cs += (uint32_t)C) {
            const uint32_t m = min((uint32_t)C, g_end - cs);
            // state left by the previous chunk (rewritten below only after the next barrier)
            const uint32_t r0 = s_r0;  // lights below r0 already have their alias
            const uint32_t pend = s_pend_item;
            const float pend_prob = s_pend_prob;
            for (uint32_t j = tid; j < m; j += NT) {
                sHkey[j] = pack_heavy_key(he.at(cs + j), A_before);
                sHitem[j] = __ldg(heavy_item + cs + j);
            }
            __syncthreads();
            // the previous chunk's last owned heavy aliases this chunk's first
            if (tid == 0 && pend != 0xffffffffu) {
                wrs_alias_row r;
                r.prob = pend_prob;
                r.alias = sHitem[0];
                if (pend < n) table[pend] = r;
            }
            // ranks: the index of the first light whose key is not below the heavy's
            // (all heavies of this chunk rank at r0 or later)
            for (uint32_t j = tid; j < m; j += NT) {
                const uint64_t kh = sHkey[j];
                uint32_t lo = r0, hi = nLt;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (sLkey[lkey_slot(mid)] < kh) lo = mid + 1; else hi = mid;
                }
                sHrank[j] = lo;
            }
            __syncthreads();
            // this thread's lights: alias = the first heavy whose rank exceeds the light's index
            if (l0 + nl > r0) {
                const uint32_t ls = max(l0, r0);
                uint32_t a = 0, hi = m;  // first heavy with rank > ls
                while (a < hi) {
                    const uint32_t mid = (a + hi) >> 1;
                    if (sHrank[mid] <= ls) a = mid + 1; else hi = mid;
                }
                uint32_t ra = a < m ? sHrank[a] : 0xffffffffu;
                uint32_t ia = a < m ? sHitem[a] : 0u;
                uint32_t li = l0;
#pragma unroll
                for (int k = 0; k < IPT; ++k) {
                    if ((lbits >> k) & 1u) {
                        if (li >= r0) {
                            while (ra <= li) {
                                ++a;
                                ra = a < m ? sHrank[a] : 0xffffffffu;
                                ia = a < m ? sHitem[a] : 0u;
                            }
                            if (a < m) al[k] = ia;
                        }
                        ++li;
                    }
                }
            }
            // rows of the owned heavies
            for (uint32_t j = tid; j < m; j += NT) {
                const uint32_t g = cs + j;
                const uint32_t rk = sHrank[j];
                if (j + 1 == m) {
                    s_r0 = rk;
                    s_pend_item = 0xffffffffu;
                }
                if (g < g_hi) {
                    const u128 Et = he.at(g);
                    const u128 A_next = (rk < nLt) ? A_before + ((u128)sLkey[lkey_slot(rk)] << 16) : A_after;
                    const float prob = heavy_row_prob(q_one() + Et - A_next);
                    if (j + 1 < m) {
                        wrs_alias_row r;
                        r.prob = prob;
                        r.alias = sHitem[j + 1];
                        if (sHitem[j] < n) table[sHitem[j]] = r;
                    } else if (g + 1 < nH) {
                        s_pend_item = sHitem[j];  // its alias opens the next chunk
                        s_pend_prob = prob;
                    } else {
                        wrs_alias_row r;  // the last heavy of the table keeps itself
                        r.prob = prob;
                        r.alias = sHitem[j];
                        if (sHitem[j] < n) table[sHitem[j]] = r;
                    }
                }
            }
            __syncthreads();  // the next chunk overwrites the chunk arrays
        }
    }

    // rows of the owned heavies of the walk form, once every key left is in place
    auto walk_heavy_rows = [&]() {
        const uint32_t m_own = g_hi - g_lo;
        for (uint32_t j = tid; j < m_own; j += NT) {
            const uint64_t nk = sWk[j];
            const u128 A_next = nk == ~0ull ? A_after : A_before + ((u128)nk << 16);
            wrs_alias_row r;
            r.prob = heavy_row_prob(q_one() + he.at(g_lo + j) - A_next);
            r.alias = (g_lo + j + 1 < nH) ? sWi[j + 1] : sWi[j];  // the last heavy keeps itself
            if (sWi[j] < n) table[sWi[j]] = r;
        }
    };
    // ---- (3) light rows: staged, then coalesced stores (heavy positions are skipped)
    if constexpr (LEFT) {
        if (walk) {
            __syncthreads();
            walk_heavy_rows();
        }
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (!((lbits >> k) & 1u)) continue;
            wrs_alias_row r;
            r.prob = pk[k];
            r.alias = al[k];
            table[ls[tid * IPT + k].item] = r;
        }
    } else {
    #pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const bool light = (lbits >> k) & 1u;
            const uint64_t row = light ? (((uint64_t)al[k] << 32) | __float_as_uint(pk[k])) : ~0ull;
            sStage[stage_pos<IPT>((uint32_t)(tid * IPT + k))] = row;
        }
        __syncthreads();
        if (walk) walk_heavy_rows();
        uint64_t* out = reinterpret_cast<uint64_t*>(table) + (uint64_t)tile * T;
        const uint32_t cnt = (uint32_t)min((uint64_t)T, n - (uint64_t)tile * T);
        if (cnt == (uint32_t)T) {
    #pragma unroll
            for (int it = 0; it < IPT; ++it) {
                const uint32_t i = (uint32_t)(it * NT + tid);
                const uint64_t row = sStage[stage_pos<IPT>(i)];
                if (row != ~0ull) out[i] = row;
            }
        } else {
            for (uint32_t i = tid; i < cnt; i += NT) {
                const uint64_t row = sStage[stage_pos<IPT>(i)];
                if (row != ~0ull) out[i] = row;
            }
        }
    }
}

template <int NT, int IPT, bool BATCH, bool LEFT, bool E64 = false>
__global__ void __launch_bounds__(NT, (NT == 256 && IPT == 8) ? 4 : 1) split_pack_kernel(const float* __restrict__ w,
                                                        const BuildHeader* hdr, const TileVals* incl,
                                                        const TileStart* __restrict__ starts,
                                                        const uint32_t* __restrict__ heavy_item,
                                                        const void* __restrict__ heavy_E_raw, uint32_t num_tiles,
                                                        wrs_alias_row* __restrict__ table, TileMap map,
                                                        const LeftSlot* __restrict__ left,
                                                        const uint32_t* __restrict__ tile_list) {
    pdl_enter();
    if constexpr (E64) {
        const uint32_t count = min(__ldg(&hdr->chunk_count), num_tiles);
        for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
            split_pack_tile<NT, IPT, BATCH, LEFT, E64>(w, hdr, incl, starts, heavy_item, heavy_E_raw,
                                                       __ldg(tile_list + i), table, map, left);
            __syncthreads();  // the next tile reuses the shared arrays
        }
    } else {
        // descending: the previous passes ended at the last tiles, still in L2
        split_pack_tile<NT, IPT, BATCH, LEFT, E64>(w, hdr, incl, starts, heavy_item, heavy_E_raw,
                                                   num_tiles - 1 - blockIdx.x, table, map, left);
    }
}

}  // namespace wrs
