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
    uint64_t pad[8];
};
static_assert(sizeof(BuildHeader) == 128, "header layout");

// ---------------------------------------------------------------- classification
// The per-item quantities; the same code runs in every pass that needs them, and the
// CPU oracle restates it operation by operation. Within a tile, deficits are summed as
// u64 in Q16.48 and excess in Q40.24 (rounded per item); tile aggregates and prefixes are
// Q64.64. A light's merge key is exact on the 2^-48 grid, so comparisons against the
// (full-resolution) corrected excess line stay exact; the per-item rounding only moves
// a heavy's reconstructed probability by at most (number of donees) x 2^-49 rows.
//
// Classes, with thresholds computed once per build from W/N (ClassParams):
//   heavy        w > H1 (H1 = largest float <= W/N, so exactly w > W/N): excess h - 1,
//                h = w * (N/W) in FP64;
//   large light  Hh <= w <= H1 (Hh = smallest float >= W/(2N)): true deficit 1 - w*(N/W)
//                in FP64, stored probability dithered (large_light_prob);
//   small light  w < Hh: stored probability p = w * fl32(N/W) in FP32 (within 2 ulp of
//                w/(W/N)), deficit 1 - p.
enum : int { kAbsent = 0, kSmallLight = 1, kLargeLight = 2, kHeavy = 3 };

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

// round(p * 2^48) (ties away from zero) for a float p in [0, 1], from its bits (branch-free:
// t = mantissa * 2^25, sh = 127 - exponent >= 1, result ((t >> (sh - 1)) + 1) >> 1).
__host__ __device__ __forceinline__ uint64_t fix48f(uint32_t b) {
    const int e = (int)((b >> 23) & 0xff);
    const uint64_t t = (uint64_t)((b & 0x7fffffu) | 0x800000u) << 25;
    const int sh = 127 - e;
    const uint64_t r = ((t >> ((sh - 1) & 63)) + 1) >> 1;
    return (e == 0 || sh > 63) ? 0ull : r;
}

struct ItemQ {
    int kind;
    float p;     // small light: stored probability
    uint64_t q;  // light: deficit in Q16.48 (stored for small, true for large); heavy: excess in Q40.24
};

// Caller guarantees wf >= 0 (a present item).
__device__ __forceinline__ ItemQ classify(float wf, const ClassParams& cp) {
    ItemQ c;
    if (wf < cp.Hh) {
        c.kind = kSmallLight;
        c.p = __fmul_rn(wf, cp.R32);
        c.q = (1ull << 48) - fix48f(__float_as_uint(c.p));
    } else {
        const double hd = __dmul_rn((double)wf, cp.R);
        const bool heavy = wf > cp.H1;
        const double v = heavy ? __dsub_rn(fmax(hd, 1.0), 1.0) : __dsub_rn(1.0, fmin(hd, 1.0));
        c.q = fixq(v, heavy ? 24 : 48);
        c.kind = heavy ? kHeavy : kLargeLight;
        c.p = 1.0f;
    }
    return c;
}

// Heavy excess only (the caller has checked wf > H1).
__device__ __forceinline__ uint64_t heavy_excess(float wf, const ClassParams& cp) {
    return fixq(__dsub_rn(fmax(__dmul_rn((double)wf, cp.R), 1.0), 1.0), 24);
}

// Stored probability of a dithered large light: deficit round24(L_i + d) - round24(L_i),
// a multiple of 2^-24, so 1 - deficit is exact in FP32.
__device__ __forceinline__ float large_light_prob(u128 L_i, uint64_t d48) {
    const u128 dd = q_round24(L_i + ((u128)d48 << 16)) - q_round24(L_i);
    const uint32_t units = (uint32_t)(dd >> 40);
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
        if (W_out) *W_out = r.hi;
        if (!(r.hi > 0.0) || isinf(r.hi)) record_status(&hdr->status, isinf(r.hi) ? kErrInvalidWeight : kErrZeroTotal);
        hdr->wsum_ticket = 0u;
    }
}

// ---------------------------------------------------------------- CTA scan helpers
struct ScanVal {
    uint32_t c;
    uint64_t a;
    uint64_t b;
};
__device__ __forceinline__ ScanVal sv_add(const ScanVal& x, const ScanVal& y) {
    ScanVal r;
    r.c = x.c + y.c;
    r.a = x.a + y.a;
    r.b = x.b + y.b;
    return r;
}
__device__ __forceinline__ ScanVal sv_zero() {
    ScanVal r;
    r.c = 0;
    r.a = 0;
    r.b = 0;
    return r;
}

// Exclusive CTA-wide scan of (count, a, b); the CTA total goes to *total.
// s_warp needs BLOCK/32 + 1 entries. Ends with a barrier (s_warp reusable).
template <int BLOCK>
__device__ __forceinline__ ScanVal cta_exclusive_scan(ScanVal v, ScanVal* s_warp, ScanVal* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    ScanVal inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        ScanVal o;
        o.c = __shfl_up_sync(0xffffffffu, inc.c, off);
        o.a = __shfl_up_sync(0xffffffffu, inc.a, off);
        o.b = __shfl_up_sync(0xffffffffu, inc.b, off);
        if (lane >= off) inc = sv_add(inc, o);
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        ScanVal acc = sv_zero();
#pragma unroll
        for (int i = 0; i < BLOCK / 32; ++i) {
            const ScanVal t = s_warp[i];
            s_warp[i] = acc;
            acc = sv_add(acc, t);
        }
        s_warp[BLOCK / 32] = acc;
    }
    __syncthreads();
    const ScanVal base = s_warp[warp];
    *total = s_warp[BLOCK / 32];
    ScanVal ex;
    ex.c = base.c + inc.c - v.c;
    ex.a = base.a + inc.a - v.a;
    ex.b = base.b + inc.b - v.b;
    __syncthreads();
    return ex;
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

// ---------------------------------------------------------------- pass 2: tile reduce
// One tile per CTA: counts and sums of the three streams, plus the tile's first and last
// heavy item. No inter-CTA waits.
template <int IPT>
__global__ void __launch_bounds__(kBuildThreads) tile_reduce_kernel(const float* __restrict__ w, uint64_t n,
                                                                    const BuildHeader* hdr, TileVals* agg,
                                                                    uint32_t* __restrict__ hmask,
                                                                    uint32_t num_tiles) {
    constexpr int T = kBuildThreads * IPT;
    constexpr int NW = kBuildThreads / 32;
    __shared__ uint32_t s_nl[NW], s_nh[NW], s_fh[NW], s_lh[NW];
    __shared__ uint64_t s_s[NW], s_l[NW], s_e[NW];
    if (load_relaxed(&hdr->status) != 0) return;
    const uint32_t tile = blockIdx.x;
    const ClassParams cp = class_params(hdr->W_N, hdr->R);
    float x[IPT];
    load_tile_items<IPT>(w, n, tile, threadIdx.x, x);
    uint32_t nL = 0, nH = 0, fh = 0xffffffffu, lh = 0xffffffffu, hbits = 0;
    uint64_t S = 0, L = 0, E = 0;
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)threadIdx.x * IPT);
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if (x[k] < 0.0f) continue;
        const ItemQ c = classify(x[k], cp);
        if (c.kind == kHeavy) {
            ++nH;
            E += c.q;
            hbits |= 1u << k;
            if (fh == 0xffffffffu) fh = item0 + k;
            lh = item0 + k;
        } else {
            ++nL;
            if (c.kind == kSmallLight) S += c.q; else L += c.q;
        }
    }
    // heavy mask: bit i of word i/32 <=> tile item i is heavy (32 / IPT lanes per word)
    {
        constexpr int LPW = 32 / IPT;
        uint32_t word = hbits << ((threadIdx.x % LPW) * IPT);
#pragma unroll
        for (int d = 1; d < LPW; d <<= 1) word |= __shfl_xor_sync(0xffffffffu, word, d);
        if (threadIdx.x % LPW == 0) hmask[(uint64_t)tile * (T / 32) + threadIdx.x / LPW] = word;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        nL += __shfl_xor_sync(0xffffffffu, nL, off);
        nH += __shfl_xor_sync(0xffffffffu, nH, off);
        S += __shfl_xor_sync(0xffffffffu, S, off);
        L += __shfl_xor_sync(0xffffffffu, L, off);
        E += __shfl_xor_sync(0xffffffffu, E, off);
        fh = min(fh, __shfl_xor_sync(0xffffffffu, fh, off));
        const uint32_t o = __shfl_xor_sync(0xffffffffu, lh, off);
        lh = (lh == 0xffffffffu) ? o : (o == 0xffffffffu ? lh : max(lh, o));
    }
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_nl[warp] = nL;
        s_nh[warp] = nH;
        s_s[warp] = S;
        s_l[warp] = L;
        s_e[warp] = E;
        s_fh[warp] = fh;
        s_lh[warp] = lh;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    uint32_t tl = 0, th = 0, mf = 0xffffffffu, ml = 0xffffffffu;
    uint64_t ts = 0, tlv = 0, te = 0;
#pragma unroll
    for (int i = 0; i < NW; ++i) {
        tl += s_nl[i];
        th += s_nh[i];
        ts += s_s[i];
        tlv += s_l[i];
        te += s_e[i];
        mf = min(mf, s_fh[i]);
        if (s_lh[i] != 0xffffffffu) ml = (ml == 0xffffffffu) ? s_lh[i] : max(ml, s_lh[i]);
    }
    TileVals a;
    a.nL = tl;
    a.nH = th;
    a.first_heavy = mf;
    a.last_heavy = ml;
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
                                                                     uint32_t num_tiles) {
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
    if (s_abort) {
        if (threadIdx.x == 0) store_release(&blocks[blk].flag, 2u);
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
            if (lane == 0) {
                blocks[0].agg = btot;
                blocks[0].incl = btot;
                store_release(&blocks[0].flag, 2u);
            }
        } else {
            if (lane == 0) {
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
                            if (global_ns() - t_start > kWaitLimitNs || load_relaxed(&hdr->status) != 0) {
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
            if (lane == 0) {
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
    }
}

// ---------------------------------------------------------------- pass 4: split
// Per light tile t, the range [u0, u1] of tiles whose heavies' corrected excess ends meet
// the tile's deficit range (A_before(t), A_after(t)] (the reference's split search, at tile
// granularity), and the item of the first heavy after tile t. links[num_tiles].next_item
// is the last heavy item of the whole table.
struct TileLink {
    uint32_t u0;
    uint32_t u1;
    uint32_t next_item;
    uint32_t pad;
};

__device__ __forceinline__ u128 excess_before(const TileVals* incl, uint32_t u) {
    return u ? ldcg_E(incl + u - 1) : (u128)0;
}

static __global__ void __launch_bounds__(256) tile_link_kernel(const BuildHeader* hdr, const TileVals* agg,
                                                               const TileVals* incl, uint32_t num_tiles,
                                                               TileLink* links) {
    if (load_relaxed(&hdr->status) != 0) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > num_tiles) return;
    const TileVals tot = ldcg_tilevals(incl + num_tiles - 1);
    if (t == num_tiles) {
        // last heavy of the table: in the last tile whose predecessors hold fewer than nH heavies
        uint32_t item = 0xffffffffu;
        if (tot.nH > 0) {
            uint32_t lo = 0, hi = num_tiles - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (ldcg_tilevals(incl + mid - 1).nH < tot.nH) lo = mid; else hi = mid - 1;
            }
            item = ldcg_tilevals(agg + lo).last_heavy;
        }
        TileLink l;
        l.u0 = 0;
        l.u1 = 0;
        l.next_item = item;
        l.pad = 0;
        links[num_tiles] = l;
        return;
    }
    const int64_t nfix = excess_correction(deficit_line(tot), tot.E);
    const u128 A_b = t ? deficit_line(ldcg_tilevals(incl + t - 1)) : (u128)0;
    const TileVals me = ldcg_tilevals(incl + t);
    const u128 A_a = deficit_line(me);
    TileLink l;
    l.pad = 0;
    // largest u with corrected E_before(u) <= x (E_before(0) = 0 <= x)
    auto last_le = [&](u128 xv) {
        uint32_t lo = 0, hi = num_tiles - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (q_scale_excess(excess_before(incl, mid), nfix) <= xv) lo = mid; else hi = mid - 1;
        }
        return lo;
    };
    l.u0 = (t == 0) ? 0u : last_le(A_b);
    l.u1 = (t == num_tiles - 1) ? num_tiles - 1 : last_le(A_a);
    // first heavy after tile t: tile v = first tile whose inclusive count exceeds g
    const uint32_t g = me.nH;
    l.next_item = 0xffffffffu;
    if (g < tot.nH) {
        uint32_t lo = t, hi = num_tiles - 1;  // last v with incl[v].nH <= g
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (ldcg_tilevals(incl + mid).nH <= g) lo = mid; else hi = mid - 1;
        }
        l.next_item = ldcg_tilevals(agg + lo + 1).first_heavy;
    }
    links[t] = l;
}

// ---------------------------------------------------------------- pass 5: pack
__device__ __forceinline__ TileVals incl_before(const TileVals* incl, uint32_t u) {
    return u ? ldcg_tilevals(incl + u - 1) : tv_zero();
}

// Shared memory of the pack kernel for T items per tile: light keys (u64), heavy keys (u64),
// heavy local excess (u64), heavy items (u32), light aliases (u32), heavy ranks (u32).
__host__ __device__ constexpr size_t pack_smem_bytes(int T) {
    return (size_t)T * (3 * sizeof(uint64_t) + 3 * sizeof(uint32_t));
}

// One light tile per CTA. Its lights' deficit-interval starts go to shared memory as keys
// in the tile's frame (A - A_before(t), Q16.48). The heavies of the partner tiles
// [u0, u1] are taken one tile at a time from the tile's heavy mask (written by the reduce
// pass): only the heavies' weights are gathered (from L2), so a partner costs work in
// proportion to its heavies. Their corrected excess ends become keys in the same frame:
// key = ceil((E~ - A_before(t)) / 2^-48), clamped, so that key(light) < key(heavy) exactly
// when A < E~. A merge path over the still unresolved lights and the chunk's heavies gives
// every thread an equal slice of the merged order; the slice only records ranks: a light's
// alias is the heavy at its rank (J(i) = #{E~ <= A_i}), a heavy's rank is the light after
// it (I(j) = #{A < E~_j}). Owned heavies then write their rows from those ranks, and the
// last heavy's rank is the number of lights resolved so far.
template <int IPT>
__global__ void __launch_bounds__(kBuildThreads, (IPT <= 8 ? 3 : 1)) split_pack_kernel(const float* __restrict__ w,
                                                                                     uint64_t n,
                                                                                     const BuildHeader* hdr,
                                                                                     const TileVals* incl,
                                                                                     const TileLink* links,
                                                                                     const uint32_t* __restrict__ hmask,
                                                                                     uint32_t num_tiles,
                                                                                     wrs_alias_row* __restrict__ table) {
    constexpr int T = kBuildThreads * IPT;
    constexpr int WPT = T / 32;  // heavy-mask words per tile
    static_assert(WPT <= kBuildThreads, "one mask word per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* sLkey = reinterpret_cast<uint64_t*>(smem_raw);
    uint64_t* sHkey = sLkey + T;
    uint64_t* sHe = sHkey + T;
    uint32_t* sHitem = reinterpret_cast<uint32_t*>(sHe + T);
    uint32_t* sLalias = sHitem + T;
    uint32_t* sHrank = sLalias + T;
    __shared__ ScanVal s_warp[kBuildThreads / 32 + 1];
    __shared__ uint32_t s_own_lo, s_own_hi;

    if (load_relaxed(&hdr->status) != 0) return;
    const uint32_t tile = num_tiles - 1 - blockIdx.x;  // descending: the previous passes ended at
                                                       // the last tiles, still in L2
    const ClassParams cp = class_params(hdr->W_N, hdr->R);
    const TileLink link = links[tile];
    const TileVals tot = ldcg_tilevals(incl + num_tiles - 1);
    const TileVals before = incl_before(incl, tile);
    const TileVals after = ldcg_tilevals(incl + tile);
    const u128 A_before = deficit_line(before);
    const u128 A_after = deficit_line(after);
    const int64_t nfix = excess_correction(deficit_line(tot), tot.E);
    const bool lo_inf = (tile == 0);
    const bool hi_inf = (tile == num_tiles - 1);
    const uint32_t nH_tot = tot.nH;

    // ---- own tile: light deficit intervals
    float x[IPT];
    load_tile_items<IPT>(w, n, tile, threadIdx.x, x);
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)threadIdx.x * IPT);
    float pk[IPT];
    ScanVal v = sv_zero();
    uint32_t lmask = 0, bigmask = 0;  // bit k: item k is a light / a large light
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        pk[k] = 0.0f;
        if (x[k] < 0.0f) continue;
        const ItemQ c = classify(x[k], cp);
        if (c.kind == kHeavy) continue;
        lmask |= 1u << k;
        v.c += 1;
        if (c.kind == kSmallLight) {
            pk[k] = c.p;
            v.a += c.q;
        } else {
            bigmask |= 1u << k;
            v.b += c.q;
        }
    }
    ScanVal tot_l;
    const ScanVal ex = cta_exclusive_scan<kBuildThreads>(v, s_warp, &tot_l);
    const uint32_t nLt = tot_l.c;
    const uint32_t l0 = ex.c;  // this thread's lights are l0 .. l0 + popc(lmask) - 1
    {
        uint32_t li = l0;
        uint64_t sr = ex.a;
        u128 Lg = before.L + ((u128)ex.b << 16);
        const u128 rb = q_round24(before.L);
        uint64_t dith = (uint64_t)((q_round24(Lg) - rb) >> 16);
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (!(lmask >> k & 1u)) continue;
            sLalias[li] = 0xffffffffu;
            sLkey[li++] = sr + dith;
            if (bigmask >> k & 1u) {
                const uint64_t q = classify(x[k], cp).q;
                pk[k] = large_light_prob(Lg, q);
                Lg += (u128)q << 16;
                dith = (uint64_t)((q_round24(Lg) - rb) >> 16);
            } else {
                sr += (1ull << 48) - fix48f(__float_as_uint(pk[k]));
            }
        }
    }
    __syncthreads();

    if (nH_tot == 0) {
        // no heavy item anywhere: every row keeps itself
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (!(lmask >> k & 1u)) continue;
            wrs_alias_row r;
            r.prob = pk[k];
            r.alias = item0 + k;
            table[item0 + k] = r;
        }
        return;
    }
    if (!lo_inf && !hi_inf && nLt == 0) return;  // empty ownership interval, no lights

    uint32_t r0 = 0;  // lights [0, r0) are resolved
    uint32_t last_item = 0xffffffffu;
    for (uint32_t u = link.u0; u <= link.u1; ++u) {
        const uint32_t nh_b = u ? __ldcg(&incl[u - 1].nH) : 0u;
        const uint32_t m = __ldcg(&incl[u].nH) - nh_b;
        if (m == 0) continue;
        const u128 E_b = excess_before(incl, u);
        // expand the heavy mask of tile u into the heavies' items, in order
        {
            const uint32_t word = threadIdx.x < WPT ? __ldg(hmask + (uint64_t)u * WPT + threadIdx.x) : 0u;
            ScanVal wv = sv_zero();
            wv.c = __popc(word);
            ScanVal wt;
            const ScanVal wex = cta_exclusive_scan<kBuildThreads>(wv, s_warp, &wt);
            uint32_t o = wex.c;
            const uint32_t base = u * (uint32_t)T + threadIdx.x * 32u;
            for (uint32_t bits = word; bits; bits &= bits - 1) sHitem[o++] = base + (uint32_t)(__ffs(bits) - 1);
        }
        if (threadIdx.x == 0) {
            s_own_lo = 0xffffffffu;
            s_own_hi = 0;
        }
        __syncthreads();
        // excess of each heavy (weights gathered from L2), contiguous blocks per thread
        const uint32_t per = (m + kBuildThreads - 1) / kBuildThreads;
        const uint32_t j0 = min(m, threadIdx.x * per), j1 = min(m, j0 + per);
        ScanVal hv = sv_zero();
        for (uint32_t j = j0; j < j1; ++j) hv.a += heavy_excess(__ldg(w + sHitem[j]), cp);
        ScanVal tot_h;
        const ScanVal hex = cta_exclusive_scan<kBuildThreads>(hv, s_warp, &tot_h);
        {
            uint64_t er = hex.a;
            uint32_t own_lo = 0xffffffffu, own_hi = 0;
            for (uint32_t j = j0; j < j1; ++j) {
                er += heavy_excess(__ldg(w + sHitem[j]), cp);
                const u128 Et = q_scale_excess(E_b + ((u128)er << 40), nfix);
                uint64_t key;
                if (Et <= A_before) {
                    key = 0;
                } else {
                    const u128 d = Et - A_before + 0xffff;
                    key = (q_hi(d) >> 16) ? ~0ull : (uint64_t)(d >> 16);
                }
                if ((lo_inf || Et > A_before) && (hi_inf || Et <= A_after)) {
                    own_lo = min(own_lo, j);
                    own_hi = j + 1;
                }
                sHkey[j] = key;
                sHe[j] = er;
            }
            if (own_hi > 0) {
                atomicMin(&s_own_lo, own_lo);
                atomicMax(&s_own_hi, own_hi);
            }
        }
        __syncthreads();
        // merge path over lights [r0, nLt) and heavies [0, m); a light precedes a heavy iff
        // its key is below the heavy's. Each thread records ranks for an equal slice.
        {
            const uint32_t nl = nLt - r0;
            const uint32_t total = nl + m;
            const uint32_t d0 = (uint32_t)(((uint64_t)total * threadIdx.x) / kBuildThreads);
            const uint32_t d1 = (uint32_t)(((uint64_t)total * (threadIdx.x + 1)) / kBuildThreads);
            uint32_t lo = d0 > m ? d0 - m : 0u;
            uint32_t hi = d0 < nl ? d0 : nl;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (sLkey[r0 + mid - 1] < sHkey[d0 - mid]) lo = mid; else hi = mid - 1;
            }
            uint32_t a = lo, b = d0 - lo;
            for (uint32_t d = d0; d < d1; ++d) {
                const bool take_light = a < nl && (b >= m || sLkey[r0 + a] < sHkey[b]);
                if (take_light) {
                    if (b < m) sLalias[r0 + a] = sHitem[b];
                    ++a;
                } else {
                    sHrank[b] = r0 + a;
                    ++b;
                }
            }
        }
        __syncthreads();
        // owned heavies [own_lo, own_hi): rows from the ranks
        const uint32_t olo = s_own_lo, ohi = s_own_hi;
        const uint32_t next_after = links[u].next_item;
        for (uint32_t j = olo + threadIdx.x; j < ohi; j += kBuildThreads) {
            const uint32_t rk = sHrank[j];
            const u128 Et = q_scale_excess(E_b + ((u128)sHe[j] << 40), nfix);
            const u128 A_next = (rk < nLt) ? A_before + ((u128)sLkey[rk] << 16) : A_after;
            uint32_t al = (j + 1 < m) ? sHitem[j + 1] : next_after;
            if (al == 0xffffffffu) al = sHitem[j];
            wrs_alias_row row;
            row.prob = heavy_row_prob(q_one() + Et - A_next);
            row.alias = al;
            table[sHitem[j]] = row;
        }
        // lights before the chunk's last heavy are resolved
        r0 = sHrank[m - 1];
        last_item = sHitem[m - 1];
        __syncthreads();
    }
    // lights past every heavy's excess (rounding residue only) alias the last heavy
    if (last_item == 0xffffffffu) last_item = links[num_tiles].next_item;
    uint32_t li = l0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if (!(lmask >> k & 1u)) continue;
        const uint32_t al = sLalias[li++];
        wrs_alias_row r;
        r.prob = pk[k];
        r.alias = al != 0xffffffffu ? al : last_item;
        table[item0 + k] = r;
    }
}

}  // namespace wrs
