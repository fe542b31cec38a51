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
// Passes: (1) wsum: compensated W; (2) tile_scan: per-tile counts and Q64.64 sums of the
// three streams (small-light deficits S, large-light true deficits L, heavy excess E),
// decoupled look-back -> inclusive tile prefixes; (3) split_pack: per light tile, locate
// the heavy tiles whose excess range covers the tile's deficit range (the split), merge
// (the pack), and write rows. Tile t owns (writes the row of) every heavy whose corrected
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
// CPU oracle restates it operation by operation.
enum : int { kAbsent = 0, kSmallLight = 1, kLargeLight = 2, kHeavy = 3 };

struct ItemClass {
    int kind;
    float p;  // small light: stored probability
    u128 q;   // small light: stored deficit; large light: true deficit; heavy: excess
};

__device__ __forceinline__ ItemClass classify(float wf, double W_N, double R) {
    ItemClass c;
    const double w = (double)wf;
    if (w > W_N) {
        c.kind = kHeavy;
        double h = w * R;
        if (h < 1.0) h = 1.0;
        c.q = q_from_double(h) - q_one();
        c.p = 1.0f;
    } else {
        double p = w * R;
        if (p > 1.0) p = 1.0;
        if (p >= 0.5) {
            c.kind = kLargeLight;
            c.q = q_from_double(1.0 - p);  // exact: 1 - p is a multiple of 2^-53 in [0, 1/2]
            c.p = 1.0f;
        } else {
            c.kind = kSmallLight;
            const float ps = __double2float_rn(p);
            c.p = ps;
            c.q = q_one() - q_from_double((double)ps);
        }
    }
    return c;
}

// Stored probability of a dithered large light from its prefix L_i and true deficit d.
__device__ __forceinline__ float large_light_prob(u128 L_i, u128 d) {
    const u128 dd = q_round24(L_i + d) - q_round24(L_i);  // multiple of 2^-24, <= 2^23 + 1 units
    const uint32_t units = (uint32_t)(dd >> 40);
    return (float)(16777216u - units) * 5.9604644775390625e-8f;  // exact
}
__device__ __forceinline__ u128 large_light_deficit(u128 L_i, u128 d) {
    return q_round24(L_i + d) - q_round24(L_i);
}

// A heavy's row probability from r in Q64.64 (clamped to [0, 1]).
__device__ __forceinline__ float heavy_row_prob(u128 r) {
    if (q_is_negative(r)) return 0.0f;
    if (r >= q_one()) return 1.0f;
    return __double2float_rn((double)(q_lo(r) >> 11) * 1.1102230246251565404e-16);
}

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
    u128 a;
    u128 b;
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
        o.a = shfl_up_u128(inc.a, off);
        o.b = shfl_up_u128(inc.b, off);
        if (lane >= off) inc = sv_add(inc, o);
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const ScanVal x = (lane < BLOCK / 32) ? s_warp[lane] : sv_zero();
        ScanVal xi = x;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            ScanVal o;
            o.c = __shfl_up_sync(0xffffffffu, xi.c, off);
            o.a = shfl_up_u128(xi.a, off);
            o.b = shfl_up_u128(xi.b, off);
            if (lane >= off) xi = sv_add(xi, o);
        }
        __syncwarp();
        if (lane < BLOCK / 32) {
            ScanVal ex;
            ex.c = xi.c - x.c;
            ex.a = xi.a - x.a;
            ex.b = xi.b - x.b;
            s_warp[lane] = ex;
        }
        if (lane == BLOCK / 32 - 1) s_warp[BLOCK / 32] = xi;
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

// ---------------------------------------------------------------- pass 2: tile scan
// One tile per CTA, tiles taken in ticket order (a CTA only ever waits for tiles whose
// CTAs are already running). Publishes the tile aggregate (flag 1), looks back warp-wide,
// publishes the inclusive prefix (flag 2). agg[] keeps first/last heavy of each tile.
template <int IPT>
__global__ void __launch_bounds__(kBuildThreads) tile_scan_kernel(const float* __restrict__ w, uint64_t n,
                                                                  BuildHeader* hdr, TileVals* agg,
                                                                  TileVals* incl, uint32_t* flags,
                                                                  uint32_t num_tiles) {
    constexpr int T = kBuildThreads * IPT;
    __shared__ uint32_t s_tile;
    __shared__ ScanVal s_warp[kBuildThreads / 32 + 1];
    __shared__ uint32_t s_fh[kBuildThreads / 32];
    __shared__ uint32_t s_lh[kBuildThreads / 32];
    __shared__ TileVals s_agg;
    __shared__ int s_abort;

    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&hdr->tile_ticket, 1u);
        s_abort = (load_relaxed(&hdr->status) != 0);
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= num_tiles) return;
    if (s_abort) {
        // publish a placeholder so that successors do not wait for the time limit
        if (threadIdx.x == 0) {
            incl[tile] = tv_zero();
            __threadfence();
            store_release(&flags[tile], 2u);
        }
        return;
    }
    const double W_N = hdr->W_N;
    const double R = hdr->R;

    float x[IPT];
    load_tile_items<IPT>(w, n, tile, threadIdx.x, x);
    uint32_t nL = 0, nH = 0, fh = 0xffffffffu, lh = 0;
    bool anyh = false;
    u128 S = 0, L = 0, E = 0;
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)threadIdx.x * IPT);
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if (x[k] < 0.0f) continue;
        const ItemClass c = classify(x[k], W_N, R);
        if (c.kind == kHeavy) {
            ++nH;
            E += c.q;
            fh = min(fh, item0 + k);
            lh = item0 + k;
            anyh = true;
        } else {
            ++nL;
            if (c.kind == kSmallLight) S += c.q; else L += c.q;
        }
    }
    ScanVal v;
    v.c = nL;
    v.a = S;
    v.b = L;
    ScanVal tot;
    (void)cta_exclusive_scan<kBuildThreads>(v, s_warp, &tot);
    ScanVal vh;
    vh.c = nH;
    vh.a = E;
    vh.b = 0;
    ScanVal toth;
    (void)cta_exclusive_scan<kBuildThreads>(vh, s_warp, &toth);
    uint32_t f = fh;
    uint32_t l = anyh ? lh : 0u;
    uint32_t has = anyh ? 1u : 0u;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        f = min(f, __shfl_xor_sync(0xffffffffu, f, off));
        l = max(l, __shfl_xor_sync(0xffffffffu, l, off));
        has |= __shfl_xor_sync(0xffffffffu, has, off);
    }
    if ((threadIdx.x & 31) == 0) {
        s_fh[threadIdx.x >> 5] = f;
        s_lh[threadIdx.x >> 5] = has ? l : 0xffffffffu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        TileVals a = tv_zero();
        uint32_t mf = 0xffffffffu, ml = 0xffffffffu;
        for (int i = 0; i < kBuildThreads / 32; ++i) {
            mf = min(mf, s_fh[i]);
            if (s_lh[i] != 0xffffffffu) ml = (ml == 0xffffffffu) ? s_lh[i] : max(ml, s_lh[i]);
        }
        a.nL = tot.c;
        a.S = tot.a;
        a.L = tot.b;
        a.nH = toth.c;
        a.E = toth.a;
        a.first_heavy = mf;
        a.last_heavy = ml;
        s_agg = a;
    }
    __syncthreads();

    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    const TileVals a = s_agg;
    if (tile == 0) {
        if (lane == 0) {
            agg[0] = a;
            incl[0] = tv_add(tv_zero(), a);
            __threadfence();
            store_release(&flags[0], 2u);
        }
        return;
    }
    if (lane == 0) {
        agg[tile] = a;
        __threadfence();
        store_release(&flags[tile], 1u);
    }
    TileVals excl = tv_zero();
    int64_t pred = (int64_t)tile - 1;
    bool timed_out = false;
    const uint64_t t_start = global_ns();
    while (true) {
        const int64_t p = pred - lane;
        uint32_t fl = 2u;
        TileVals pv = tv_zero();
        if (p >= 0) {
            uint32_t spins = 0;
            while ((fl = load_acquire(&flags[p])) == 0u) {
                __nanosleep(32);
                if ((++spins & 255u) == 0u) {
                    if (global_ns() - t_start > kWaitLimitNs || load_relaxed(&hdr->status) != 0) {
                        timed_out = true;
                        break;
                    }
                }
            }
            if (!timed_out) pv = ldcg_tilevals((fl == 2u) ? (incl + p) : (agg + p));
        }
        if (__any_sync(0xffffffffu, timed_out)) {
            if (lane == 0) record_status(&hdr->status, kErrTimeout);
            break;
        }
        const uint32_t incl_mask = __ballot_sync(0xffffffffu, fl == 2u);
        const int stop = incl_mask ? (__ffs(incl_mask) - 1) : 31;
        if (lane > stop) pv = tv_zero();
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            TileVals o;
            o.nL = __shfl_xor_sync(0xffffffffu, pv.nL, off);
            o.nH = __shfl_xor_sync(0xffffffffu, pv.nH, off);
            o.S = shfl_xor_u128(pv.S, off);
            o.L = shfl_xor_u128(pv.L, off);
            o.E = shfl_xor_u128(pv.E, off);
            pv = tv_add(pv, o);
        }
        excl = tv_add(excl, pv);
        if (incl_mask) break;
        pred -= 32;
    }
    if (lane == 0) {
        incl[tile] = tv_add(excl, a);
        __threadfence();
        store_release(&flags[tile], 2u);
    }
}

// ---------------------------------------------------------------- pass 3: split + pack
// Tile-level prefix access used by the pack kernel.
__device__ __forceinline__ TileVals incl_before(const TileVals* incl, uint32_t u) {
    return u ? ldcg_tilevals(incl + u - 1) : tv_zero();
}

// Warp-cooperative search: largest u in [lo, hi] with pred(u) true, given pred(lo) true and
// pred monotone (true on a prefix). All 32 lanes must call it; every lane gets the answer.
template <typename Pred>
__device__ __forceinline__ uint32_t warp_last_true(uint32_t lo, uint32_t hi, Pred pred) {
    const int lane = threadIdx.x & 31;
    while (hi > lo) {
        const uint64_t span = (uint64_t)(hi - lo);
        const uint32_t pos = lo + (uint32_t)((span * (uint64_t)(lane + 1) + 31) / 32);
        const bool t = (pos <= hi) && pred(pos);
        const uint32_t mask = __ballot_sync(0xffffffffu, t);
        const int c = __popc(mask);
        const uint32_t pos0 = __shfl_sync(0xffffffffu, pos, 0);
        if (c == 0) {
            hi = pos0 - 1;
        } else {
            const uint32_t posc1 = __shfl_sync(0xffffffffu, pos, c - 1);
            const uint32_t posc = __shfl_sync(0xffffffffu, pos, c < 32 ? c : 31);
            lo = posc1;
            if (c < 32) hi = posc - 1;
        }
    }
    return lo;
}

template <int IPT>
__global__ void __launch_bounds__(kBuildThreads, 2) split_pack_kernel(const float* __restrict__ w, uint64_t n,
                                                                     const BuildHeader* hdr,
                                                                     const TileVals* agg,
                                                                     const TileVals* incl,
                                                                     uint32_t num_tiles,
                                                                     wrs_alias_row* __restrict__ table) {
    constexpr int T = kBuildThreads * IPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u128* sA = reinterpret_cast<u128*>(smem_raw);          // light deficit-interval starts
    u128* sE = sA + T;                                     // chunk heavy excess ends (corrected)
    uint32_t* sLalias = reinterpret_cast<uint32_t*>(sE + T);  // alias of each own light
    uint32_t* sHitem = sLalias + T;                        // chunk heavy items
    __shared__ ScanVal s_warp[kBuildThreads / 32 + 1];
    __shared__ uint32_t s_u0, s_u1, s_next, s_r0, s_last_item, s_nlt;

    if (load_relaxed(&hdr->status) != 0) return;
    const uint32_t tile = num_tiles - 1 - blockIdx.x;  // descending: the last tiles of the
                                                       // previous pass are still in L2
    const double W_N = hdr->W_N;
    const double R = hdr->R;
    const TileVals tot = ldcg_tilevals(incl + num_tiles - 1);
    const TileVals before = incl_before(incl, tile);
    const TileVals after = ldcg_tilevals(incl + tile);
    const u128 A_before = before.S + q_round24(before.L);
    const u128 A_after = after.S + q_round24(after.L);
    const u128 A_tot = tot.S + q_round24(tot.L);
    const int64_t nfix = excess_correction(A_tot, tot.E);
    const bool lo_inf = (tile == 0);
    const bool hi_inf = (tile == num_tiles - 1);
    const uint32_t nH_tot = tot.nH;

    // ---- own tile: light deficit intervals
    float x[IPT];
    load_tile_items<IPT>(w, n, tile, threadIdx.x, x);
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)threadIdx.x * IPT);
    ScanVal v = sv_zero();
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if (x[k] < 0.0f) continue;
        const ItemClass c = classify(x[k], W_N, R);
        if (c.kind == kHeavy) continue;
        v.c += 1;
        if (c.kind == kSmallLight) v.a += c.q; else v.b += c.q;
    }
    ScanVal tot_l;
    const ScanVal ex = cta_exclusive_scan<kBuildThreads>(v, s_warp, &tot_l);
    const uint32_t nLt = tot_l.c;
    float pk[IPT];
    uint32_t lk[IPT];
    {
        uint32_t li = ex.c;
        u128 Sr = before.S + ex.a;
        u128 Lr = before.L + ex.b;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            lk[k] = 0xffffffffu;
            pk[k] = 0.0f;
            if (x[k] < 0.0f) continue;
            const ItemClass c = classify(x[k], W_N, R);
            if (c.kind == kHeavy) continue;
            sA[li] = Sr + q_round24(Lr);
            lk[k] = li;
            if (c.kind == kSmallLight) {
                pk[k] = c.p;
                Sr += c.q;
            } else {
                pk[k] = large_light_prob(Lr, c.q);
                Lr += c.q;
            }
            ++li;
        }
    }
    __syncthreads();

    if (nH_tot == 0) {
        // no heavy item anywhere: every row keeps itself
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (lk[k] == 0xffffffffu) continue;
            wrs_alias_row r;
            r.prob = pk[k];
            r.alias = item0 + k;
            table[item0 + k] = r;
        }
        return;
    }
    if (!lo_inf && !hi_inf && nLt == 0) return;  // empty ownership interval, no lights

    // ---- split: heavy tiles whose corrected excess range meets (A_before, A_after]
    if (threadIdx.x < 32) {
        auto key_le = [&](uint32_t u, u128 xv) {
            const u128 eb = q_scale_excess(incl_before(incl, u).E, nfix);
            return eb <= xv;
        };
        const uint32_t u0 = lo_inf ? 0u : warp_last_true(0u, num_tiles - 1, [&](uint32_t u) { return key_le(u, A_before); });
        const uint32_t u1 = hi_inf ? num_tiles - 1 : warp_last_true(0u, num_tiles - 1, [&](uint32_t u) { return key_le(u, A_after); });
        if (threadIdx.x == 0) {
            s_u0 = u0;
            s_u1 = u1;
            s_r0 = 0;
            s_last_item = 0xffffffffu;
            s_nlt = nLt;
        }
    }
    __syncthreads();
    const uint32_t u0 = s_u0, u1 = s_u1;

    for (uint32_t u = u0; u <= u1; ++u) {
        const TileVals ub = incl_before(incl, u);
        const TileVals ua = ldcg_tilevals(incl + u);
        const uint32_t m = ua.nH - ub.nH;
        if (m == 0) continue;
        // heavies of tile u: corrected excess ends + items
        float y[IPT];
        load_tile_items<IPT>(w, n, u, threadIdx.x, y);
        const uint32_t uitem0 = (uint32_t)((uint64_t)u * T + (uint64_t)threadIdx.x * IPT);
        ScanVal hv = sv_zero();
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (y[k] < 0.0f || !((double)y[k] > W_N)) continue;
            const ItemClass c = classify(y[k], W_N, R);
            hv.c += 1;
            hv.a += c.q;
        }
        ScanVal tot_h;
        const ScanVal hex = cta_exclusive_scan<kBuildThreads>(hv, s_warp, &tot_h);
        {
            uint32_t hj = hex.c;
            u128 Er = ub.E + hex.a;
#pragma unroll
            for (int k = 0; k < IPT; ++k) {
                if (y[k] < 0.0f || !((double)y[k] > W_N)) continue;
                const ItemClass c = classify(y[k], W_N, R);
                Er += c.q;
                sE[hj] = q_scale_excess(Er, nfix);
                sHitem[hj] = uitem0 + k;
                ++hj;
            }
        }
        // the heavy after this tile's last heavy (alias of that heavy when owned here)
        if (threadIdx.x < 32) {
            const uint32_t g = ua.nH;  // heavies through tile u
            uint32_t nxt = 0xffffffffu;
            if (g < nH_tot) {
                // first tile v > u with incl[v].nH > g  <=>  last tile v' with incl[v'].nH <= g, plus one
                const uint32_t vp = warp_last_true(u, num_tiles - 1, [&](uint32_t vv) { return ldcg_tilevals(incl + vv).nH <= g; });
                nxt = ldcg_tilevals(agg + vp + 1).first_heavy;
            }
            if (threadIdx.x == 0) s_next = nxt;
        }
        __syncthreads();
        const uint32_t r0 = s_r0;
        const uint32_t nl = nLt - r0;
        const uint32_t total = nl + m;
        const uint32_t next_after = s_next;
        // merge path: lights [r0, nLt) (keys sA) against heavies [0, m) (keys sE);
        // a light precedes a heavy iff A < E.
        const uint32_t d0 = (uint32_t)(((uint64_t)total * threadIdx.x) / kBuildThreads);
        const uint32_t d1 = (uint32_t)(((uint64_t)total * (threadIdx.x + 1)) / kBuildThreads);
        uint32_t lo = d0 > m ? d0 - m : 0u;
        uint32_t hi = d0 < nl ? d0 : nl;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (sA[r0 + mid - 1] < sE[d0 - mid]) lo = mid; else hi = mid - 1;
        }
        uint32_t a = lo, b = d0 - lo;
        for (uint32_t d = d0; d < d1; ++d) {
            if (a < nl && (b >= m || sA[r0 + a] < sE[b])) {
                if (b < m) sLalias[r0 + a] = sHitem[b];
                ++a;
            } else {
                const u128 Ev = sE[b];
                const bool owned = (lo_inf || Ev > A_before) && (hi_inf || Ev <= A_after);
                if (owned) {
                    const u128 A_next = (r0 + a < nLt) ? sA[r0 + a] : A_after;
                    const u128 r = q_one() + Ev - A_next;
                    uint32_t al = (b + 1 < m) ? sHitem[b + 1] : next_after;
                    if (al == 0xffffffffu) al = sHitem[b];
                    wrs_alias_row row;
                    row.prob = heavy_row_prob(r);
                    row.alias = al;
                    table[sHitem[b]] = row;
                }
                ++b;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            // lights placed before the chunk's last heavy are resolved
            const u128 elast = sE[m - 1];
            uint32_t l2 = r0, h2 = nLt;  // first x in [r0, nLt) with A[x] >= elast
            while (l2 < h2) {
                const uint32_t mid = (l2 + h2) >> 1;
                if (sA[mid] < elast) l2 = mid + 1; else h2 = mid;
            }
            s_r0 = l2;
            s_last_item = sHitem[m - 1];
        }
        __syncthreads();
    }
    // lights past every heavy's excess (rounding residue only): alias the last heavy
    uint32_t r0 = s_r0;
    if (r0 < nLt) {
        if (threadIdx.x < 32) {
            uint32_t last_item = s_last_item;
            if (last_item == 0xffffffffu) {
                const uint32_t vp = warp_last_true(0u, num_tiles - 1, [&](uint32_t vv) { return incl_before(incl, vv).nH < nH_tot; });
                last_item = ldcg_tilevals(agg + vp).last_heavy;
            }
            if (threadIdx.x == 0) s_last_item = last_item;
        }
        __syncthreads();
        const uint32_t last_item = s_last_item;
        for (uint32_t xx = r0 + threadIdx.x; xx < nLt; xx += kBuildThreads) sLalias[xx] = last_item;
    }
    __syncthreads();
    // own light rows, in item order
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if (lk[k] == 0xffffffffu) continue;
        wrs_alias_row r;
        r.prob = pk[k];
        r.alias = sLalias[lk[k]];
        table[item0 + k] = r;
    }
}

}  // namespace wrs
