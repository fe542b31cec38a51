// split_kernels.cuh — the single-table split build after the weight total.
//
// The arithmetic is the one of build_kernels.cuh (classes, per-item fixed-point quantities,
// dithering of large lights, the corrected excess line, the merge of the deficit line with
// the excess line), so the tables are bit for bit those of the CPU oracle's or_exact_build;
// what changes is how the work is cut into launches:
//   scan  — one pass over the weights, groups of tiles per CTA: per-tile sums (aggregates for
//           tile_prefix_kernel), a decoupled look-back over the groups for the heavy count and
//           excess before each group, and the heavy list in heavy order (item and excess end in
//           Q40.24, 12 bytes per heavy). The reduce and heavy-list passes and the second
//           read of the heavies' weights from DRAM are gone.
//   tile_prefix (build_kernels.cuh) — the deficit-line prefixes of the tiles.
//   link  — per tile boundary, the tile start and the number of heavies whose corrected excess
//           end lies at or below the boundary's deficit line (the reference's split search at
//           tile granularity, SplitMethodBasic.cu:14-50).
//   pack  — per light tile, in descending tile order: the merge of its lights with the heavies
//           of its range (walk form, pack_walk_kernel); tiles whose heavies exceed the walk
//           arrays take split_pack_kernel's chunked form.
// The excess ends are stored uncorrected: a reader maps E (Q40.24) to the corrected line by
// corrected_end(E, nfix), exactly the value the earlier passes stored in Q64.64.
#pragma once

#include "build_kernels.cuh"

namespace wrs {

// Exclusive CTA-wide scan of four values (a count and three u64 sums); `total` gets the sums
// of the whole CTA. s must hold NT/32 entries and must not be rewritten before a barrier
// that follows every read of it.
struct Scan4 {
    uint32_t c;
    uint64_t e, s, l;
};
__device__ __forceinline__ Scan4 s4_add(const Scan4& x, const Scan4& y) {
    Scan4 r;
    r.c = x.c + y.c;
    r.e = x.e + y.e;
    r.s = x.s + y.s;
    r.l = x.l + y.l;
    return r;
}
__device__ __forceinline__ Scan4 s4_shfl_up(const Scan4& v, int d) {
    Scan4 o;
    o.c = __shfl_up_sync(0xffffffffu, v.c, d);
    o.e = __shfl_up_sync(0xffffffffu, v.e, d);
    o.s = __shfl_up_sync(0xffffffffu, v.s, d);
    o.l = __shfl_up_sync(0xffffffffu, v.l, d);
    return o;
}
__device__ __forceinline__ Scan4 s4_shfl(const Scan4& v, int src) {
    Scan4 o;
    o.c = __shfl_sync(0xffffffffu, v.c, src);
    o.e = __shfl_sync(0xffffffffu, v.e, src);
    o.s = __shfl_sync(0xffffffffu, v.s, src);
    o.l = __shfl_sync(0xffffffffu, v.l, src);
    return o;
}
template <int NT>
__device__ __forceinline__ Scan4 block_scan4(const Scan4 v, Scan4* s, Scan4& total) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Scan4 inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Scan4 o = s4_shfl_up(inc, off);
        if (lane >= off) inc = s4_add(inc, o);
    }
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    Scan4 t = {0u, 0ull, 0ull, 0ull};
    if (lane < NW) t = s[lane];
#pragma unroll
    for (int off = 1; off < NW; off <<= 1) {
        const Scan4 o = s4_shfl_up(t, off);
        if (lane >= off) t = s4_add(t, o);
    }
    total = s4_shfl(t, NW - 1);
    const Scan4 base = s4_shfl(t, warp > 0 ? warp - 1 : 0);
    Scan4 ex;
    ex.c = (warp ? base.c : 0u) + inc.c - v.c;
    ex.e = (warp ? base.e : 0ull) + inc.e - v.e;
    ex.s = (warp ? base.s : 0ull) + inc.s - v.s;
    ex.l = (warp ? base.l : 0ull) + inc.l - v.l;
    return ex;
}

// Exclusive CTA-wide scan of two u64 sums (same contract as block_scan4).
struct Scan2 {
    uint64_t a, b;
};
template <int NT>
__device__ __forceinline__ Scan2 block_scan2(const Scan2 v, Scan2* s) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Scan2 inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint64_t oa = __shfl_up_sync(0xffffffffu, inc.a, off);
        const uint64_t ob = __shfl_up_sync(0xffffffffu, inc.b, off);
        if (lane >= off) {
            inc.a += oa;
            inc.b += ob;
        }
    }
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    Scan2 t = {0ull, 0ull};
    if (lane < NW) t = s[lane];
#pragma unroll
    for (int off = 1; off < NW; off <<= 1) {
        const uint64_t oa = __shfl_up_sync(0xffffffffu, t.a, off);
        const uint64_t ob = __shfl_up_sync(0xffffffffu, t.b, off);
        if (lane >= off) {
            t.a += oa;
            t.b += ob;
        }
    }
    const int src = warp > 0 ? warp - 1 : 0;
    const uint64_t ba = __shfl_sync(0xffffffffu, t.a, src);
    const uint64_t bb = __shfl_sync(0xffffffffu, t.b, src);
    Scan2 ex;
    ex.a = (warp ? ba : 0ull) + inc.a - v.a;
    ex.b = (warp ? bb : 0ull) + inc.b - v.b;
    return ex;
}

// ---------------------------------------------------------------- scan
// One group of U consecutive tiles (NT x IPT items each) per CTA, groups taken in ticket order
// (so every predecessor of a group has started); the next tile's weights are loaded while the
// current one is summed. Per tile it writes the tile's sums as a TileVals aggregate (for
// tile_prefix_kernel, which turns them into the deficit-line starts) and keeps in shared
// memory each thread's heavy bits and its exclusive heavy count and excess within the tile.
// The group is the unit of a decoupled look-back over (heavy count, heavy excess) only: one
// 16-byte word per group, {flag << 62 | count, excess (Q40.24)}, stored and loaded by single
// 16-byte accesses, so a look-back step is one L2 round trip. With the group's exclusive count
// and excess, the CTA writes the heavies of its tiles at their global heavy index (heavy_item,
// heavy_E = inclusive excess end, Q40.24; the heavies' weights gathered again from L1/L2).
// Every wait is bounded (wc); heavy list writes are bounded by n whatever a failed look-back
// left in the prefixes.
constexpr int kScanThreads = 256;
constexpr int kScanGroup = 8;  // most tiles per look-back unit
// Tiles per look-back unit for a build of num_tiles tiles: kScanGroup, halved while that leaves
// fewer than kScanMinGroups units, so that a small table's scan spreads over the SMs (2^20 items
// in 2048-item tiles: 512 units of one tile instead of 64 of eight).
constexpr uint64_t kScanMinGroups = 592;
__host__ __device__ inline uint32_t scan_group_tiles(uint64_t num_tiles) {
    uint32_t g = kScanGroup;
    while (g > 1 && (num_tiles + g - 1) / g < kScanMinGroups) g >>= 1;
    return g;
}

// Look-back word of a group: a = flag << 62 | heavy count, b = heavy excess (Q40.24); flag 1 =
// the group's own sums, 2 = the sums of every group up to it.
struct __align__(16) LbWord {
    unsigned long long a, b;
};
__device__ __forceinline__ void lb_store(LbWord* p, uint64_t flag, uint64_t count, uint64_t excess) {
    __stcg(reinterpret_cast<ulonglong2*>(p), make_ulonglong2((flag << 62) | count, excess));
}
__device__ __forceinline__ ulonglong2 lb_load(const LbWord* p) {
    return __ldcg(reinterpret_cast<const ulonglong2*>(p));
}

// Inclusive warp scan of a count and a u64 sum; the warp's totals in *tc, *te.
__device__ __forceinline__ void warp_scan_ce(uint32_t& c, uint64_t& e) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t oc = __shfl_up_sync(0xffffffffu, c, off);
        const uint64_t oe = __shfl_up_sync(0xffffffffu, e, off);
        if (lane >= off) {
            c += oc;
            e += oe;
        }
    }
}
// Warp sum of values below 2^51 by two 32-bit reductions (25-bit low parts, 26-bit high parts).
__device__ __forceinline__ uint64_t warp_sum_u51(uint64_t v) {
    const uint32_t lo = __reduce_add_sync(0xffffffffu, (uint32_t)v & ((1u << 25) - 1u));
    const uint32_t hi = __reduce_add_sync(0xffffffffu, (uint32_t)(v >> 25));
    return ((uint64_t)hi << 25) + lo;
}
__device__ __forceinline__ uint64_t warp_sum_u64x(uint64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

template <int IPT>
__global__ void __launch_bounds__(kScanThreads) scan_kernel(const float* __restrict__ w, uint64_t n, BuildHeader* hdr,
                                                            LbWord* lb, uint32_t num_tiles, TileVals* agg,
                                                            uint32_t* __restrict__ heavy_item,
                                                            uint64_t* __restrict__ heavy_E, WaitCfg wc, uint32_t gt) {
    pdl_enter();
    constexpr int NT = kScanThreads;
    constexpr int NW = NT / 32;
    constexpr int T = NT * IPT;
    constexpr int U = kScanGroup;
    static_assert(IPT >= 4 && IPT <= 32 && (IPT & (IPT - 1)) == 0, "items per thread");
    __shared__ uint32_t s_group;
    __shared__ int s_abort;
    __shared__ uint32_t s_wc[U][NW];     // per tile and warp: heavy count
    __shared__ uint64_t s_we[U][NW];     // ... heavy excess (Q40.24)
    __shared__ uint64_t s_ws[U][NW];     // ... small-light deficits (Q16.48)
    __shared__ uint64_t s_wl[U][NW];     // ... large-light true deficits (Q16.48)
    __shared__ uint32_t s_hbits[U][NT];  // per tile and thread: heavy bits of its IPT items
    __shared__ uint32_t s_hc[U][NT];     // ... inclusive heavy count within its warp
    __shared__ uint64_t s_he[U][NT];     // ... inclusive heavy excess within its warp (Q40.24)
    __shared__ uint32_t s_tc0[U + 1][NW];  // heavies before (tile, warp) within the group
    __shared__ uint64_t s_te0[U + 1][NW];  // ... their excess
    __shared__ uint64_t s_base_c, s_base_e;

    const uint32_t num_groups = (num_tiles + gt - 1) / gt;  // gt = scan_group_tiles(num_tiles) <= U
    if (threadIdx.x == 0) {
        s_group = atomicAdd(&hdr->tile_ticket, 1u);
        s_abort = load_relaxed(&hdr->status) != 0;
    }
    __syncthreads();
    const uint32_t group = s_group;
    if (group >= num_groups) return;
    const bool publish = group != wc.hold;  // a held unit (failure-detection tests) publishes nothing
    if (s_abort) {
        if (threadIdx.x == 0 && publish) lb_store(lb + group, 2u, 0u, 0u);
        return;
    }
    const ClassParams cp = load_class_params(hdr);
    const float R48 = cp.R32 * 281474976710656.0f;
    const uint32_t tile0 = group * gt;
    const uint32_t ntl = min(min(gt, (uint32_t)U), num_tiles - tile0);  // tiles of this group
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    // one tile's sums from its weights in registers; warp-level only (no CTA barrier)
    auto sum_tile = [&](const float (&x)[IPT], uint32_t u) {
        const uint32_t tile = tile0 + u;
        const uint64_t item0 = (uint64_t)tile * T + (uint64_t)threadIdx.x * IPT;
        uint32_t lbits = 0, sbits = 0, hbits = 0;
        uint64_t S = 0;
        if ((uint64_t)(tile + 1) * T <= n && R48 < __int_as_float(0x7f800000)) {
            // a full tile: p * 2^48 = w * (fl32(N/W) * 2^48) exactly, small_deficit(p) = 2^48 - rne(p * 2^48)
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
        // rare items (large lights and heavies): from the registers when a thread has many, else
        // gathered again from L1
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
                const uint64_t q = rare_q(__ldg(w + item0 + k), heavy, cp);
                E += heavy ? q : 0ull;
                L += heavy ? 0ull : q;
            }
        }
        const uint32_t c = (uint32_t)__popc(hbits);
        uint32_t ci = c;
        uint64_t ei = E;
        warp_scan_ce(ci, ei);
        s_hbits[u][threadIdx.x] = hbits;
        s_hc[u][threadIdx.x] = ci;
        s_he[u][threadIdx.x] = ei;
        S = warp_sum_u51(S);  // at most IPT deficits of at most 2^48 each
        L = warp_sum_u51(L);
        if (lane == 31) {
            s_wc[u][warp] = ci;
            s_we[u][warp] = ei;
            s_ws[u][warp] = S;
            s_wl[u][warp] = L;
        }
    };

    float xa[IPT], xb[IPT];
    load_items<NT, IPT>(w, n, tile0, threadIdx.x, xa);
    for (uint32_t u = 0; u < ntl; u += 2) {
        if (u + 1 < ntl) load_items<NT, IPT>(w, n, tile0 + u + 1, threadIdx.x, xb);
        sum_tile(xa, u);
        if (u + 1 >= ntl) break;
        if (u + 2 < ntl) load_items<NT, IPT>(w, n, tile0 + u + 2, threadIdx.x, xa);
        sum_tile(xb, u + 1);
    }
    __syncthreads();
    // per tile (thread u < ntl): its aggregate; warp 1 lane 0: the heavies before every
    // (tile, warp) of the group, in item order
    if (threadIdx.x < ntl) {
        const uint32_t u = threadIdx.x;
        const uint32_t tile = tile0 + u;
        uint32_t tc = 0;
        uint64_t te = 0, ts = 0, tl = 0;
#pragma unroll
        for (int v = 0; v < NW; ++v) {
            tc += s_wc[u][v];
            te += s_we[u][v];
            ts += s_ws[u][v];
            tl += s_wl[u][v];
        }
        const uint64_t valid = min((uint64_t)T, n - (uint64_t)tile * T);
        TileVals a;
        a.nL = (uint32_t)valid - tc;
        a.nH = tc;
        a.first_heavy = 0xffffffffu;
        a.last_heavy = 0xffffffffu;
        a.S = (u128)ts << 16;
        a.L = (u128)tl << 16;
        a.E = (u128)te << 40;
        agg[tile] = a;
    }
    if (threadIdx.x == 32) {
        uint32_t c = 0;
        uint64_t e = 0;
        for (uint32_t u = 0; u < ntl; ++u) {
#pragma unroll
            for (int v = 0; v < NW; ++v) {
                s_tc0[u][v] = c;
                s_te0[u][v] = e;
                c += s_wc[u][v];
                e += s_we[u][v];
            }
        }
        s_tc0[U][0] = c;
        s_te0[U][0] = e;
    }
    __syncthreads();
    const uint64_t gc = s_tc0[U][0], ge = s_te0[U][0];

    // decoupled look-back over the groups (warp 0): lane l reads the word of group (pred - l)
    if (threadIdx.x < 32) {
        uint64_t xc = 0, xe = 0;
        if (group == 0) {
            if (lane == 0 && publish) lb_store(lb, 2u, gc, ge);
        } else {
            if (lane == 0 && publish) lb_store(lb + group, 1u, gc, ge);
            int64_t pred = (int64_t)group - 1;
            bool timed_out = false;
            const uint64_t t_start = global_ns();
            while (true) {
                const int64_t p = pred - lane;
                ulonglong2 v = make_ulonglong2(2ull << 62, 0ull);
                if (p >= 0) {
                    uint32_t spins = 0;
                    while (((v = lb_load(lb + p)).x >> 62) == 0u) {
                        __nanosleep(32);
                        if ((++spins & 63u) == 0u) {
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
                const uint32_t incl_mask = __ballot_sync(0xffffffffu, (v.x >> 62) == 2u);
                const int stop = incl_mask ? (__ffs(incl_mask) - 1) : 31;
                uint64_t c = (lane <= stop) ? (v.x & ((1ull << 62) - 1)) : 0ull;
                uint64_t e = (lane <= stop) ? v.y : 0ull;
                c = warp_sum_u64x(c);
                e = warp_sum_u64x(e);
                xc += c;
                xe += e;
                if (incl_mask) break;
                pred -= 32;
            }
            if (lane == 0 && publish) lb_store(lb + group, 2u, xc + gc, xe + ge);
        }
        if (lane == 0) {
            s_base_c = xc;
            s_base_e = xe;
        }
    }
    __syncthreads();
    // the heavies of the group's tiles at their global heavy index, each thread's from its last
    // one back: the last one's excess end is the thread's inclusive prefix, an earlier one's the
    // later one's minus the later one's excess (gathered again only for a thread with several)
    const uint64_t base_c = s_base_c, base_e = s_base_e;
    for (uint32_t u = 0; u < ntl; ++u) {
        const uint32_t hbits = s_hbits[u][threadIdx.x];
        if (hbits) {
            const uint64_t item0 = (uint64_t)(tile0 + u) * T + (uint64_t)threadIdx.x * IPT;
            uint64_t g = base_c + s_tc0[u][warp] + s_hc[u][threadIdx.x];  // one past the thread's last
            uint64_t er = base_e + s_te0[u][warp] + s_he[u][threadIdx.x];
            for (uint32_t bits = hbits;;) {
                const int k = 31 - __clz(bits);
                --g;
                if (g < n) {
                    heavy_item[g] = (uint32_t)(item0 + k);
                    heavy_E[g] = er;
                }
                bits &= ~(1u << k);
                if (!bits) break;
                er -= rare_q(__ldg(w + item0 + k), true, cp);
            }
        }
    }
}

// ---------------------------------------------------------------- link
// A group of kLinkLanes lanes per tile boundary b (0 .. num_tiles): the start of the deficit
// line A_before(b) and the base of its dithering from the tile prefixes (incl, tile_prefix_kernel),
// and bound = #{heavies with corrected excess end <= A_before(b)} by a (kLinkLanes + 1)-ary search
// of the heavy list (the reference's split search at tile granularity, SplitMethodBasic.cu:14-50):
// each step tests kLinkLanes pivots at once, one L2 round trip, so a search over 2^21 heavies takes
// 7 round trips instead of 21. bound = 0 at b = 0 and the heavy count at b = num_tiles (which also
// goes to the header). The interval shrinks at every step whatever the list holds, so the loop ends
// on any input.
constexpr int kLinkLanes = 8;
__global__ void __launch_bounds__(256) link_kernel(BuildHeader* hdr, const TileVals* incl, uint32_t num_tiles,
                                                   const uint64_t* __restrict__ heavy_E, TileStart* starts) {
    pdl_enter();
    constexpr uint32_t G = kLinkLanes;
    static_assert(32 % G == 0, "lane groups");
    if (earlier_status(hdr) != 0) return;  // the same for every thread
    const uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint32_t j = threadIdx.x % G;
    const uint32_t gfirst = (threadIdx.x & 31u) & ~(G - 1);  // the group's first lane in the warp
    const bool active = b <= num_tiles;
    const uint32_t nH = __ldg(&incl[num_tiles - 1].nH);
    const int64_t nfix = __ldg(&hdr->nfix);
    const TileVals pv = (active && b) ? ldcg_tilevals(incl + b - 1) : tv_zero();
    const u128 X = deficit_line(pv);
    // the bound lies in [lo, hi]: every heavy before lo ends at or below X, every one from hi on above
    uint32_t lo = 0, hi = 0;
    if (active && b == num_tiles) lo = hi = nH;
    else if (active && b > 0) hi = nH;
    while (__any_sync(0xffffffffu, lo < hi)) {
        const uint32_t len = hi - lo;
        bool pred = false;
        if (lo < hi) {
            const bool small = len <= G;
            const uint32_t p = small ? lo + j : lo + (uint32_t)(((uint64_t)(j + 1) * len) / (G + 1));
            if (!small || j < len) pred = corrected_end(__ldg(heavy_E + p), nfix) <= X;
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
    if (b == num_tiles) hdr->nH_total = nH;
    TileStart ts;
    ts.A_lo = q_lo(X);
    ts.A_hi = q_hi(X);
    ts.c0 = make_dither(pv.L).c0;
    ts.bound = lo;
    ts.pad = 0;
    starts[b] = ts;
}

// ---------------------------------------------------------------- pack (walk form)
// Stage slots: thread t's IPT items at t * (IPT + 1) + k (one padding slot per thread), so a
// warp's 8-byte accesses at a fixed k fall on distinct bank pairs and every access is a
// constant offset from the thread's base.
template <int IPT>
__host__ __device__ constexpr uint32_t pad_slot(uint32_t i) { return i + i / IPT; }
// Shared memory of pack_walk_kernel: padded stage slots (u64), heavy keys (u64 x C), heavy
// items (u32 x C).
__host__ __device__ constexpr size_t pack_walk_smem_bytes(int T, int IPT) {
    return (size_t)(T + T / IPT) * sizeof(uint64_t) + (size_t)walk_cap(T) * (sizeof(uint64_t) + sizeof(uint32_t));
}
// A large light's stage slot holds its step on the deficit line with this bit set.
constexpr uint64_t kLargeStep = 1ull << 63;

// One light tile per CTA of NT threads, IPT consecutive items per thread, tiles in descending
// order (the scan ended at the last tiles, which may still be in L2). A tile whose heavies
// (the owned ones and the next one) exceed walk_cap(T) is appended to chunk_list (its length in
// the header's chunk_count) and left to split_pack_kernel's chunked form. The merge is that of
// split_pack_kernel's walk form, with each light's step on the tile's deficit line prepared
// before the walk so that the walk itself keeps one running key:
//  (1) every small light's deficit (2^48 - rne(p 2^48)) goes to its stage slot, every large
//      light's true deficit too, and the thread sums both kinds;
//  (2) a CTA scan of the two sums gives each thread's start on the tile's deficit line;
//  (3) the thread's large lights replace their deficits by their dithered steps (flagged);
//  (4) thread t takes the heavies whose keys lie in [b_t, b_t+1) (b_t: its first light's key)
//      and walks its lights in order: heavies with key <= the light's key rank at that light
//      (their A_next is the light's key) and the light's alias is the first heavy left; the
//      light's row replaces its step in the stage slot;
//  (5) the owned heavies' rows are written (scattered), the staged light rows stored coalesced
//      (heavy positions skipped).
template <int NT, int IPT>
__global__ void __launch_bounds__(NT) pack_walk_kernel(const float* __restrict__ w, uint64_t n, BuildHeader* hdr,
                                                       const TileStart* __restrict__ starts,
                                                       const uint32_t* __restrict__ heavy_item,
                                                       const uint64_t* __restrict__ heavy_E, uint32_t num_tiles,
                                                       wrs_alias_row* __restrict__ table, uint32_t* chunk_list) {
    pdl_enter();
    constexpr int T = NT * IPT;
    constexpr int TS = T + T / IPT;
    constexpr int CW = walk_cap(T);
    static_assert(IPT >= 4 && IPT <= 32 && (IPT & (IPT - 1)) == 0, "items per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* sStage = reinterpret_cast<uint64_t*>(smem_raw);  // steps, then rows
    uint64_t* sWk = sStage + TS;                                // heavy keys, then A_next keys
    uint32_t* sWi = reinterpret_cast<uint32_t*>(sWk + CW);      // heavy items
    __shared__ Scan2 s_scan[NT / 32];
    __shared__ uint32_t s_wa[NT];

    const int tid = threadIdx.x;
    const uint32_t tile = num_tiles - 1 - blockIdx.x;
    float x[IPT];
    load_items<NT, IPT>(w, n, tile, tid, x);  // first: independent of the header
    if (earlier_status(hdr) != 0) return;
    const uint32_t nH = __ldg(&hdr->nH_total);
    const TileStart st0 = starts[tile], st1 = starts[tile + 1];
    const uint32_t g_lo = st0.bound, g_hi = st1.bound;
    if (g_hi < g_lo || g_hi > nH) return;  // bounds out of order: an earlier pass failed
    const uint32_t g_end = min(g_hi + 1u, nH);  // the owned heavies and the next one
    const uint32_t m_w = nH ? g_end - g_lo : 0u;
    if (m_w > (uint32_t)CW) {  // the chunked form's tile: listed for split_pack_kernel
        if (tid == 0) chunk_list[atomicAdd(&hdr->chunk_count, 1u)] = tile;
        return;
    }
    const ClassParams cp = load_class_params(hdr);
    const int64_t nfix = __ldg(&hdr->nfix);
    const u128 A_before = q_make(st0.A_hi, st0.A_lo);
#pragma unroll 4
    for (uint32_t j = tid; j < m_w; j += NT) {
        sWk[j] = pack_heavy_key(corrected_end(__ldg(heavy_E + g_lo + j), nfix), A_before);
        sWi[j] = __ldg(heavy_item + g_lo + j);
    }
    // (1) deficits into the stage slots, and the thread's sums
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)tid * IPT);
    uint64_t* my = sStage + (uint32_t)tid * (IPT + 1);
    uint32_t lbits = 0, gbits = 0;  // bit k: item k is a light / a large light
    uint64_t asum = 0, lsum = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const float wk = x[k];
        const bool light = wk >= 0.0f && !(wk > cp.H1);
        const bool small = wk >= 0.0f && wk < cp.Hh;
        const uint64_t d = small_deficit(__fmul_rn(wk, cp.R32));
        my[k] = d;
        asum += small ? d : 0ull;
        lbits |= (uint32_t)light << k;
        gbits |= (uint32_t)(light && !small) << k;
    }
    for (uint32_t bits = gbits; bits; bits &= bits - 1) {  // large lights: true deficits (FP64)
        const int k = __ffs(bits) - 1;
        const uint64_t q = rare_q(__ldg(w + item0 + k), false, cp);
        my[k] = q;
        lsum += q;
    }
    // (2) the thread's start on the tile's deficit line
    const Scan2 ex = block_scan2<NT>(Scan2{asum, lsum}, s_scan);
    Dither dth;
    dth.c0 = st0.c0;
    dth.c0h = st0.c0 >> 24;
    // (3) large lights: their dithered steps on the line
    uint64_t D = dither_at(dth, ex.b);
    const uint64_t key0 = ex.a + D;  // this thread's first light's key
    {
        uint64_t lr = ex.b;
        for (uint32_t bits = gbits; bits; bits &= bits - 1) {
            const int k = __ffs(bits) - 1;
            lr += my[k];
            const uint64_t D1 = dither_at(dth, lr);
            my[k] = (D1 - D) | kLargeStep;
            D = D1;
        }
    }
    // (4) the walk: rows into the stage slots
    if (nH == 0) {
        // no heavy item anywhere: every row keeps itself
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint64_t v = my[k];
            const bool light = (lbits >> k) & 1u;
            const float prob = (v & kLargeStep) ? dithered_prob(v & ~kLargeStep) : __fmul_rn(x[k], cp.R32);
            my[k] = light ? (((uint64_t)(item0 + k) << 32) | __float_as_uint(prob)) : ~0ull;
        }
        __syncthreads();
    } else {
        const uint32_t last_heavy = __ldg(heavy_item + nH - 1);
        uint32_t a = 0;
        {
            uint32_t hi = m_w;
            while (a < hi) {
                const uint32_t mid = (a + hi) >> 1;
                if (sWk[mid] < key0) a = mid + 1; else hi = mid;
            }
        }
        s_wa[tid] = a;
        __syncthreads();  // every range known; from here a thread touches only its own keys
        const uint32_t a_end = (tid + 1 < NT) ? s_wa[tid + 1] : m_w;
        uint64_t hk = a < a_end ? sWk[a] : ~0ull;
        uint32_t cur = a < m_w ? sWi[a] : last_heavy;  // the first heavy left: the lights' alias
        uint64_t key = key0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint64_t v = my[k];
            const bool light = (lbits >> k) & 1u;
            if (light && hk <= key) {
                do {  // heavy a ranks at this light (a < a_end bounds the loop whatever the keys)
                    sWk[a] = key;
                    ++a;
                    hk = a < a_end ? sWk[a] : ~0ull;
                } while (a < a_end && hk <= key);
                cur = a < m_w ? sWi[a] : last_heavy;
            }
            const float prob = (v & kLargeStep) ? dithered_prob(v & ~kLargeStep) : __fmul_rn(x[k], cp.R32);
            my[k] = light ? (((uint64_t)cur << 32) | __float_as_uint(prob)) : ~0ull;
            key += light ? (v & ~kLargeStep) : 0ull;
        }
        // the heavies left rank at the next thread's first light (the tile's end for the last)
        for (; a < a_end; ++a) sWk[a] = key;
        __syncthreads();
        // (5) rows of the owned heavies
        const uint32_t m_own = g_hi - g_lo;
        for (uint32_t j = tid; j < m_own; j += NT) {
            const u128 A_next = A_before + ((u128)sWk[j] << 16);
            wrs_alias_row r;
            r.prob = heavy_row_prob(q_one() + corrected_end(__ldg(heavy_E + g_lo + j), nfix) - A_next);
            r.alias = (g_lo + j + 1 < nH) ? sWi[j + 1] : sWi[j];  // the last heavy keeps itself
            if (sWi[j] < n) table[sWi[j]] = r;
        }
    }
    // light rows, coalesced (heavy positions skipped)
    uint64_t* out = reinterpret_cast<uint64_t*>(table) + (uint64_t)tile * T;
    const uint32_t cnt = (uint32_t)min((uint64_t)T, n - (uint64_t)tile * T);
    if (cnt == (uint32_t)T) {
#pragma unroll
        for (int it = 0; it < IPT; ++it) {
            const uint32_t i = (uint32_t)(it * NT + tid);
            const uint64_t row = sStage[pad_slot<IPT>(i)];
            if (row != ~0ull) out[i] = row;
        }
    } else {
        for (uint32_t i = tid; i < cnt; i += NT) {
            const uint64_t row = sStage[pad_slot<IPT>(i)];
            if (row != ~0ull) out[i] = row;
        }
    }
}

}  // namespace wrs
