// split_kernels.cuh — the single-table split build after the weight total, in three passes.
//
// The arithmetic is the one of build_kernels.cuh (classes, per-item fixed-point quantities,
// dithering of large lights, the corrected excess line, the merge of the deficit line with
// the excess line), so the tables are bit for bit those of the CPU oracle's or_exact_build;
// what changes is how the work is cut into launches:
//   scan  — one pass over the weights, one tile per CTA in ticket order: per-tile sums of the
//           three streams, a decoupled look-back over the tiles for their exclusive prefixes,
//           each tile's start on the deficit line, and the heavy list in heavy order (item and
//           excess end in Q40.24, 12 bytes per heavy). It replaces the reduce, prefix and
//           heavy-list passes and their second read of the heavies' weights.
//   link  — per tile boundary, the number of heavies whose corrected excess end lies at or
//           below the boundary's deficit line (the reference's split search at tile
//           granularity, SplitMethodBasic.cu:14-50).
//   pack  — per light tile, in descending tile order: the merge of its lights with the heavies
//           of its range (walk form, pack_walk_kernel); tiles whose heavies exceed the walk
//           arrays take split_pack_kernel's chunked form.
// The excess ends are stored uncorrected: a reader maps E (Q40.24) to the corrected line by
// q_scale_excess((u128)E << 40, nfix), exactly the value the earlier passes stored in Q64.64.
#pragma once

#include "build_kernels.cuh"

namespace wrs {

// Look-back payload of one tile (or of every tile up to it): heavy count, heavy excess
// (Q40.24), small-light stored deficits and large-light true deficits (Q64.64).
struct __align__(16) ScanVals {
    uint32_t nH;
    uint32_t pad;
    uint64_t E;
    u128 S;
    u128 L;
};
static_assert(sizeof(ScanVals) == 48, "ScanVals layout");

__device__ __forceinline__ ScanVals sv_zero() {
    ScanVals v;
    v.nH = 0;
    v.pad = 0;
    v.E = 0;
    v.S = 0;
    v.L = 0;
    return v;
}
__device__ __forceinline__ ScanVals sv_add(const ScanVals& a, const ScanVals& b) {
    ScanVals r;
    r.nH = a.nH + b.nH;
    r.pad = 0;
    r.E = a.E + b.E;
    r.S = a.S + b.S;
    r.L = a.L + b.L;
    return r;
}
__device__ __forceinline__ ScanVals sv_shfl_xor(const ScanVals& v, int d) {
    ScanVals o;
    o.nH = __shfl_xor_sync(0xffffffffu, v.nH, d);
    o.pad = 0;
    o.E = __shfl_xor_sync(0xffffffffu, v.E, d);
    o.S = shfl_xor_u128(v.S, d);
    o.L = shfl_xor_u128(v.L, d);
    return o;
}
__device__ __forceinline__ void sv_store(ScanVals* dst, const ScanVals& v) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    __stcg(d + 0, make_uint4(v.nH, 0u, (uint32_t)v.E, (uint32_t)(v.E >> 32)));
    __stcg(d + 1, make_uint4((uint32_t)q_lo(v.S), (uint32_t)(q_lo(v.S) >> 32), (uint32_t)q_hi(v.S),
                             (uint32_t)(q_hi(v.S) >> 32)));
    __stcg(d + 2, make_uint4((uint32_t)q_lo(v.L), (uint32_t)(q_lo(v.L) >> 32), (uint32_t)q_hi(v.L),
                             (uint32_t)(q_hi(v.L) >> 32)));
}
__device__ __forceinline__ ScanVals sv_load(const ScanVals* src) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    const uint4 a = __ldcg(s + 0), b = __ldcg(s + 1), c = __ldcg(s + 2);
    ScanVals v;
    v.nH = a.x;
    v.pad = 0;
    v.E = ((uint64_t)a.w << 32) | a.z;
    v.S = q_make(((uint64_t)b.w << 32) | b.z, ((uint64_t)b.y << 32) | b.x);
    v.L = q_make(((uint64_t)c.w << 32) | c.z, ((uint64_t)c.y << 32) | c.x);
    return v;
}

// Look-back records of the scan pass, one per tile. flag: 0 = nothing yet, 1 = agg holds the
// tile's own sums, 2 = incl holds the sums of every tile up to it. agg is never rewritten, so a
// reader that saw flag 1 reads a complete agg.
struct ScanRecs {
    uint32_t* flag;
    ScanVals* agg;
    ScanVals* incl;
};

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
// One tile of NT x IPT items per CTA, tiles taken in ticket order (so every predecessor of a
// tile has started). Writes starts[tile] (deficit line, dither base; bound left for link),
// the tile's heavies at their global heavy index (heavy_item, heavy_E = inclusive excess end,
// Q40.24) and, from the last tile, starts[num_tiles] (line totals, bound = heavy count), the
// excess correction and the heavy count into the header. Every wait is bounded (wc); heavy
// list writes are bounded by n whatever a failed look-back left in the prefixes.
constexpr int kScanThreads = 256;

template <int IPT>
__global__ void __launch_bounds__(kScanThreads) scan_kernel(const float* __restrict__ w, uint64_t n, BuildHeader* hdr,
                                                            ScanRecs rec, uint32_t num_tiles, TileStart* starts,
                                                            uint32_t* __restrict__ heavy_item,
                                                            uint64_t* __restrict__ heavy_E, WaitCfg wc) {
    constexpr int NT = kScanThreads;
    constexpr int T = NT * IPT;
    static_assert(IPT >= 4 && IPT <= 32 && (IPT & (IPT - 1)) == 0, "items per thread");
    __shared__ uint32_t s_tile;
    __shared__ int s_abort;
    __shared__ Scan4 s_scan[NT / 32];
    __shared__ ScanVals s_base;

    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&hdr->tile_ticket, 1u);
        s_abort = load_relaxed(&hdr->status) != 0;
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= num_tiles) return;
    const bool publish = tile != wc.hold;  // a held tile (failure-detection tests) publishes nothing
    if (s_abort) {
        if (threadIdx.x == 0 && publish) {
            sv_store(rec.incl + tile, sv_zero());
            __threadfence();
            store_release(rec.flag + tile, 2u);
        }
        return;
    }
    float x[IPT];
    load_items<NT, IPT>(w, n, tile, threadIdx.x, x);
    const ClassParams cp = load_class_params(hdr);
    const uint64_t item0 = (uint64_t)tile * T + (uint64_t)threadIdx.x * IPT;
    uint32_t lbits = 0, sbits = 0, hbits = 0;
    uint64_t S = 0;
    const float R48 = cp.R32 * 281474976710656.0f;
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
    Scan4 tot;
    const Scan4 ex = block_scan4<NT>(Scan4{(uint32_t)__popc(hbits), E, S, L}, s_scan, tot);
    ScanVals agg;
    agg.nH = tot.c;
    agg.pad = 0;
    agg.E = tot.e;
    agg.S = (u128)tot.s << 16;
    agg.L = (u128)tot.l << 16;

    // decoupled look-back (warp 0): lane l reads the record of tile (pred - l)
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        ScanVals excl = sv_zero();
        if (tile == 0) {
            if (lane == 0 && publish) {
                sv_store(rec.incl, agg);
                __threadfence();
                store_release(rec.flag, 2u);
            }
        } else {
            if (lane == 0 && publish) {
                sv_store(rec.agg + tile, agg);
                __threadfence();
                store_release(rec.flag + tile, 1u);
            }
            int64_t pred = (int64_t)tile - 1;
            bool timed_out = false;
            const uint64_t t_start = global_ns();
            while (true) {
                const int64_t p = pred - lane;
                uint32_t fl = 2u;
                ScanVals pv = sv_zero();
                if (p >= 0) {
                    uint32_t spins = 0;
                    while ((fl = load_acquire(rec.flag + p)) == 0u) {
                        __nanosleep(32);
                        if ((++spins & 63u) == 0u) {
                            if (wait_expired(t_start, wc) || load_relaxed(&hdr->status) != 0) {
                                timed_out = true;
                                break;
                            }
                        }
                    }
                    if (!timed_out) pv = sv_load(fl == 2u ? rec.incl + p : rec.agg + p);
                }
                if (__any_sync(0xffffffffu, timed_out)) {
                    if (lane == 0) record_status(&hdr->status, kErrTimeout);
                    break;
                }
                const uint32_t incl_mask = __ballot_sync(0xffffffffu, fl == 2u);
                const int stop = incl_mask ? (__ffs(incl_mask) - 1) : 31;
                if (lane > stop) pv = sv_zero();
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) pv = sv_add(pv, sv_shfl_xor(pv, d));
                excl = sv_add(excl, pv);
                if (incl_mask) break;
                pred -= 32;
            }
            if (lane == 0 && publish) {
                sv_store(rec.incl + tile, sv_add(excl, agg));
                __threadfence();
                store_release(rec.flag + tile, 2u);
            }
        }
        if (lane == 0) {
            s_base = excl;
            TileStart ts;
            const u128 A = excl.S + q_round24(excl.L);
            ts.A_lo = q_lo(A);
            ts.A_hi = q_hi(A);
            ts.c0 = make_dither(excl.L).c0;
            ts.bound = 0;  // the split search (link_kernel) fills it in
            ts.pad = 0;
            starts[tile] = ts;
            if (tile == num_tiles - 1) {
                const ScanVals t = sv_add(excl, agg);
                const u128 At = t.S + q_round24(t.L);
                TileStart te;
                te.A_lo = q_lo(At);
                te.A_hi = q_hi(At);
                te.c0 = make_dither(t.L).c0;
                te.bound = t.nH;
                te.pad = 0;
                starts[num_tiles] = te;
                hdr->nfix = excess_correction(At, (u128)t.E << 40);
                hdr->nH_total = t.nH;
            }
        }
    }
    __syncthreads();
    // the tile's heavies, in item order, at their global heavy index
    if (hbits) {
        const ScanVals base = s_base;
        uint64_t g = (uint64_t)base.nH + ex.c;
        uint64_t er = base.E + ex.e;
        for (uint32_t bits = hbits; bits; bits &= bits - 1) {
            const int k = __ffs(bits) - 1;
            er += rare_q(__ldg(w + item0 + k), true, cp);
            if (g < n) {
                heavy_item[g] = (uint32_t)(item0 + k);
                heavy_E[g] = er;
            }
            ++g;
        }
    }
}

// ---------------------------------------------------------------- link
// One thread per inner tile boundary b (1 .. num_tiles - 1): bound = #{heavies with corrected
// excess end <= the boundary's deficit line}, by a binary search of the heavy list. starts[0]
// (bound 0) and starts[num_tiles] (bound = heavy count) come from the scan.
__global__ void __launch_bounds__(256) link_kernel(const BuildHeader* hdr, uint32_t num_tiles,
                                                   const uint64_t* __restrict__ heavy_E, TileStart* starts) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (b >= num_tiles) return;
    if (earlier_status(hdr) != 0) return;
    const uint32_t nH = __ldg(&hdr->nH_total);
    const int64_t nfix = __ldg(&hdr->nfix);
    const u128 X = q_make(starts[b].A_hi, starts[b].A_lo);
    uint32_t lo = 0, hi = nH;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (corrected_end(__ldg(heavy_E + mid), nfix) <= X) lo = mid + 1; else hi = mid;
    }
    starts[b].bound = lo;
}

// ---------------------------------------------------------------- pack (walk form)
// Shared memory of pack_walk_kernel: staged rows (u64 x T), heavy keys (u64 x C), heavy items
// (u32 x C).
__host__ __device__ constexpr size_t pack_walk_smem_bytes(int T) {
    return (size_t)T * sizeof(uint64_t) + (size_t)walk_cap(T) * (sizeof(uint64_t) + sizeof(uint32_t));
}

// One light tile per CTA of NT threads, IPT consecutive items per thread, tiles in descending
// order (the scan ended at the last tiles, which may still be in L2). A tile whose heavies
// (the owned ones and the next one) exceed walk_cap(T) returns at once: split_pack_kernel's
// chunked form builds it. The merge is that of split_pack_kernel's walk form:
//  (1) every light's deficit (small lights: 2^48 - rne(p 2^48); large lights: the true
//      deficit) goes to the stage slot of its item, and the thread sums them;
//  (2) a CTA scan of the two sums gives each thread's start on the tile's deficit line;
//  (3) thread t takes the heavies whose keys lie in [b_t, b_t+1) (b_t: its first light's key)
//      and walks its lights in order: heavies with key <= the light's key rank at that light
//      (their A_next is the light's key) and the light's alias is the first heavy left; the
//      light's row replaces its deficit in the stage slot;
//  (4) the owned heavies' rows are written (scattered), the staged light rows stored coalesced
//      (heavy positions skipped).
template <int NT, int IPT>
__global__ void __launch_bounds__(NT) pack_walk_kernel(const float* __restrict__ w, uint64_t n,
                                                       const BuildHeader* hdr, const TileStart* __restrict__ starts,
                                                       const uint32_t* __restrict__ heavy_item,
                                                       const uint64_t* __restrict__ heavy_E, uint32_t num_tiles,
                                                       wrs_alias_row* __restrict__ table) {
    constexpr int T = NT * IPT;
    constexpr int CW = walk_cap(T);
    static_assert(IPT >= 4 && IPT <= 32 && (IPT & (IPT - 1)) == 0, "items per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* sStage = reinterpret_cast<uint64_t*>(smem_raw);  // deficits, then rows
    uint64_t* sWk = sStage + T;                                 // heavy keys, then A_next keys
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
    if (m_w > (uint32_t)CW) return;  // the chunked form's tile
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
    const uint32_t sbase = (uint32_t)(tid * IPT);
    uint32_t lbits = 0, gbits = 0;  // bit k: item k is a light / a large light
    uint64_t asum = 0, lsum = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const float wk = x[k];
        const bool small = wk >= 0.0f && wk < cp.Hh;
        lbits |= (uint32_t)(wk >= 0.0f && !(wk > cp.H1)) << k;
        gbits |= (uint32_t)(wk >= cp.Hh && !(wk > cp.H1)) << k;
        const uint64_t d = small_deficit(__fmul_rn(wk, cp.R32));
        if (small) {
            asum += d;
            sStage[stage_pos<IPT>(sbase + k)] = d;
        }
    }
    for (uint32_t bits = gbits; bits; bits &= bits - 1) {  // large lights: true deficits (FP64)
        const int k = __ffs(bits) - 1;
        const uint64_t q = rare_q(__ldg(w + item0 + k), false, cp);
        sStage[stage_pos<IPT>(sbase + k)] = q;
        lsum += q;
    }
    // (2) the thread's start on the tile's deficit line
    const Scan2 ex = block_scan2<NT>(Scan2{asum, lsum}, s_scan);
    Dither dth;
    dth.c0 = st0.c0;
    dth.c0h = st0.c0 >> 24;
    const uint64_t D0 = dither_at(dth, ex.b);
    if (nH == 0) {
        // no heavy item anywhere: every row keeps itself
        uint64_t D = D0, lr = ex.b;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const uint32_t slot = stage_pos<IPT>(sbase + k);
            uint64_t row = ~0ull;
            if ((lbits >> k) & 1u) {
                float prob = __fmul_rn(x[k], cp.R32);
                if ((gbits >> k) & 1u) {
                    lr += sStage[slot];
                    const uint64_t D1 = dither_at(dth, lr);
                    prob = dithered_prob(D1 - D);
                    D = D1;
                }
                row = ((uint64_t)(item0 + k) << 32) | __float_as_uint(prob);
            }
            sStage[slot] = row;
        }
        __syncthreads();
    } else {
        // (3) this thread's lights merged with the heavies of its key range
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
            const uint32_t slot = stage_pos<IPT>(sbase + k);
            uint64_t row = ~0ull;
            if ((lbits >> k) & 1u) {
                const uint64_t key = sr + D;
                if (hk <= key) {
                    do {  // heavy a ranks at this light
                        sWk[a] = key;
                        ++a;
                        hk = a < a_end ? sWk[a] : ~0ull;
                    } while (hk <= key);
                    cur = a < m_w ? sWi[a] : last_heavy;
                }
                const uint64_t d = sStage[slot];
                float prob;
                if ((gbits >> k) & 1u) {  // the dithering after a large light
                    lr += d;
                    const uint64_t D1 = dither_at(dth, lr);
                    prob = dithered_prob(D1 - D);
                    D = D1;
                } else {
                    prob = __fmul_rn(x[k], cp.R32);
                    sr += d;
                }
                row = ((uint64_t)cur << 32) | __float_as_uint(prob);
            }
            sStage[slot] = row;
        }
        // the heavies left rank at the next thread's first light (the tile's end for the last)
        const uint64_t nxt = sr + D;
        for (; a < a_end; ++a) sWk[a] = nxt;
        __syncthreads();
        // (4) rows of the owned heavies
        const uint32_t m_own = g_hi - g_lo;
        for (uint32_t j = tid; j < m_own; j += NT) {
            const uint64_t nk = sWk[j];
            const u128 A_next = A_before + ((u128)nk << 16);
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

}  // namespace wrs
