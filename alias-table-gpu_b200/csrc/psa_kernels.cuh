// psa_kernels.cuh — the PSA+ build (WRS_METHOD_PSA_PLUS) for sm_100a.
//
// The reference's PSA+ (AliasTableSplitGpu::psaPlus + PsaPlusNormal::kernel,
// construction/aliasTable/buildMethod/AliasTableSplitGpu.cu:342-386,
// construction/aliasTable/psaPlus/PsaPlusNormal.cu:12-152) packs every section greedily on
// its own first and sends what it cannot finish (with one residual-weight item per packer)
// through the global split/pack. Here the sections are the build's tiles, and the local pass
// works on the split build's exact lines restricted to the tile and measured from the tile's
// start: the deficit line A (with its dithering) and the corrected excess line E~. In a tile
// with total deficit D and total excess Et:
//   * a light is finished when a heavy of the tile has E~ > A (alias: the first such heavy);
//   * a heavy with E~ <= D is finished with r = 1 + E~ - A_next (A_next = the first light
//     start >= E~, else D) and aliases the tile's next heavy; the tile's last heavy, if
//     finished, keeps r but waits for its alias: it becomes the tile's first leftover light,
//     with deficit A_next - E~ rounded up to the 2^-48 grid;
//   * lights starting at or after Et are leftover lights; the first heavy with E~ > D is a
//     leftover heavy with residual excess E~ - D, the heavies after it leftover heavies.
// The leftovers (per tile in slots: lights from the front, heavies from the back) then go
// through the split passes as lists: tile prefixes of their counts and sums, a heavy list of
// the leftover heavies, the tile links, and split_pack in its leftover mode.
#pragma once

#include "build_kernels.cuh"

namespace wrs {

// ceil(x / 2^-48) clamped to [0, 2^64 - 1]: the key of an excess value (Q64.64), so that
// key(light) < key(x) exactly when A < x for a light start A on the 2^-48 grid.
__device__ __forceinline__ uint64_t excess_key(u128 x) {
    const u128 d = x + 0xffff;
    return (q_hi(d) >> 16) ? ~0ull : (uint64_t)(d >> 16);
}

// Shared memory of the local pass: light keys (u64 x T), heavy keys (u64 x T), heavies'
// local E~ (u128 x T), heavy items (u32 x T).
__host__ __device__ constexpr size_t psa_local_smem_bytes(int T) {
    return (size_t)T * (2 * sizeof(uint64_t) + sizeof(u128) + sizeof(uint32_t));
}

template <int NT, int IPT>
__global__ void __launch_bounds__(NT) psa_local_kernel(const float* __restrict__ w, uint64_t n,
                                                       const BuildHeader* hdr, const TileVals* incl,
                                                       wrs_alias_row* __restrict__ table, LeftSlot* slots,
                                                       TileVals* agg2, BuildHeader* hdr2) {
    pdl_enter();
    constexpr int T = NT * IPT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u128* sHe = reinterpret_cast<u128*>(smem_raw);
    uint64_t* sLkey = reinterpret_cast<uint64_t*>(sHe + T);
    uint64_t* sHkey = sLkey + T;
    uint32_t* sHitem = reinterpret_cast<uint32_t*>(sHkey + T);
    uint64_t* sSlotQ = sHkey;  // own-tile phase: large lights' quantities per item slot
    uint64_t* sStage = sHkey;  // row phase: staged light rows
    __shared__ Scan3 s_scan3[NT / 32];
    __shared__ Scan3 s_scanh[NT / 32];
    __shared__ uint64_t s_convd;

    const int tid = threadIdx.x;
    const uint32_t tile = blockIdx.x;
    float x[IPT];
    load_items<NT, IPT>(w, n, tile, tid, x);
    const uint32_t st = earlier_status(hdr);
    if (st != 0) {
        if (tid == 0) record_status(&hdr2->status, st);  // the leftover passes stop too
        return;
    }
    const ClassParams cp = load_class_params(hdr);
    const int64_t nfix = __ldg(&hdr->nfix);
    const TileVals before = tile ? ldcg_tilevals(incl + tile - 1) : tv_zero();
    const u128 A_before = deficit_line(before);
    const u128 A_after = deficit_line(ldcg_tilevals(incl + tile));
    const uint64_t D48 = (uint64_t)((A_after - A_before) >> 16);  // the tile's deficit, Q16.48
    const u128 Eb = q_scale_excess(before.E, nfix);
    const uint32_t item0 = (uint32_t)((uint64_t)tile * T + (uint64_t)tid * IPT);

    // ---- lights: keys as in split_pack
    float pk[IPT];
    uint32_t lbits = 0, gbits = 0, hbits = 0;
    uint64_t asum = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const float wk = x[k];
        const bool small = wk >= 0.0f && wk < cp.Hh;
        const float p = __fmul_rn(wk, cp.R32);
        pk[k] = p;
        asum += small ? small_deficit(p) : 0ull;
        lbits |= (uint32_t)(wk >= 0.0f && !(wk > cp.H1)) << k;
        gbits |= (uint32_t)(wk >= cp.Hh && !(wk > cp.H1)) << k;
        hbits |= (uint32_t)(wk > cp.H1) << k;
    }
    // the rare items' FP64 quantities, from the weights in registers
    uint64_t lsum = 0, hsum = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        if ((gbits >> k) & 1u) {
            const uint64_t q = rare_q(x[k], false, cp);
            sSlotQ[tid * IPT + k] = q;
            lsum += q;
        }
        if ((hbits >> k) & 1u) hsum += rare_q(x[k], true, cp);
    }
    const uint32_t nl = (uint32_t)__popc(lbits), nh = (uint32_t)__popc(hbits);
    Scan3 tot_l, tot_h;
    const Scan3 ex = block_scan3<NT>(Scan3{nl, asum, lsum}, s_scan3, tot_l);
    const Scan3 exh = block_scan3<NT>(Scan3{nh, hsum, 0ull}, s_scanh, tot_h);
    const uint32_t nLt = tot_l.c, nHt = tot_h.c;
    const uint32_t l0 = ex.c;
    Dither dth = make_dither(before.L);
    const uint64_t D0 = dither_at(dth, ex.b);
    {
        uint64_t sr = ex.a, D = D0, lr = ex.b;
        uint32_t li = l0;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            const bool light = (lbits >> k) & 1u;
            if (light) sLkey[lkey_slot(li)] = sr + D;
            li += light ? 1u : 0u;
            sr += (light && !((gbits >> k) & 1u)) ? small_deficit(pk[k]) : 0ull;
            if ((gbits >> k) & 1u) {  // the dithering after a large light
                lr += sSlotQ[tid * IPT + k];
                const uint64_t D1 = dither_at(dth, lr);
                pk[k] = dithered_prob(D1 - D);
                D = D1;
            }
        }
    }
    __syncthreads();  // light keys complete; the slot quantities are free
    // ---- heavies: their corrected excess ends, measured from the tile's start
    {
        uint64_t er = exh.a;
        uint32_t hj = exh.c;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            if (!((hbits >> k) & 1u)) continue;
            er += rare_q(x[k], true, cp);
            const u128 El = q_scale_excess(before.E + ((u128)er << 40), nfix) - Eb;
            sHe[hj] = El;
            sHkey[hj] = excess_key(El);
            sHitem[hj] = item0 + k;
            ++hj;
        }
    }
    if (tid == 0) s_convd = 0;
    __syncthreads();
    const u128 Et = nHt ? sHe[nHt - 1] : (u128)0;
    const u128 D128 = (u128)D48 << 16;
    // first light starting at or after Et (lights before it are finished)
    uint32_t L0;
    {
        const uint64_t kEt = excess_key(Et);
        uint32_t lo = 0, hi = nLt;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sLkey[lkey_slot(mid)] < kEt) lo = mid + 1; else hi = mid;
        }
        L0 = lo;
    }
    // first heavy with E~ > D (heavies before it are finished)
    uint32_t Js;
    {
        uint32_t lo = 0, hi = nHt;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sHkey[mid] <= D48) lo = mid + 1; else hi = mid;
        }
        Js = lo;
    }
    const bool conv = nHt > 0 && Js == nHt;
    LeftSlot* ts = slots + (uint64_t)tile * T;
    for (uint32_t j = tid; j < nHt; j += NT) {
        const u128 El = sHe[j];
        if (j < Js) {
            uint32_t lo = 0, hi = nLt;  // the first light whose key is not below the heavy's
            const uint64_t kh = sHkey[j];
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (sLkey[lkey_slot(mid)] < kh) lo = mid + 1; else hi = mid;
            }
            const u128 A_next = (lo < nLt) ? ((u128)sLkey[lkey_slot(lo)] << 16) : D128;
            const float prob = heavy_row_prob(q_one() + El - A_next);
            if (j + 1 < nHt) {
                wrs_alias_row r;
                r.prob = prob;
                r.alias = sHitem[j + 1];
                table[sHitem[j]] = r;
            } else {  // the tile's last heavy, finished: the first leftover light
                const u128 g = ((u128)1 << 16) - 1;
                const uint64_t d = (uint64_t)(((A_next - El + g) & ~g) >> 16);
                LeftSlot sl;
                sl.item = sHitem[j];
                sl.prob_bits = __float_as_uint(prob);
                sl.lo = d;
                sl.hi = 0;
                ts[0] = sl;
                s_convd = d;
            }
        } else {
            const u128 e = (j == Js) ? El - D128 : El - sHe[j - 1];
            LeftSlot sl;
            sl.item = sHitem[j];
            sl.prob_bits = 0;
            sl.lo = q_lo(e);
            sl.hi = q_hi(e);
            ts[T - (nHt - j)] = sl;
        }
    }
    // ---- lights: finished ones staged for the row write, leftovers to the slots
    {
        uint32_t li = l0, j = 0;
        bool found = false;
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
            uint64_t row = ~0ull;
            if ((lbits >> k) & 1u) {
                const uint64_t kl = sLkey[lkey_slot(li)];
                if (li < L0) {
                    if (!found) {  // the first heavy whose key exceeds the light's
                        uint32_t lo = 0, hi = nHt;
                        while (lo < hi) {
                            const uint32_t mid = (lo + hi) >> 1;
                            if (sHkey[mid] > kl) hi = mid; else lo = mid + 1;
                        }
                        j = lo;
                        found = true;
                    }
                    while (sHkey[j] <= kl) ++j;  // a heavy with a larger key exists (li < L0)
                    row = ((uint64_t)sHitem[j] << 32) | __float_as_uint(pk[k]);
                } else {
                    const uint64_t kn = (li + 1 < nLt) ? sLkey[lkey_slot(li + 1)] : D48;
                    LeftSlot sl;
                    sl.item = item0 + k;
                    sl.prob_bits = __float_as_uint(pk[k]);
                    sl.lo = kn - kl;
                    sl.hi = 0;
                    ts[(conv ? 1u : 0u) + li - L0] = sl;
                }
                ++li;
            }
            x[k] = __uint_as_float((uint32_t)(row >> 32));  // reuse as the staged alias
            pk[k] = __uint_as_float((uint32_t)row);
        }
    }
    __syncthreads();  // every read of the heavy keys is done; sStage overlays them
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const uint64_t row = ((uint64_t)__float_as_uint(x[k]) << 32) | __float_as_uint(pk[k]);
        sStage[stage_pos<IPT>((uint32_t)(tid * IPT + k))] = row;
    }
    __syncthreads();
    uint64_t* out = reinterpret_cast<uint64_t*>(table) + (uint64_t)tile * T;
    const uint32_t cnt = (uint32_t)min((uint64_t)T, n - (uint64_t)tile * T);
    for (uint32_t i = tid; i < cnt; i += NT) {
        const uint64_t row = sStage[stage_pos<IPT>(i)];
        if (row != ~0ull) out[i] = row;
    }
    if (tid == 0) {
        const uint64_t kL0 = (L0 < nLt) ? sLkey[lkey_slot(L0)] : D48;
        TileVals a;
        a.nL = (conv ? 1u : 0u) + (nLt - L0);
        a.nH = nHt - Js;
        a.first_heavy = 0xffffffffu;
        a.last_heavy = 0xffffffffu;
        a.S = (u128)(s_convd + (D48 - kL0)) << 16;
        a.L = 0;
        a.E = (Js < nHt) ? Et - D128 : (u128)0;
        agg2[tile] = a;
    }
}

// Leftover heavy list: one tile per warp; the tile's leftover heavies (slots from the back),
// their excess prefix from the leftover tile prefixes, corrected by the leftover excess
// correction, written at their index among all leftover heavies.
__device__ __forceinline__ u128 warp_excl_scan_u128(u128 v, u128& total) {
    const int lane = threadIdx.x & 31;
    u128 inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const u128 o = shfl_up_u128(inc, off);
        if (lane >= off) inc += o;
    }
    total = q_make(__shfl_sync(0xffffffffu, q_hi(inc), 31), __shfl_sync(0xffffffffu, q_lo(inc), 31));
    return inc - v;
}

template <int T>
__global__ void __launch_bounds__(128) psa_heavy_list_kernel(const BuildHeader* hdr2, const TileVals* agg2,
                                                             const TileVals* incl2, const LeftSlot* slots,
                                                             uint32_t num_tiles, uint32_t* heavy_item,
                                                             uint4* heavy_E) {
    pdl_enter();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t u = blockIdx.x * 4 + warp;
    if (u >= num_tiles || earlier_status(hdr2) != 0) return;
    const uint32_t m = __ldcg(&agg2[u].nH);
    if (m == 0) return;
    const int64_t nfix = __ldg(&hdr2->nfix);
    const uint32_t g0 = u ? __ldcg(&incl2[u - 1].nH) : 0u;
    const u128 Eb = u ? ldcg_E(incl2 + u - 1) : (u128)0;
    const LeftSlot* hs = slots + (uint64_t)u * T + (T - m);
    const uint32_t per = (m + 31) / 32;
    const uint32_t j0 = min(m, (uint32_t)lane * per), j1 = min(m, j0 + per);
    u128 sum = 0;
    for (uint32_t j = j0; j < j1; ++j) sum += q_make(hs[j].hi, hs[j].lo);
    u128 tot;
    u128 er = warp_excl_scan_u128(sum, tot);
    for (uint32_t j = j0; j < j1; ++j) {
        er += q_make(hs[j].hi, hs[j].lo);
        heavy_item[g0 + j] = hs[j].item;
        store_u128(heavy_E + g0 + j, q_scale_excess(Eb + er, nfix));
    }
}

// Copies the leftover passes' status into the build's header (read by wrs_scratch_status).
__global__ void copy_status_kernel(const BuildHeader* from, BuildHeader* to) {
    pdl_enter();
    const uint32_t st = from->status;
    if (st != 0) record_status(&to->status, st);
}

}  // namespace wrs
