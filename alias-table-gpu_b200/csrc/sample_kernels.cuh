// sample_kernels.cuh — alias-table samplers for sm_100a.
//
// Replaces SamplerGpuBasic (sampling/aliasTable/SamplerGpuBasic.cu:28-133) and
// SamplerGpuSectioned[Shared] (SamplerGpuSectioned.cu:19-166, SamplerGpuSectionedShared.cu:19-111).
// The reference draws an FP64 uniform u from clock-seeded XORWOW, takes row = (int)(u*N) and
// compares W/N * frac(u*N) with the row weight; it writes no output. Here every sample is
// a pure function of (seed, counter_base, output position) through Philox4x32-10:
//   block b = counter_base + s gives words x0..x3; row = floor((x1:x0) * len / 2^64) + offset
//   (a 64-bit uniform, so every row's share is exact to within len / 2^64),
//   coin = (x2 >> 8) 2^-24, result = coin < prob[row] ? row : alias[row]
// — the reference's decision (SamplerGpuBasic.cu:48-69) with frac := coin and
// weight := prob * W/N. Each sample is one 8-byte gather of a packed {prob, alias} row.
#pragma once

#include <cstdint>

#include "binomial.cuh"
#include "wrs_common.cuh"

namespace wrs {

__device__ __forceinline__ uint32_t alias_pick(const uint2 row, uint32_t r, uint32_t coin_bits) {
    return coin24(coin_bits) < __uint_as_float(row.x) ? r : row.y;
}

// A random row gather that asks L2 to fetch 64 bytes around the row (the prefetch-size
// qualifier of ld): without it a random 8-byte gather from a table larger than L2 cost about
// 107 bytes of DRAM reads (3.6 sectors), with it about 58. The sampling rate is the same
// either way (the random DRAM access rate bounds it), at half the DRAM traffic.
__device__ __forceinline__ uint2 ld_row_64B(const uint2* p) {
    uint2 v;
    asm("ld.global.nc.L2::64B.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}
// The same for the rejection sampler's random slot and acceptance gathers.
__device__ __forceinline__ uint32_t ld_u32_64B(const uint32_t* p) {
    uint32_t v;
    asm("ld.global.nc.L2::64B.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_f32_64B(const float* p) {
    float v;
    asm("ld.global.nc.L2::64B.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

// The rows and coins of the eight consecutive output positions whose Philox blocks start at b.
__device__ __forceinline__ void draw_octet(uint64_t b, uint32_t n, uint32_t k0, uint32_t k1, uint32_t (&rows)[8],
                                           uint32_t (&coins)[8]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const uint64_t bj = b + j;
        const Philox4 r = philox4x32_10((uint32_t)bj, (uint32_t)(bj >> 32), 0u, 0u, k0, k1);
        rows[j] = scale_u64(r.x[0], r.x[1], n);
        coins[j] = r.x[2];
    }
}

// Plain sampling: each thread handles octets of consecutive output positions (8 Philox
// blocks, 8 independent gathers in flight, two 16-byte stores). The next octet's Philox
// blocks are drawn while the current octet's gathers are in flight (drawn just before them,
// 2^28 samples from a 2^26-row table took 5.80 ms instead of 5.13 ms). The launch bounds allow
// about 60 registers (four CTAs per SM), with which the fold mode takes 4.73 ms instead of 5.26.
// MODE 0 writes sample s at out[s]; MODE 1 counts the samples instead (out[row] += 1 per
// sample); MODE 2 folds them into out[0] ^= (the XOR of all samples).
template <int MODE>
__global__ void __launch_bounds__(256, 4) sample_plain_kernel(const uint2* __restrict__ table, uint32_t n, uint64_t m,
                                                           uint32_t k0, uint32_t k1, uint64_t cbase,
                                                           uint32_t* __restrict__ out) {
    const uint64_t noct = (m + 7) >> 3;
    const uint64_t gsize = (uint64_t)gridDim.x * blockDim.x;
    const bool out_aligned = ((uintptr_t)out & 15u) == 0;
    uint32_t fold = 0;
    uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t rows[8], coins[8];
    if (g < noct) draw_octet(cbase + 8 * g, n, k0, k1, rows, coins);
    for (; g < noct; g += gsize) {
        uint2 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = ld_row_64B(table + rows[j]);
        uint32_t rows_n[8], coins_n[8];
        draw_octet(cbase + 8 * (g + gsize), n, k0, k1, rows_n, coins_n);  // unused past the last octet
        uint32_t res[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            res[j] = alias_pick(v[j], rows[j], coins[j]);
            rows[j] = rows_n[j];
            coins[j] = coins_n[j];
        }
        const uint64_t s0 = 8 * g;
        if constexpr (MODE == 2) {
#pragma unroll
            for (int j = 0; j < 8; ++j) fold ^= (s0 + j < m) ? res[j] : 0u;
            continue;
        }
        if constexpr (MODE == 1) {
            // lanes of the warp that drew the same row add together: one atomic per distinct
            // row (hot rows of skewed weights would otherwise serialise on one counter)
            const uint32_t act = __activemask();
            const int lane = threadIdx.x & 31;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const bool valid = s0 + j < m;
                const uint32_t key = valid ? res[j] : 0xffffffffu;
                const uint32_t peers = __match_any_sync(act, key);
                if (valid && lane == __ffs(peers) - 1) atomicAdd(out + res[j], (uint32_t)__popc(peers));
            }
            continue;
        }
        if (out_aligned && s0 + 8 <= m) {
            uint4* o4 = reinterpret_cast<uint4*>(out + s0);
            __stcs(o4, make_uint4(res[0], res[1], res[2], res[3]));
            __stcs(o4 + 1, make_uint4(res[4], res[5], res[6], res[7]));
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (s0 + j < m) out[s0 + j] = res[j];
        }
    }
    if constexpr (MODE == 2) {
        __shared__ uint32_t s_fold[8];
        fold = __reduce_xor_sync(0xffffffffu, fold);
        if ((threadIdx.x & 31) == 0) s_fold[threadIdx.x >> 5] = fold;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t f = 0;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) f ^= s_fold[i];
            atomicXor(out, f);
        }
    }
}

// The random-access ceiling of the plain sampler's table: the same 8-byte row gathers (with the
// .L2::64B prefetch size), eight in flight per thread, at rows from a cheap integer hash instead
// of Philox and with nothing written but one XOR word per CTA. A diagnostic, timed beside the
// sampler.
__device__ __forceinline__ uint32_t probe_row(uint64_t s, uint32_t n) {
    uint64_t z = s * 0x9E3779B97F4A7C15ull;
    z ^= z >> 29;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 32;
    return (uint32_t)__umul64hi(z, (uint64_t)n);
}
__global__ void __launch_bounds__(256, 4) gather_probe_kernel(const uint2* __restrict__ table, uint32_t n, uint64_t m,
                                                              uint64_t seed, uint32_t* __restrict__ sink) {
    const uint64_t noct = (m + 7) >> 3;
    const uint64_t gsize = (uint64_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < noct; g += gsize) {
        uint2 v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = ld_row_64B(table + probe_row(seed + 8 * g + j, n));
#pragma unroll
        for (int j = 0; j < 8; ++j) acc ^= v[j].x ^ v[j].y;
    }
    acc = __reduce_xor_sync(0xffffffffu, acc);
    if ((threadIdx.x & 31) == 0) atomicXor(sink, acc);
}

// Sectioned sampling: rows cut into K sections of S rows; section k receives an exact
// multinomial share of the m samples (binomial tree, section_count) and writes them at its
// output offset. CTA c handles sections c, c + gridDim.x, ... in that order, so the sections
// being sampled at any moment (grid size x section bytes) stay inside L2; with STAGE each
// section is first copied into shared memory and gathered from there. The counts and offsets
// of a CTA's sections are computed up front, one thread per section (each a walk down the
// binomial tree), so no thread waits for them between sections. Each thread draws eight
// consecutive output positions at a time (eight Philox blocks, eight gathers in flight).
// The staged form runs two CTAs per SM (at most 64 registers: the once-per-section binomial
// walk may spill, the sampling loop does not); the L2 form one CTA per SM, so that the
// sections in flight stay in L2. J output positions per thread and step (Philox blocks and
// gathers in flight): 8, or 4 for the L2 form's large sections (2^16 rows of a 2^26-row table:
// 3.77 ms instead of 4.28 for 2^30 samples; 2^14 rows: 3.37 instead of 3.20).
constexpr int kSectThreads = 512;
template <bool STAGE, int J>
__global__ void __launch_bounds__(kSectThreads, STAGE ? 2 : 1) sample_sectioned_kernel(const uint2* __restrict__ table, uint32_t n,
                                                                        uint64_t m, uint32_t S, uint32_t K,
                                                                        uint32_t k0, uint32_t k1, uint64_t cbase,
                                                                        uint32_t* __restrict__ out,
                                                                        uint64_t* __restrict__ counts_out) {
    static_assert(J == 4 || J == 8, "positions per step");
    extern __shared__ __align__(16) uint2 s_rows[];
    __shared__ uint64_t s_cnt[kSectThreads], s_off[kSectThreads];
    const uint32_t nsec = K > blockIdx.x ? (K - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
    const bool out16 = ((uintptr_t)out & 15u) == 0;
    for (uint32_t i0 = 0; i0 < nsec; i0 += kSectThreads) {
        {
            const uint32_t i = i0 + threadIdx.x;
            if (i < nsec) {
                const uint32_t sec = blockIdx.x + i * gridDim.x;
                uint64_t c, o;
                section_count(sec, K, S, n, m, k0, k1, cbase, &c, &o);
                s_cnt[threadIdx.x] = c;
                s_off[threadIdx.x] = o;
                if (counts_out) counts_out[sec] = c;
            }
        }
        __syncthreads();
        const uint32_t ni = min(nsec - i0, (uint32_t)kSectThreads);
        for (uint32_t ii = 0; ii < ni; ++ii) {
            const uint32_t sec = blockIdx.x + (i0 + ii) * gridDim.x;
            const uint32_t start = sec * S;
            const uint32_t len = (uint32_t)section_rows(sec, sec + 1, S, n);
            if (STAGE) {
                const uint4* src = reinterpret_cast<const uint4*>(table + start);
                uint4* dst = reinterpret_cast<uint4*>(s_rows);
                const uint32_t n16 = len >> 1;
                for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
                if ((len & 1u) && threadIdx.x == 0) s_rows[len - 1] = __ldg(table + start + len - 1);
                __syncthreads();
            }
            const uint64_t cnt = s_cnt[ii], off = s_off[ii];
            if (cnt > 0) {
                // output positions [off, off + cnt) in groups of J aligned to the global
                // position (position p draws Philox block cbase + p)
                const uint64_t p_lo = off & ~(uint64_t)(J - 1);
                const uint64_t ng = ((off + cnt - 1 - p_lo) / J) + 1;
                for (uint64_t gi = threadIdx.x; gi < ng; gi += blockDim.x) {
                    const uint64_t s0 = p_lo + (uint64_t)J * gi;  // output position of res[0]
                    uint32_t rows[J], coins[J];
#pragma unroll
                    for (int j = 0; j < J; ++j) {
                        const uint64_t bb = cbase + s0 + j;
                        const Philox4 r = philox4x32_10((uint32_t)bb, (uint32_t)(bb >> 32), 0u, 0u, k0, k1);
                        rows[j] = scale_u64(r.x[0], r.x[1], len);
                        coins[j] = r.x[2];
                    }
                    uint2 v[J];
#pragma unroll
                    for (int j = 0; j < J; ++j) v[j] = STAGE ? s_rows[rows[j]] : __ldg(table + start + rows[j]);
                    uint32_t res[J];
#pragma unroll
                    for (int j = 0; j < J; ++j) res[j] = alias_pick(v[j], start + rows[j], coins[j]);
                    if (s0 >= off && s0 + J <= off + cnt && out16) {
                        uint4* o4 = reinterpret_cast<uint4*>(out + s0);
#pragma unroll
                        for (int q = 0; q < J / 4; ++q)
                            __stcs(o4 + q, make_uint4(res[4 * q], res[4 * q + 1], res[4 * q + 2], res[4 * q + 3]));
                    } else {
#pragma unroll
                        for (int j = 0; j < J; ++j)
                            if (s0 + j >= off && s0 + j < off + cnt) out[s0 + j] = res[j];
                    }
                }
            }
            if (STAGE) __syncthreads();  // before the next section overwrites s_rows
        }
        __syncthreads();  // s_cnt / s_off are rewritten
    }
}

// Slot of a try: floor(u * |A| / 2^64) for the 64-bit uniform u = x1:x0, so that every slot
// of a large array gets its share to within |A| / 2^64 (a 32-bit uniform would leave shares
// differing by up to |A| / 2^32 relative: about 3% at 1.3e8 slots).
__device__ __forceinline__ uint32_t slot_of(uint32_t x0, uint32_t x1, uint32_t asz) { return scale_u64(x0, x1, asz); }

// ---------------------------------------------------------------- rejection sampling
// Replaces SamplerRejection::sample / SamplerRejectionGiveUp::sample
// (sampling/rejectionSampling/SamplerRejection.cu:17-35, SamplerRejectionGiveUp.cu:17-37):
// pick a uniform slot of A; a slot that is not its item's first is accepted, the first
// slot is accepted with probability frac(n w / W). Try t of sample s uses Philox block
// (counter_base + s, t, 0x52454a00): the slot from x0 and x1 (64 bits), the coin from x2. The first-slot test reads a flag bit in
// the slot itself instead of comparing with A[index - 1].
// J consecutive samples per thread with their tries interleaved: the J slot gathers of a try
// are in flight together, then the fraction gathers of the first slots among them.
constexpr int kRejJ = 4;
__global__ void __launch_bounds__(256) rejection_sample_kernel(const uint32_t* __restrict__ A,
                                                               const uint64_t* __restrict__ a_size_ptr,
                                                               const float* __restrict__ frac, uint64_t m,
                                                               uint32_t k0, uint32_t k1, uint64_t cbase,
                                                               uint32_t max_tries, uint32_t* __restrict__ out,
                                                               uint32_t* status) {
    constexpr int J = kRejJ;
    static_assert(J % 4 == 0, "16-byte stores");
    const uint64_t asz64 = *a_size_ptr;
    const uint64_t gsize = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool failed = false;
    if (asz64 == 0 || asz64 > 0xffffffffull) {  // no (or an unusable) slot array: nothing to sample
        for (uint64_t s = g0; s < m; s += gsize) out[s] = 0xffffffffu;
        if (status && blockIdx.x == 0 && threadIdx.x == 0) record_status(status, kErrCapacity);
        return;
    }
    const uint32_t asz = (uint32_t)asz64;
    const bool out16 = ((uintptr_t)out & 15u) == 0;
    for (uint64_t s0 = g0 * J; s0 < m; s0 += gsize * J) {
        uint32_t res[J];
        uint32_t open = 0;  // bit j: sample s0 + j still drawing
#pragma unroll
        for (int j = 0; j < J; ++j) {
            res[j] = 0xffffffffu;
            if (s0 + j < m) open |= 1u << j;
        }
        for (uint32_t t = 0; t < max_tries && open; ++t) {
            uint32_t xc[J], e[J];
#pragma unroll
            for (int j = 0; j < J; ++j) {
                if ((open >> j) & 1u) {
                    const uint64_t b = cbase + s0 + j;
                    const Philox4 r = philox4x32_10((uint32_t)b, (uint32_t)(b >> 32), t, 0x52454a00u, k0, k1);
                    xc[j] = r.x[2];
                    e[j] = ld_u32_64B(A + slot_of(r.x[0], r.x[1], asz));
                }
            }
            float f[J];
#pragma unroll
            for (int j = 0; j < J; ++j)
                if (((open >> j) & 1u) && (e[j] >> 31) != 0u) f[j] = ld_f32_64B(frac + (e[j] & 0x7fffffffu));
#pragma unroll
            for (int j = 0; j < J; ++j) {
                if ((open >> j) & 1u) {
                    if ((e[j] >> 31) == 0u || coin24(xc[j]) < f[j]) {
                        res[j] = e[j] & 0x7fffffffu;
                        open &= ~(1u << j);
                    }
                }
            }
        }
        if (open) failed = true;
        if (out16 && s0 + J <= m) {
#pragma unroll
            for (int q = 0; q < J / 4; ++q)
                reinterpret_cast<uint4*>(out + s0)[q] = make_uint4(res[4 * q], res[4 * q + 1], res[4 * q + 2], res[4 * q + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < J; ++j)
                if (s0 + j < m) out[s0 + j] = res[j];
        }
    }
    if (failed && status) record_status(status, kErrTooManyTries);
}

// ---------------------------------------------------------------- packed rejection slots
// The slot array with each first slot's acceptance fraction beside it: slots[s] = {A[s], the
// FP32 bits of frac[item] on the item's first slot, else 0}. A try then reads one 8-byte slot
// (one random gather) where the unpacked form reads the slot and, on a first slot, the item's
// fraction (a second random gather at another address).
__global__ void __launch_bounds__(256) rejection_pack_kernel(const uint32_t* __restrict__ A,
                                                             const uint64_t* __restrict__ a_size_ptr,
                                                             const float* __restrict__ frac, uint32_t n,
                                                             uint64_t a_capacity, uint2* __restrict__ slots) {
    const uint64_t asz = min(*a_size_ptr, a_capacity);
    const uint64_t gsize = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < asz; s += gsize) {
        const uint32_t e = A[s];
        const uint32_t item = e & 0x7fffffffu;
        const float f = ((e >> 31) != 0u && item < n) ? __ldg(frac + item) : 0.0f;
        slots[s] = make_uint2(e, __float_as_uint(f));
    }
}

// Rejection sampling from packed slots: the tries and decisions of rejection_sample_kernel
// (same Philox blocks, same slot, same comparison, so the same samples). A thread owns R
// consecutive samples of its CTA's chunk and keeps J of them in flight: a sample that is
// accepted (or runs out of tries) writes its result to shared memory and its place is taken by
// the thread's next sample, so that J gathers stay in flight until the thread's last samples;
// the chunk's results then go out coalesced.
constexpr int kRejPackedJ = 8;   // samples in flight per thread
constexpr int kRejPackedR = 32;  // samples per thread and chunk
__global__ void __launch_bounds__(256) rejection_sample_packed_kernel(const uint2* __restrict__ slots,
                                                                      uint64_t slot_capacity,
                                                                      const uint64_t* __restrict__ a_size_ptr,
                                                                      uint64_t m, uint32_t k0, uint32_t k1,
                                                                      uint64_t cbase, uint32_t max_tries,
                                                                      uint32_t* __restrict__ out, uint32_t* status) {
    constexpr int J = kRejPackedJ;
    constexpr uint32_t R = kRejPackedR;
    constexpr int NT = 256;
    __shared__ uint32_t s_res[NT * (R + 1)];  // thread t's sample k at t * (R + 1) + k (no bank conflicts)
    const uint64_t asz64 = *a_size_ptr;
    const uint64_t gsize = (uint64_t)gridDim.x * blockDim.x;
    bool failed = false;
    if (asz64 == 0 || asz64 > 0xffffffffull || asz64 > slot_capacity) {  // no (or an unusable) slot array
        for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gsize) out[s] = 0xffffffffu;
        if (status && blockIdx.x == 0 && threadIdx.x == 0) record_status(status, kErrCapacity);
        return;
    }
    const uint32_t asz = (uint32_t)asz64;
    const uint64_t chunk = (uint64_t)NT * R;
    for (uint64_t c0 = (uint64_t)blockIdx.x * chunk; c0 < m; c0 += (uint64_t)gridDim.x * chunk) {
        const uint64_t t0 = c0 + (uint64_t)threadIdx.x * R;  // the thread's first sample
        const uint32_t cnt = t0 < m ? (uint32_t)min((uint64_t)R, m - t0) : 0u;
        uint32_t* res = s_res + threadIdx.x * (R + 1);
        uint32_t idx[J], tr[J];  // the sample (within the thread's R; R = none) and its next try
        uint32_t next = 0;
#pragma unroll
        for (int j = 0; j < J; ++j) {
            idx[j] = next < cnt ? next++ : R;
            tr[j] = 0;
        }
        while (true) {
            bool any = false;
            uint32_t xc[J];
            uint2 v[J];
#pragma unroll
            for (int j = 0; j < J; ++j) {
                if (idx[j] < R) {
                    any = true;
                    const uint64_t b = t0 + idx[j] + cbase;
                    const Philox4 r = philox4x32_10((uint32_t)b, (uint32_t)(b >> 32), tr[j], 0x52454a00u, k0, k1);
                    xc[j] = r.x[2];
                    v[j] = ld_row_64B(slots + slot_of(r.x[0], r.x[1], asz));
                }
            }
            if (!any) break;
#pragma unroll
            for (int j = 0; j < J; ++j) {
                if (idx[j] < R) {
                    const uint32_t e = v[j].x;
                    bool done = true;
                    uint32_t val = e & 0x7fffffffu;
                    if ((e >> 31) != 0u && !(coin24(xc[j]) < __uint_as_float(v[j].y))) {  // rejected
                        if (++tr[j] < max_tries) {
                            done = false;
                        } else {
                            val = 0xffffffffu;
                            failed = true;
                        }
                    }
                    if (done) {
                        res[idx[j]] = val;
                        idx[j] = next < cnt ? next++ : R;
                        tr[j] = 0;
                    }
                }
            }
        }
        __syncthreads();
        const uint32_t n_out = (uint32_t)min(chunk, m - c0);
        for (uint32_t i = threadIdx.x; i < n_out; i += NT) out[c0 + i] = s_res[i + i / R];
        __syncthreads();  // before the next chunk's results
    }
    if (failed && status) record_status(status, kErrTooManyTries);
}

}  // namespace wrs
