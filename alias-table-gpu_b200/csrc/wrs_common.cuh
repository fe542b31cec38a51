// wrs_common.cuh — device building blocks shared by the build and sampling kernels.
//
//  * Q64.64 fixed point (unsigned __int128, value = raw / 2^64). All light-deficit and
//    heavy-excess prefix sums of the alias build are exact in this format, so every
//    comparison between a light's deficit interval and a heavy's excess interval gives
//    the same answer in every CTA that evaluates it.
//  * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
//    1, 2, 3", SC'11): the counter-based generator behind every sample.
//  * acquire/release flag access for the decoupled look-back scans.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "wrs.h"

namespace wrs {

typedef unsigned __int128 u128;

// ---------------------------------------------------------------- status word
// Device-side errors are recorded (first one wins) in a u32 that the host reads back.
enum : uint32_t {
    kOk = 0,
    kErrInvalidWeight = WRS_ERR_INVALID_WEIGHT,
    kErrZeroTotal = WRS_ERR_ZERO_TOTAL,
    kErrTimeout = WRS_ERR_DEVICE_TIMEOUT,
    kErrTooManyTries = WRS_ERR_TOO_MANY_TRIES,
    kErrCapacity = WRS_ERR_CAPACITY,
};

__device__ __forceinline__ void record_status(uint32_t* status, uint32_t code) {
    atomicCAS(status, 0u, code);
}

// Rejection slots of one item: c = floor(n w / W) + 1 and the first slot's acceptance
// frac(n w / W), with the FP64 expression of the reference's CalcNumOccurrencesOperator
// (construction/rejectionSampling/RejectionSampling.cu:26-33).
__device__ __forceinline__ void rej_item(float wf, double nd, double W, uint32_t& c, float& fr) {
    const double x = __ddiv_rn(__dmul_rn(nd, (double)wf), W);
    const double fl = floor(x);
    c = (uint32_t)fl + 1u;
    fr = __double2float_rn(x - fl);
}

__device__ __forceinline__ uint32_t load_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void store_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t load_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ---------------------------------------------------------------- Q64.64 helpers
__host__ __device__ __forceinline__ u128 q_make(uint64_t hi, uint64_t lo) {
    return ((u128)hi << 64) | (u128)lo;
}
__host__ __device__ __forceinline__ uint64_t q_hi(u128 x) { return (uint64_t)(x >> 64); }
__host__ __device__ __forceinline__ uint64_t q_lo(u128 x) { return (uint64_t)x; }
__host__ __device__ __forceinline__ u128 q_one() { return (u128)1 << 64; }

// Signed view of a Q64.64 difference (two's complement in 128 bits).
__host__ __device__ __forceinline__ bool q_is_negative(u128 x) { return (q_hi(x) >> 63) != 0; }

__host__ __device__ __forceinline__ uint64_t double_bits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    union {
        double d;
        uint64_t u;
    } c;
    c.d = x;
    return c.u;
#endif
}

// Non-negative finite double below 2^63 to Q64.64 by its bits; binary digits below 2^-64
// are truncated (exact for every double >= 2^-11 and for every multiple of 2^-64).
// Subnormal doubles map to 0.
__host__ __device__ __forceinline__ u128 q_from_double(double x) {
    const uint64_t b = double_bits(x);
    const int e = (int)((b >> 52) & 0x7ff);
    if (e == 0) return 0;
    const u128 m = (u128)((b & 0xfffffffffffffull) | 0x10000000000000ull);  // 53-bit mantissa
    const int sh = e - 1075 + 64;  // value = m * 2^(e-1075)
    if (sh >= 0) return m << sh;
    if (sh <= -53) return 0;
    return m >> (-sh);
}

// round(x * 2^fb) (ties away from zero) for a finite double x >= 0, from its bits; the
// caller keeps the result below 2^62. Subnormal inputs give 0. Branch-free: with
// t = mantissa * 2^10 and sh = 1085 - fb - exponent (>= 1), the result is
// ((t >> (sh - 1)) + 1) >> 1, or 0 when sh > 63.
__host__ __device__ __forceinline__ uint64_t fixq(double x, int fb) {
    const uint64_t b = double_bits(x);
    const int e = (int)((b >> 52) & 0x7ff);
    const uint64_t t = ((b & 0xfffffffffffffull) | 0x10000000000000ull) << 10;
    const int sh = 1085 - fb - e;
    const uint64_t r = ((t >> ((sh - 1) & 63)) + 1) >> 1;
    return (e == 0 || sh > 63) ? 0ull : r;
}

// Q64.64 (interpreted as signed) to double. Separate multiply and add (never fused), so
// the CPU oracle reproduces the value bit for bit.
__host__ __device__ __forceinline__ double q_to_double_signed(u128 x) {
    bool neg = q_is_negative(x);
    u128 m = neg ? (u128)0 - x : x;
#ifdef __CUDA_ARCH__
    double v = __dadd_rn((double)q_hi(m), __dmul_rn((double)q_lo(m), 5.421010862427522170037e-20));  // 2^-64
#else
    double v = (double)q_hi(m) + (double)q_lo(m) * 5.421010862427522170037e-20;
#endif
    return neg ? -v : v;
}

// Round a Q64.64 value to the nearest multiple of 2^-24 (ties up): the grid of FP32
// values in [1/2, 1], used to dither the stored probabilities of light items.
__host__ __device__ __forceinline__ u128 q_round24(u128 x) {
    const u128 half = (u128)1 << 39;
    const u128 mask = ~(((u128)1 << 40) - 1);
    return (x + half) & mask;
}

// Heavy-excess prefix correction: E -> E + sign * floor(E * |N| / 2^64). Monotone
// non-decreasing in E for |N| <= 2^62 and per-heavy excess >= 2^-52, which keeps the
// corrected excess line sorted.
__host__ __device__ __forceinline__ u128 q_scale_excess(u128 e, int64_t n_fix) {
    if (n_fix == 0) return e;
    const uint64_t an = n_fix < 0 ? (uint64_t)(-(n_fix + 1)) + 1u : (uint64_t)n_fix;
    const uint64_t ehi = q_hi(e), elo = q_lo(e);
#ifdef __CUDA_ARCH__
    const uint64_t mh = __umul64hi(elo, an);
#else
    const uint64_t mh = (uint64_t)(((u128)elo * an) >> 64);
#endif
    const u128 corr = (u128)ehi * an + mh;
    return n_fix < 0 ? e - corr : e + corr;
}

// N = round(2^64 * (A_total - E_total) / E_total), clamped to |N| <= 2^62 (a relative
// correction of at most 1/4; larger mismatches only arise from degenerate inputs).
__host__ __device__ __forceinline__ int64_t excess_correction(u128 a_total, u128 e_total) {
    if (e_total == 0) return 0;
    const double d = q_to_double_signed(a_total - e_total);
    const double e = q_to_double_signed(e_total);
    double r = d / e;
    if (r > 0.25) r = 0.25;
    if (r < -0.25) r = -0.25;
    const double s = r * 18446744073709551616.0;
#ifdef __CUDA_ARCH__
    return __double2ll_rn(s);
#else
    return (int64_t)__builtin_llrint(s);
#endif
}

// ---------------------------------------------------------------- Philox4x32-10
struct Philox4 {
    uint32_t x[4];
};

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
    lo = a * b;
    hi = __umulhi(a, b);
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    lo = (uint32_t)p;
    hi = (uint32_t)(p >> 32);
#endif
}

// Philox4x32 with 10 rounds; multipliers and Weyl increments from the SC'11 paper.
__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                         uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c0, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c2, hi1, lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    Philox4 r;
    r.x[0] = c0;
    r.x[1] = c1;
    r.x[2] = c2;
    r.x[3] = c3;
    return r;
}

// index in [0, len) from the 64-bit uniform u = x1:x0, exactly floor(u * len / 2^64): every
// index gets its share to within len / 2^64 (a 32-bit uniform would leave shares differing by
// up to len / 2^32 relative, about 2% at 1e8 rows).
__host__ __device__ __forceinline__ uint32_t scale_u64(uint32_t x0, uint32_t x1, uint32_t len) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__umul64hi(((uint64_t)x1 << 32) | x0, (uint64_t)len);
#else
    return (uint32_t)(((unsigned __int128)((((uint64_t)x1) << 32) | x0) * len) >> 64);
#endif
}

// coin in [0, 1) with 24 random bits.
__host__ __device__ __forceinline__ float coin24(uint32_t x) {
    return (float)(x >> 8) * 5.9604644775390625e-8f;  // 2^-24
}

// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ u128 shfl_up_u128(u128 v, int delta) {
    uint64_t hi = __shfl_up_sync(0xffffffffu, q_hi(v), delta);
    uint64_t lo = __shfl_up_sync(0xffffffffu, q_lo(v), delta);
    return q_make(hi, lo);
}
__device__ __forceinline__ u128 shfl_xor_u128(u128 v, int mask) {
    uint64_t hi = __shfl_xor_sync(0xffffffffu, q_hi(v), mask);
    uint64_t lo = __shfl_xor_sync(0xffffffffu, q_lo(v), mask);
    return q_make(hi, lo);
}

// ---------------------------------------------------------------- programmatic dependent launch
// A kernel of a build's chain is launched with programmatic stream serialisation (launch_pdl):
// the launch is staged while the previous kernel runs, and the kernel's CTAs are scheduled as
// the previous kernel's CTAs exit (no explicit trigger: one at the start of each kernel let the
// dependents' CTAs sit on the SMs early and cost more than it saved). Every such kernel starts
// with pdl_enter(), which waits until the previous kernel has completed and its writes are
// visible (griddepcontrol.wait; immediate for a kernel launched without the attribute). Every
// kernel of a chain waits before anything else, early exits included, so that the completion of
// a kernel implies the completion of all kernels before it.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---------------------------------------------------------------- bounded waits
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any legitimate wait

// Limits of the bounded device waits, passed to every kernel that waits: a look-back wait
// gives up after limit_ns (records WRS_ERR_DEVICE_TIMEOUT and returns); look-back block or
// tile `hold` (~0u: none) publishes nothing, so that its successors' waits run out — the
// failure-detection tests' way of making a wait that nothing ends.
struct WaitCfg {
    uint64_t limit_ns;
    uint32_t hold;
    uint32_t pad;
};
__device__ __forceinline__ bool wait_expired(uint64_t t_start, const WaitCfg& wc) {
    return global_ns() - t_start > wc.limit_ns;
}

}  // namespace wrs
