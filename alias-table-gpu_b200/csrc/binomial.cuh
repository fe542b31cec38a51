// binomial.cuh — exact, bit-reproducible binomial variates for the sectioned sampler.
//
// The reference splits samples across table sections with a normal approximation of the
// binomial, truncated to int (utils/Prng.cuh:190-199, sampling/aliasTable/SamplerGpuSectioned.cu:58-96),
// which is neither exact nor reproducible (clock64-seeded XORWOW). Here the per-section
// counts come from a binary tree of exact Binomial(count, rows_left / rows_node) draws:
//   * n*p >= 10: BTRD, the transformed-rejection-with-decomposition method of
//     W. Hörmann, "The generation of binomial random variates", J. Statist. Comput. Simul.
//     46 (1993) 101-110;
//   * n*p < 10: geometric waiting times (count successes by jumping over failures).
// Uniforms come from Philox4x32-10. Every floating-point operation is an explicit
// correctly-rounded IEEE operation (no contraction, a self-contained logarithm), so the CPU
// oracle reproduces every draw bit for bit.
#pragma once

#include <cstdint>

#include "wrs_common.cuh"

namespace wrs {

#ifdef __CUDA_ARCH__
#define WRS_DMUL(a, b) __dmul_rn((a), (b))
#define WRS_DADD(a, b) __dadd_rn((a), (b))
#define WRS_DSUB(a, b) __dsub_rn((a), (b))
#define WRS_DDIV(a, b) __ddiv_rn((a), (b))
#define WRS_DSQRT(a) __dsqrt_rn((a))
#else
#define WRS_DMUL(a, b) ((a) * (b))
#define WRS_DADD(a, b) ((a) + (b))
#define WRS_DSUB(a, b) ((a) - (b))
#define WRS_DDIV(a, b) ((a) / (b))
#define WRS_DSQRT(a) __builtin_sqrt((a))
#endif

__host__ __device__ __forceinline__ double bits_double(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    union {
        uint64_t u;
        double d;
    } c;
    c.u = b;
    return c.d;
#endif
}

// 2 * atanh(s) = 2 (s + s^3/3 + s^5/5 + ...), |s| <= 0.1716 (12 terms).
__host__ __device__ __forceinline__ double det_2atanh(double s) {
    const double z = WRS_DMUL(s, s);
    double p = 1.0 / 25.0;
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 23.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 21.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 19.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 17.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 15.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 13.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 11.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 9.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 7.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 5.0);
    p = WRS_DADD(WRS_DMUL(p, z), 1.0 / 3.0);
    const double s2 = WRS_DADD(s, s);
    return WRS_DADD(s2, WRS_DMUL(WRS_DMUL(s2, z), p));
}

// Natural logarithm of x >= 0 (returns -inf for 0): x = m * 2^e, m in (sqrt(2)/2, sqrt(2)],
// log m = 2 atanh((m - 1) / (m + 1)).
__host__ __device__ __forceinline__ double det_log(double x) {
    if (!(x > 0.0)) return -1.0 / 0.0;
    uint64_t b = double_bits(x);
    int e = (int)((b >> 52) & 0x7ff);
    if (e == 0) {  // subnormal: scale by 2^54 (exact)
        x = WRS_DMUL(x, 18014398509481984.0);
        b = double_bits(x);
        e = (int)((b >> 52) & 0x7ff) - 54;
    }
    int ex = e - 1023;
    double m = bits_double((b & 0xfffffffffffffull) | (1023ull << 52));  // [1, 2)
    if (m > 1.4142135623730951) {
        m = WRS_DMUL(m, 0.5);
        ex += 1;
    }
    const double f = WRS_DSUB(m, 1.0);
    const double s = WRS_DDIV(f, WRS_DADD(2.0, f));
    const double lm = det_2atanh(s);
    return WRS_DADD(WRS_DMUL((double)ex, 0.6931471805599453094), lm);
}

// log(1 - p) for p in [0, 1).
__host__ __device__ __forceinline__ double det_log1m(double p) {
    if (p < 0.25) {
        // 1 - p = (1 - s) / (1 + s) with s = p / (2 - p): log(1 - p) = -2 atanh(s)
        const double s = WRS_DDIV(p, WRS_DSUB(2.0, p));
        return -det_2atanh(s);
    }
    return det_log(WRS_DSUB(1.0, p));
}

// 53-bit uniforms from Philox words: [0, 1) and (0, 1].
__host__ __device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
    const uint64_t v = (((uint64_t)hi << 21) ^ ((uint64_t)lo >> 11)) & ((1ull << 53) - 1);
    return (double)v * 1.1102230246251565404e-16;
}
__host__ __device__ __forceinline__ double u53_open0(uint32_t hi, uint32_t lo) {
    const uint64_t v = (((uint64_t)hi << 21) ^ ((uint64_t)lo >> 11)) & ((1ull << 53) - 1);
    return (double)(v + 1) * 1.1102230246251565404e-16;
}

// Stirling-series correction fc(k) = log(k!) - [(k + 1/2) log(k + 1) - (k + 1) + log(2 pi)/2].
__host__ __device__ __forceinline__ double stirling_fc(double k) {
    if (k < 10.0) {
        // exact factorial (k <= 9), logs by det_log
        double f = 1.0;
        for (double i = 2.0; i <= k; i = WRS_DADD(i, 1.0)) f = WRS_DMUL(f, i);
        const double k1 = WRS_DADD(k, 1.0);
        const double half_log_2pi = WRS_DMUL(0.5, det_log(6.283185307179586477));
        double r = det_log(f);
        r = WRS_DSUB(r, WRS_DMUL(WRS_DADD(k, 0.5), det_log(k1)));
        r = WRS_DADD(r, k1);
        r = WRS_DSUB(r, half_log_2pi);
        return r;
    }
    const double k1 = WRS_DADD(k, 1.0);
    const double k1sq = WRS_DMUL(k1, k1);
    double t = WRS_DSUB(1.0 / 360.0, WRS_DDIV(WRS_DDIV(1.0 / 1260.0, k1sq), 1.0));
    t = WRS_DSUB(1.0 / 12.0, WRS_DDIV(t, k1sq));
    return WRS_DDIV(t, k1);
}

// Philox counter domain of the tree draws: c3 = (iteration << 8) | 0xA5.
struct BinomStream {
    uint32_t k0, k1;  // key
    uint32_t c0, c1;  // counter_base
    uint32_t node;    // tree node id
};

__host__ __device__ __forceinline__ Philox4 binom_draw_words(const BinomStream& st, uint32_t iter) {
    return philox4x32_10(st.c0, st.c1, st.node, (iter << 8) | 0xA5u, st.k0, st.k1);
}

// Binomial(n, p) for 0 <= p <= 1/2 with n*p < 10: count successes by geometric jumps.
__host__ __device__ __forceinline__ uint64_t binom_small(uint64_t n, double p, const BinomStream& st) {
    if (n == 0 || !(p > 0.0)) return 0;
    const double l1m = det_log1m(p);  // < 0
    uint64_t x = 0;
    double pos = 0.0;
    const double nd = (double)n;
    for (uint32_t it = 0; it < 4096; ++it) {
        const Philox4 r = binom_draw_words(st, it);
        for (int h = 0; h < 2; ++h) {
            const double u = u53_open0(r.x[2 * h], r.x[2 * h + 1]);
            const double g = WRS_DADD(floor(WRS_DDIV(det_log(u), l1m)), 1.0);  // trials to next success
            pos = WRS_DADD(pos, g);
            if (pos > nd) return x;
            ++x;
        }
    }
    return x;  // unreachable in practice (expected n*p + 1 < 11 jumps)
}

// Binomial(n, p) for 0 < p <= 1/2 and n*p >= 10 (BTRD).
__host__ __device__ __forceinline__ uint64_t binom_btrd(uint64_t n, double p, const BinomStream& st) {
    const double nd = (double)n;
    const double q = WRS_DSUB(1.0, p);
    const double m = floor(WRS_DMUL(WRS_DADD(nd, 1.0), p));
    const double r = WRS_DDIV(p, q);
    const double nr = WRS_DMUL(WRS_DADD(nd, 1.0), r);
    const double npq = WRS_DMUL(WRS_DMUL(nd, p), q);
    const double spq = WRS_DSQRT(npq);
    const double b = WRS_DADD(1.15, WRS_DMUL(2.53, spq));
    const double a = WRS_DADD(WRS_DADD(-0.0873, WRS_DMUL(0.0248, b)), WRS_DMUL(0.01, p));
    const double c = WRS_DADD(WRS_DMUL(nd, p), 0.5);
    const double alpha = WRS_DMUL(WRS_DADD(2.83, WRS_DDIV(5.1, b)), spq);
    const double vr = WRS_DSUB(0.92, WRS_DDIV(4.2, b));
    const double urvr = WRS_DMUL(0.86, vr);
    for (uint32_t it = 0; it < 256; ++it) {
        const Philox4 w = binom_draw_words(st, it);
        double v = u53(w.x[0], w.x[1]);
        double u;
        if (v <= urvr) {
            u = WRS_DSUB(WRS_DDIV(v, vr), 0.43);
            const double au = u < 0.0 ? -u : u;
            const double kk = floor(WRS_DADD(WRS_DMUL(WRS_DADD(WRS_DDIV(WRS_DMUL(2.0, a), WRS_DSUB(0.5, au)), b), u), c));
            if (kk < 0.0) return 0;
            if (kk > nd) return n;
            return (uint64_t)kk;
        }
        if (v >= vr) {
            u = WRS_DSUB(u53(w.x[2], w.x[3]), 0.5);
        } else {
            u = WRS_DSUB(WRS_DDIV(v, vr), 0.93);
            u = WRS_DSUB(u < 0.0 ? -0.5 : 0.5, u);
            v = WRS_DMUL(u53(w.x[2], w.x[3]), vr);
        }
        const double au = u < 0.0 ? -u : u;
        const double us = WRS_DSUB(0.5, au);
        const double kk = floor(WRS_DADD(WRS_DMUL(WRS_DADD(WRS_DDIV(WRS_DMUL(2.0, a), us), b), u), c));
        if (kk < 0.0 || kk > nd) continue;
        v = WRS_DDIV(WRS_DMUL(v, alpha), WRS_DADD(WRS_DDIV(a, WRS_DMUL(us, us)), b));
        const double km = kk > m ? WRS_DSUB(kk, m) : WRS_DSUB(m, kk);
        if (km <= 15.0) {
            double f = 1.0;
            if (m < kk) {
                for (double i = WRS_DADD(m, 1.0); i <= kk; i = WRS_DADD(i, 1.0))
                    f = WRS_DMUL(f, WRS_DSUB(WRS_DDIV(nr, i), r));
            } else if (m > kk) {
                for (double i = WRS_DADD(kk, 1.0); i <= m; i = WRS_DADD(i, 1.0))
                    v = WRS_DMUL(v, WRS_DSUB(WRS_DDIV(nr, i), r));
            }
            if (v <= f) return (uint64_t)kk;
            continue;
        }
        // squeeze on log f(k) / f(m)
        v = det_log(v);
        const double rho = WRS_DMUL(WRS_DDIV(km, npq),
                                    WRS_DADD(WRS_DDIV(WRS_DADD(WRS_DMUL(WRS_DADD(WRS_DDIV(km, 3.0), 0.625), km), 1.0 / 6.0), npq), 0.5));
        const double t = WRS_DDIV(-WRS_DMUL(km, km), WRS_DMUL(2.0, npq));
        if (v < WRS_DSUB(t, rho)) return (uint64_t)kk;
        if (v > WRS_DADD(t, rho)) continue;
        const double nm = WRS_DADD(WRS_DSUB(nd, m), 1.0);
        const double h = WRS_DADD(WRS_DADD(WRS_DMUL(WRS_DADD(m, 0.5), det_log(WRS_DDIV(WRS_DADD(m, 1.0), WRS_DMUL(r, nm)))),
                                           stirling_fc(m)),
                                  stirling_fc(WRS_DSUB(nd, m)));
        const double nk = WRS_DADD(WRS_DSUB(nd, kk), 1.0);
        double rhs = WRS_DADD(h, WRS_DMUL(WRS_DADD(nd, 1.0), det_log(WRS_DDIV(nm, nk))));
        rhs = WRS_DADD(rhs, WRS_DMUL(WRS_DADD(kk, 0.5), det_log(WRS_DDIV(WRS_DMUL(nk, r), WRS_DADD(kk, 1.0)))));
        rhs = WRS_DSUB(rhs, stirling_fc(kk));
        rhs = WRS_DSUB(rhs, stirling_fc(WRS_DSUB(nd, kk)));
        if (v <= rhs) return (uint64_t)kk;
    }
    return (uint64_t)m;  // unreachable in practice (acceptance rate > 0.5 per iteration)
}

// Binomial(n, p) for any p in [0, 1].
__host__ __device__ __forceinline__ uint64_t binomial(uint64_t n, double p, const BinomStream& st) {
    if (n == 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    const bool flip = p > 0.5;
    const double pp = flip ? WRS_DSUB(1.0, p) : p;
    const uint64_t x = (WRS_DMUL((double)n, pp) < 10.0) ? binom_small(n, pp, st) : binom_btrd(n, pp, st);
    return flip ? n - x : x;
}

// Rows of sections [a, b) in a table of n rows cut into sections of S rows.
__host__ __device__ __forceinline__ uint64_t section_rows(uint64_t a, uint64_t b, uint64_t S, uint64_t n) {
    const uint64_t hi = b * S < n ? b * S : n;
    return hi - a * S;
}

// Count and output offset of section k out of K for m samples (tree walk from the root).
__host__ __device__ __forceinline__ void section_count(uint64_t k, uint64_t K, uint64_t S, uint64_t n, uint64_t m,
                                                       uint32_t k0, uint32_t k1, uint64_t counter_base,
                                                       uint64_t* count, uint64_t* offset) {
    uint64_t lo = 0, hi = K, cnt = m, off = 0;
    uint32_t node = 1;
    BinomStream st;
    st.k0 = k0;
    st.k1 = k1;
    st.c0 = (uint32_t)counter_base;
    st.c1 = (uint32_t)(counter_base >> 32);
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        const double pl = WRS_DDIV((double)section_rows(lo, mid, S, n), (double)section_rows(lo, hi, S, n));
        st.node = node;
        const uint64_t cl = binomial(cnt, pl, st);
        if (k < mid) {
            hi = mid;
            cnt = cl;
            node = 2 * node;
        } else {
            lo = mid;
            off += cl;
            cnt -= cl;
            node = 2 * node + 1;
        }
    }
    *count = cnt;
    *offset = off;
}

}  // namespace wrs
