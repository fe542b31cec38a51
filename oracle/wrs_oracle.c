/*
 * wrs_oracle.c — CPU oracle of the weighted-random-sampling hot path (see wrs_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: checker and timed CPU reference; never part of the library.
 * Built with -ffp-contract=off so that every floating-point expression rounds exactly as
 * written (the GPU code that these functions are compared with bit for bit uses explicitly
 * rounded operations for the same expressions).
 */
#include "wrs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

#define EPSILON_REF 1e-10 /* construction/SamplingAlgorithm.cuh:14 */

/* ------------------------------------------------------------------ exact sum */
/* Shewchuk's non-overlapping expansion (the algorithm of Python's math.fsum). */
double or_exact_sum_f32(const float* w, int64_t n) {
    size_t cap = 64, np = 0;
    double* part = (double*)malloc(cap * sizeof(double));
    for (int64_t k = 0; k < n; ++k) {
        double x = (double)w[k];
        size_t i = 0;
        for (size_t j = 0; j < np; ++j) {
            double y = part[j];
            if (fabs(x) < fabs(y)) {
                double t = x;
                x = y;
                y = t;
            }
            double hi = x + y;
            double lo = y - (hi - x);
            if (lo != 0.0) part[i++] = lo;
            x = hi;
        }
        if (i >= cap) {
            cap *= 2;
            part = (double*)realloc(part, cap * sizeof(double));
        }
        part[i++] = x;
        np = i;
    }
    /* sum the partials from the top with correct rounding */
    double hi = 0.0;
    if (np > 0) {
        size_t k = np;
        hi = part[--k];
        double lo = 0.0;
        while (k > 0) {
            double x = hi, y = part[--k];
            hi = x + y;
            double yr = hi - x;
            lo = y - yr;
            if (lo != 0.0) break;
        }
        if (k > 0 && ((lo < 0.0 && part[k - 1] < 0.0) || (lo > 0.0 && part[k - 1] > 0.0))) {
            double y = lo * 2.0;
            double x = hi + y;
            double yr = x - hi;
            if (y == yr) hi = x;
        }
    }
    free(part);
    return hi;
}

/* ------------------------------------------------------------------ Philox4x32-10 */
/* Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11. */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static inline void philox_block(uint64_t b, uint32_t c2, uint32_t c3, uint64_t seed, uint32_t out[4]) {
    uint32_t ctr[4] = {(uint32_t)b, (uint32_t)(b >> 32), c2, c3};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    or_philox4x32_10(ctr, key, out);
}

/* an alias row: floor(u len / 2^64) for the 64-bit uniform u = x1:x0 */
static inline uint32_t row_of(const uint32_t x[4], uint64_t len) {
    return (uint32_t)((((unsigned __int128)(((uint64_t)x[1] << 32) | x[0])) * len) >> 64);
}
/* a rejection try's slot: floor(u |A| / 2^64) for the 64-bit uniform u = x1:x0 */
static inline uint32_t slot_of(uint32_t x0, uint32_t x1, uint64_t asz) {
    return (uint32_t)((((unsigned __int128)(((uint64_t)x1 << 32) | x0)) * asz) >> 64);
}
static inline float coin24(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-8f; }
static inline float bits_f(uint32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}
static inline uint32_t f_bits(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return b;
}

/* ------------------------------------------------------------------ reference CPU builds */
/* AliasTableSweep::build (construction/aliasTable/buildMethod/AliasTableSweep.cu:12-60). */
int or_sweep_build(const double* win, int64_t n64, double* weight, int32_t* alias, double* W_out) {
    const int N = (int)n64;
    double* weights = (double*)malloc((size_t)(N + 2) * sizeof(double));
    memcpy(weights, win, (size_t)N * sizeof(double));
    double W = 0;
    for (int i = 0; i < N; i++) W += weights[i]; /* sumWeightsCpu, SamplingAlgorithm.cu:14-19 */
    weights[N] = INFINITY;
    weights[N + 1] = 0;
    for (int i = 0; i < N; ++i) {
        weight[i] = NAN;
        alias[i] = -1;
    }
    int i = 0;
    while (weights[i] > W / N) i++;
    int j = 0;
    while (weights[j] <= W / N) j++;
    double w = weights[j];
    for (int64_t guard = 0; guard < 4 * (int64_t)N + 16; ++guard) {
        int exhausted = w <= W / N + EPSILON_REF;
        if (exhausted && j >= N) exhausted = 0;
        else if (!exhausted && i >= N) exhausted = 1;
        if (exhausted) {
            if (j >= N) break;
            weight[j] = w;
            int j_ = j;
            do { j_++; } while (j < N + 2 && weights[j_] <= W / N);
            alias[j] = j_;
            w += weights[j_] - W / N;
            j = j_;
        } else {
            if (i >= N) break;
            weight[i] = weights[i];
            alias[i] = j;
            w += weights[i] - W / N;
            do { i++; } while (i < N + 2 && weights[i] > W / N);
        }
    }
    if (W_out) *W_out = W;
    free(weights);
    return 0;
}

/* The same sweep with every quantity in FP32 (the weights, W summed in input order, W/N, the
 * running residual w and EPSILON): the "all-FP32" build of the precision comparison. Rows are
 * returned as doubles on the scale W_f32 / N. */
int or_sweep_build_f32(const float* win, int64_t n64, double* weight, int32_t* alias, double* W_out) {
    const int N = (int)n64;
    float* weights = (float*)malloc((size_t)(N + 2) * sizeof(float));
    memcpy(weights, win, (size_t)N * sizeof(float));
    volatile float Wv = 0.0f;  /* no reassociation or wider accumulation */
    for (int i = 0; i < N; i++) Wv = Wv + weights[i];
    const float W = Wv;
    const float WN = W / (float)N;
    const float eps = (float)EPSILON_REF;
    weights[N] = INFINITY;
    weights[N + 1] = 0.0f;
    for (int i = 0; i < N; ++i) {
        weight[i] = NAN;
        alias[i] = -1;
    }
    int i = 0;
    while (weights[i] > WN) i++;
    int j = 0;
    while (weights[j] <= WN) j++;
    volatile float w = weights[j];
    for (int64_t guard = 0; guard < 4 * (int64_t)N + 16; ++guard) {
        int exhausted = w <= WN + eps;
        if (exhausted && j >= N) exhausted = 0;
        else if (!exhausted && i >= N) exhausted = 1;
        if (exhausted) {
            if (j >= N) break;
            weight[j] = (double)w;
            int j_ = j;
            do { j_++; } while (j < N + 2 && weights[j_] <= WN);
            alias[j] = j_;
            w = w + (weights[j_] - WN);
            j = j_;
        } else {
            if (i >= N) break;
            weight[i] = (double)weights[i];
            alias[i] = j;
            w = w + (weights[i] - WN);
            do { i++; } while (i < N + 2 && weights[i] > WN);
        }
    }
    if (W_out) *W_out = (double)W;
    free(weights);
    return 0;
}

typedef struct {
    int i;
    int j;
    double spill;
} SplitCfg; /* buildMethod/SplitConfig.cuh:4-8 */

typedef struct {
    int item;
    double weight;
} LhItem; /* buildMethod/LhType.cuh:15-35 */

/* SplitMethodBasic::split (splitMethod/SplitMethodBasic.cu:14-50) */
static int ref_split(int k, SplitCfg* splits, int N, double W, int p, const LhItem* h, const double* pH, int h_size,
                     const double* pL, int l_size) {
    if (k == 1) {
        splits[0].i = 0;
        splits[0].j = 0;
        splits[0].spill = 0;
        splits[p].i = l_size - 1;
        splits[p].j = h_size - 1;
        splits[p].spill = 0;
    }
    int n_ = (int)ceil(((double)N * k) / p);
    int a = 0;
    int b = (n_ < h_size ? n_ : h_size) - 1;
    double wpb = (W * n_) / N;
    for (int it = 0; it < 200; ++it) {
        int j = (a + b) / 2;
        int i = (n_ - j) < (l_size - 1) ? (n_ - j) : (l_size - 1);
        int status;
        double sigma = 0;
        /* BinarySearchChecker::check (SplitMethodBasic.cuh:22-40) */
        if (j + 1 >= h_size || i - 1 < 0) {
            status = 1;
        } else if (i >= l_size || j < 0) {
            status = 2;
        } else {
            sigma = pL[i] + pH[j];
            double sigmaNext = pL[i - 1] + pH[j + 1];
            if (sigma <= wpb && sigmaNext > wpb) status = 0;
            else if (sigma <= wpb) status = 2;
            else status = 1;
        }
        if (status == 0) {
            splits[k].i = i;
            splits[k].j = j;
            splits[k].spill = sigma + h[j].weight - wpb;
            return 0;
        } else if (status == 2) {
            a = j + 1;
        } else {
            b = j;
        }
    }
    return -1;
}

/* PackMethodSweep::pack (packMethod/PackMethodSweep.cu:3-65) */
static void ref_pack_sweep(int k, const SplitCfg* splits, double W_N, const LhItem* h, const LhItem* l,
                           double* tw, int32_t* ta, const double* weights) {
    SplitCfg cur = splits[k], prev = splits[k - 1];
    int i = l[prev.i].item, j = h[prev.j].item;
    int iMax = l[cur.i].item, jMax = h[cur.j].item;
    double w = prev.spill;
    if (prev.spill == 0) w = h[prev.j].weight;
    for (int64_t guard = 0; guard < (int64_t)1 << 40; ++guard) {
        int exhausted = w <= W_N + EPSILON_REF;
        if (exhausted && j >= jMax) exhausted = 0;
        else if (!exhausted && i >= iMax) exhausted = 1;
        if (exhausted) {
            if (j >= jMax) return;
            int j_ = j;
            do { j_++; } while (j < jMax && weights[j_] <= W_N);
            tw[j] = w;
            ta[j] = j_;
            w += weights[j_] - W_N;
            j = j_;
        } else {
            if (i >= iMax) return;
            tw[i] = weights[i];
            ta[i] = j;
            w += tw[i] - W_N;
            do { i++; } while (i < iMax && weights[i] > W_N);
        }
    }
}

/* AliasTableSplit::build (buildMethod/AliasTableSplit.cu:24-80); threads > 1 runs the
 * independent split and pack loops over k on several cores (they write disjoint outputs). */
int or_split_build(const double* win, int64_t n64, int64_t p64, double* tw, int32_t* ta, double* W_out, int threads) {
    const int N = (int)n64;
    int p = (int)p64;
    if (p > N / 2) p = N / 10; /* AliasTableSplit constructor, :9-18 */
    if (p < 1) p = 1;
    double* weights = (double*)malloc((size_t)(N + 2) * sizeof(double));
    memcpy(weights, win, (size_t)N * sizeof(double));
    double W = 0;
    for (int i = 0; i < N; i++) W += weights[i];
    weights[N] = INFINITY;
    weights[N + 1] = 0;
    for (int i = 0; i < N; i++) {
        tw[i] = weights[i];
        ta[i] = -1;
    }
    int* pre = (int*)malloc((size_t)(N + 2) * sizeof(int));
    int sum = 0;
    for (int i = 0; i < N + 2; i++) {
        int f = (weights[i] > W / N) ? 1 : 0;
        pre[i] = sum;
        sum += f;
    }
    int numH = pre[N + 1];
    int numL = (N + 2) - numH;
    LhItem* l = (LhItem*)malloc((size_t)numL * sizeof(LhItem));
    LhItem* h = (LhItem*)malloc((size_t)numH * sizeof(LhItem));
    double* pL = (double*)malloc((size_t)numL * sizeof(double));
    double* pH = (double*)malloc((size_t)numH * sizeof(double));
    SplitCfg* splits = (SplitCfg*)calloc((size_t)p + 1, sizeof(SplitCfg));
    for (int i = 0; i < N + 2; i++) {
        if (weights[i] > W / N) {
            h[pre[i]].item = i;
            h[pre[i]].weight = weights[i];
            pH[pre[i]] = weights[i];
        } else {
            l[i - pre[i]].item = i;
            l[i - pre[i]].weight = weights[i];
            pL[i - pre[i]] = weights[i];
        }
    }
    double s = 0;
    for (int i = 0; i < numL; i++) {
        double it = pL[i];
        pL[i] = s;
        s += it;
    }
    s = 0;
    for (int i = 0; i < numH; i++) {
        double it = pH[i];
        pH[i] = s;
        s += it;
    }
    int bad = 0;
    if (numH < 2 || numL < 2) {
        bad = -1; /* the reference asserts here (AliasTableSplit.cu:43-44) */
    } else {
        ref_split(1, splits, N, W, p, h, pH, numH, pL, numL);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 16) reduction(| : bad)
#endif
        for (int k = 2; k <= p - 1; k++) bad |= ref_split(k, splits, N, W, p, h, pH, numH, pL, numL) ? 1 : 0;
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 16)
#endif
        for (int k = 1; k <= p; k++) ref_pack_sweep(k, splits, W / N, h, l, tw, ta, weights);
    }
    (void)threads;
    if (W_out) *W_out = W;
    free(weights);
    free(pre);
    free(l);
    free(h);
    free(pL);
    free(pH);
    free(splits);
    return bad;
}

/* ------------------------------------------------------------------ table checks */
static int cmp_double(const void* a, const void* b) {
    double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

static double quantile_sorted_copy(double* v, int64_t m, double q) {
    if (m <= 0) return 0.0;
    qsort(v, (size_t)m, sizeof(double), cmp_double);
    int64_t idx = (int64_t)floor(q * (double)(m - 1));
    return v[idx];
}

/* Per-item check: got_i = sum over rows r of [r == i] p_r + [alias_r == i] (1 - p_r), in
 * long double; expected_i = n w_i / W with W the exact sum (AliasTable::verifyTableCorrectness,
 * construction/aliasTable/AliasTable.cu:24-65, with a relative instead of absolute tolerance). */
static int check_common_w(const float* w32, const double* w64, int64_t n, const float* probs_or_null,
                          const uint32_t* rows, const double* ref_weight, const int32_t* ref_alias, double W_N,
                          double W_expect, double* stats) {
    long double* got = (long double*)calloc((size_t)n, sizeof(long double));
    int64_t bad_rows = 0;
    for (int64_t r = 0; r < n; ++r) {
        long double p;
        int64_t a;
        if (rows) {
            p = (long double)bits_f(rows[2 * r]);
            a = (int64_t)rows[2 * r + 1];
        } else {
            p = (long double)ref_weight[r] / (long double)W_N;
            a = (int64_t)ref_alias[r];
            if (ref_weight[r] >= W_N) a = r; /* alias uninitialised when the row is full */
        }
        (void)probs_or_null;
        if (!(p >= 0.0L) || p > 1.0L + 1e-6L || a < 0 || a >= n) {
            ++bad_rows;
            if (!(p >= 0.0L)) p = 0.0L;
            if (a < 0 || a >= n) a = r;
        }
        got[r] += p;
        got[a] += 1.0L - p;
    }
    double* rel = (double*)malloc((size_t)n * sizeof(double));
    int64_t m = 0, worst = -1, zero_bad = 0;
    double maxrel = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        long double wi = w32 ? (long double)w32[i] : (long double)w64[i];
        long double expct = (long double)n * wi / (long double)W_expect;
        if (wi == 0.0L) {
            if (got[i] != 0.0L) ++zero_bad;
            continue;
        }
        long double e = got[i] - expct;
        if (e < 0) e = -e;
        double re = (double)(e / expct);
        rel[m++] = re;
        if (re > maxrel || worst < 0) {
            if (re >= maxrel) worst = i;
            if (re > maxrel) maxrel = re;
        }
    }
    stats[0] = maxrel;
    stats[1] = quantile_sorted_copy(rel, m, 0.9999);
    stats[2] = (double)worst;
    stats[3] = (double)zero_bad;
    stats[4] = (double)bad_rows;
    free(rel);
    free(got);
    return 0;
}

static int check_common(const float* w32, const double* w64, int64_t n, const float* probs_or_null,
                        const uint32_t* rows, const double* ref_weight, const int32_t* ref_alias, double W,
                        double* stats) {
    return check_common_w(w32, w64, n, probs_or_null, rows, ref_weight, ref_alias, W / (double)n, W, stats);
}

/* A reference-format table whose rows hold weights on its own scale W_N_table (the average
 * weight its build used), checked against n w_i / W_exact. */
int or_check_ref_table_w(const float* w, int64_t n, const double* weight, const int32_t* alias, double W_N_table,
                         double W_exact, double* stats) {
    return check_common_w(w, NULL, n, NULL, NULL, weight, alias, W_N_table, W_exact, stats);
}

int or_check_table(const float* w, int64_t n, const uint32_t* rows, double* stats, double* W_used) {
    double W = or_exact_sum_f32(w, n);
    if (W_used) *W_used = W;
    return check_common(w, NULL, n, NULL, rows, NULL, NULL, W, stats);
}

int or_check_ref_table(const double* w, int64_t n, const double* weight, const int32_t* alias, double W,
                       double* stats) {
    return check_common(NULL, w, n, NULL, NULL, weight, alias, W, stats);
}

/* ------------------------------------------------------------------ exact merge build */
static inline uint64_t dbits(double x) {
    uint64_t b;
    memcpy(&b, &x, 8);
    return b;
}
static inline u128 q_one(void) { return (u128)1 << 64; }
static inline int q_neg(u128 x) { return (int)((uint64_t)(x >> 64) >> 63); }
static inline u128 q_from_double(double x) {
    uint64_t b = dbits(x);
    int e = (int)((b >> 52) & 0x7ff);
    if (e == 0) return 0;
    u128 m = (u128)((b & 0xfffffffffffffull) | 0x10000000000000ull);
    int sh = e - 1075 + 64;
    if (sh >= 0) return m << sh;
    if (sh <= -53) return 0;
    return m >> (-sh);
}
static inline double q_to_double_signed(u128 x) {
    int neg = q_neg(x);
    u128 m = neg ? (u128)0 - x : x;
    double v = (double)(uint64_t)(m >> 64) + (double)(uint64_t)m * 5.421010862427522170037e-20;
    return neg ? -v : v;
}
static inline u128 q_round24(u128 x) {
    const u128 half = (u128)1 << 39;
    const u128 mask = ~(((u128)1 << 40) - 1);
    return (x + half) & mask;
}
static inline u128 q_scale_excess(u128 e, int64_t nfix) {
    if (nfix == 0) return e;
    uint64_t an = nfix < 0 ? (uint64_t)(-(nfix + 1)) + 1u : (uint64_t)nfix;
    uint64_t ehi = (uint64_t)(e >> 64), elo = (uint64_t)e;
    uint64_t mh = (uint64_t)(((u128)elo * an) >> 64);
    u128 corr = (u128)ehi * an + mh;
    return nfix < 0 ? e - corr : e + corr;
}
static inline int64_t excess_correction(u128 a_total, u128 e_total) {
    if (e_total == 0) return 0;
    double d = q_to_double_signed(a_total - e_total);
    double e = q_to_double_signed(e_total);
    double r = d / e;
    if (r > 0.25) r = 0.25;
    if (r < -0.25) r = -0.25;
    return (int64_t)llrint(r * 18446744073709551616.0);
}
static inline float heavy_row_prob(u128 r) {
    if (q_neg(r)) return 0.0f;
    if (r >= q_one()) return 1.0f;
    return (float)((double)((uint64_t)r >> 11) * 1.1102230246251565404e-16);
}
static inline float large_light_prob(u128 Li, uint64_t d48) {
    u128 dd = q_round24(Li + ((u128)d48 << 16)) - q_round24(Li);
    uint32_t units = (uint32_t)(dd >> 40);
    return (float)(16777216u - units) * 5.9604644775390625e-8f;
}

/* round(x * 2^fb) for x >= 0, to nearest with ties to even: x * 2^fb is exact in FP64
 * and llrint rounds in the default (nearest-even) mode. */
static inline uint64_t fixq(double x, int fb) { return (uint64_t)llrint(ldexp(x, fb)); }

enum { K_SMALL = 1, K_LARGE = 2, K_HEAVY = 3 };

/* round(p * 2^48) for a float p in [0, 1/2), ties to even (p * 2^48 is exact). */
static inline uint64_t fix48f(float p) { return (uint64_t)llrint(ldexp((double)p, 48)); }

typedef struct {
    double R;
    float R32, H1, Hh;
} ClassParams;

/* The build's class thresholds: H1 = largest float <= W/N, Hh = smallest float >= W/(2N). */
static ClassParams class_params(double W_N, double R) {
    ClassParams c;
    c.R = R;
    c.R32 = (float)R;
    float h1 = (float)W_N;
    if ((double)h1 > W_N) h1 = nextafterf(h1, -INFINITY);
    c.H1 = h1;
    double half = 0.5 * W_N;
    float hh = (float)half;
    if ((double)hh < half) hh = nextafterf(hh, INFINITY);
    c.Hh = hh;
    return c;
}

/* classify(): the per-item quantities of the build, restated: light deficits in Q16.48
 * (stored for small lights, true for large ones), heavy excess in Q40.24. */
static inline int classify(float wf, const ClassParams* cp, float* p_out, uint64_t* q_out) {
    if (wf > cp->H1) {
        double h = (double)wf * cp->R;
        if (h < 1.0) h = 1.0;
        *q_out = fixq(h - 1.0, 24);
        *p_out = 1.0f;
        return K_HEAVY;
    }
    if (wf >= cp->Hh) {
        double p = (double)wf * cp->R;
        if (p > 1.0) p = 1.0;
        *q_out = fixq(1.0 - p, 48);
        *p_out = 1.0f;
        return K_LARGE;
    }
    float ps = wf * cp->R32;
    *p_out = ps;
    *q_out = (1ull << 48) - fix48f(ps);
    return K_SMALL;
}

int or_exact_build(const float* w, int64_t n, double W, uint32_t* rows) {
    const double W_N = W / (double)n;
    const double R = 1.0 / W_N;
    const ClassParams cp = class_params(W_N, R);
    int64_t nL = 0, nH = 0;
    u128 S = 0, L = 0, E = 0;
    for (int64_t i = 0; i < n; ++i) {
        float p;
        uint64_t q;
        int k = classify(w[i], &cp, &p, &q);
        if (k == K_HEAVY) {
            ++nH;
            E += (u128)q << 40;
        } else {
            ++nL;
            if (k == K_SMALL) S += (u128)q << 16;
            else L += (u128)q << 16;
        }
    }
    const u128 A_tot = S + q_round24(L);
    const int64_t nfix = excess_correction(A_tot, E);
    u128* A = (u128*)malloc((size_t)(nL ? nL : 1) * sizeof(u128));
    float* lp = (float*)malloc((size_t)(nL ? nL : 1) * sizeof(float));
    uint32_t* litem = (uint32_t*)malloc((size_t)(nL ? nL : 1) * sizeof(uint32_t));
    u128* Eh = (u128*)malloc((size_t)(nH ? nH : 1) * sizeof(u128));
    uint32_t* hitem = (uint32_t*)malloc((size_t)(nH ? nH : 1) * sizeof(uint32_t));
    int64_t li = 0, hj = 0;
    u128 Sr = 0, Lr = 0, Er = 0;
    for (int64_t i = 0; i < n; ++i) {
        float p;
        uint64_t q;
        int k = classify(w[i], &cp, &p, &q);
        if (k == K_HEAVY) {
            Er += (u128)q << 40;
            Eh[hj] = q_scale_excess(Er, nfix);
            hitem[hj] = (uint32_t)i;
            ++hj;
        } else {
            A[li] = Sr + q_round24(Lr);
            litem[li] = (uint32_t)i;
            if (k == K_SMALL) {
                lp[li] = p;
                Sr += (u128)q << 16;
            } else {
                lp[li] = large_light_prob(Lr, q);
                Lr += (u128)q << 16;
            }
            ++li;
        }
    }
    int64_t i = 0, j = 0;
    while (i < nL || j < nH) {
        if (i < nL && (j >= nH || A[i] < Eh[j])) {
            uint32_t al = nH == 0 ? litem[i] : (j < nH ? hitem[j] : hitem[nH - 1]);
            rows[2 * (int64_t)litem[i]] = f_bits(lp[i]);
            rows[2 * (int64_t)litem[i] + 1] = al;
            ++i;
        } else {
            u128 A_next = (i < nL) ? A[i] : A_tot;
            u128 r = q_one() + Eh[j] - A_next;
            uint32_t al = (j + 1 < nH) ? hitem[j + 1] : hitem[j];
            rows[2 * (int64_t)hitem[j]] = f_bits(heavy_row_prob(r));
            rows[2 * (int64_t)hitem[j] + 1] = al;
            ++j;
        }
    }
    free(A);
    free(lp);
    free(litem);
    free(Eh);
    free(hitem);
    return 0;
}

/* ------------------------------------------------------------------ PSA+ */
/* PSA+ (AliasTableSplitGpu::psaPlus + PsaPlusNormal::kernel,
 * construction/aliasTable/buildMethod/AliasTableSplitGpu.cu:342-386,
 * construction/aliasTable/psaPlus/PsaPlusNormal.cu:12-152): every section is packed locally
 * first; the items the local pass cannot finish, one of them with a residual weight, go
 * through the global split/pack. Restated on this library's exact quantities: sections are
 * tiles of T items, and the lines are those of or_exact_build (the global deficit line A with
 * its dithering, the corrected excess line E~) restricted to the tile and measured from the
 * tile's start (A_b, E~_b). In a tile with total deficit D and total excess Et:
 *   - a light is finished when a heavy of the tile has E > A_i (alias: the first such heavy);
 *   - a heavy with E_j <= D is finished with r_j = 1 + E_j - A_next (A_next = the first light
 *     start >= E_j, else D) and aliases the tile's next heavy; the tile's last heavy, if
 *     finished, keeps r_j as its row probability but waits for its alias: it becomes the
 *     tile's first leftover light, with deficit A_next - E_j rounded up to the 2^-48 grid;
 *   - lights starting at or after Et are leftover lights; the first heavy with E_j > D is a
 *     leftover heavy with residual excess E_j - D, the heavies after it leftover heavies with
 *     their whole excess.
 * The leftovers of all tiles, in tile order, are merged as or_exact_build merges lights and
 * heavies (their excess line corrected for what remains of the mismatch, a rounding residue). */
typedef struct {
    uint32_t item;
    float prob;
    u128 q;
} OrLeft;

int or_psa_plus_build(const float* w, int64_t n, double W, int64_t T, uint32_t* rows) {
    const double W_N = W / (double)n;
    const double R = 1.0 / W_N;
    const ClassParams cp = class_params(W_N, R);
    /* global lines, as or_exact_build */
    u128 S = 0, L = 0, E = 0;
    for (int64_t i = 0; i < n; ++i) {
        float p;
        uint64_t q;
        const int k = classify(w[i], &cp, &p, &q);
        if (k == K_HEAVY) E += (u128)q << 40;
        else if (k == K_SMALL) S += (u128)q << 16;
        else L += (u128)q << 16;
    }
    const int64_t nfix = excess_correction(S + q_round24(L), E);
    OrLeft* L2 = (OrLeft*)malloc((size_t)(n + 1) * sizeof(OrLeft));
    OrLeft* H2 = (OrLeft*)malloc((size_t)(n + 1) * sizeof(OrLeft));
    u128* A = (u128*)malloc((size_t)(T + 1) * sizeof(u128));
    u128* Eh = (u128*)malloc((size_t)(T + 1) * sizeof(u128));
    float* lp = (float*)malloc((size_t)T * sizeof(float));
    uint32_t* litem = (uint32_t*)malloc((size_t)T * sizeof(uint32_t));
    uint32_t* hitem = (uint32_t*)malloc((size_t)T * sizeof(uint32_t));
    int64_t nL2 = 0, nH2 = 0;
    u128 Sr = 0, Lr = 0, Er = 0;
    for (int64_t i0 = 0; i0 < n; i0 += T) {
        const int64_t i1 = (i0 + T < n) ? i0 + T : n;
        const u128 A_b = Sr + q_round24(Lr);
        const u128 E_b = q_scale_excess(Er, nfix);
        int64_t nl = 0, nh = 0;
        for (int64_t i = i0; i < i1; ++i) {
            float p;
            uint64_t q;
            const int k = classify(w[i], &cp, &p, &q);
            if (k == K_HEAVY) {
                Er += (u128)q << 40;
                Eh[nh] = q_scale_excess(Er, nfix) - E_b;
                hitem[nh++] = (uint32_t)i;
            } else {
                A[nl] = Sr + q_round24(Lr) - A_b;
                litem[nl] = (uint32_t)i;
                if (k == K_SMALL) {
                    lp[nl] = p;
                    Sr += (u128)q << 16;
                } else {
                    lp[nl] = large_light_prob(Lr, q);
                    Lr += (u128)q << 16;
                }
                ++nl;
            }
        }
        const u128 D = Sr + q_round24(Lr) - A_b;
        A[nl] = D;
        const u128 Et = q_scale_excess(Er, nfix) - E_b;
        /* lights */
        int64_t L0 = nl, j = 0;
        for (int64_t li = 0; li < nl; ++li) {
            if (!(A[li] < Et)) {
                L0 = li;
                break;
            }
            while (Eh[j] <= A[li]) ++j;
            rows[2 * (int64_t)litem[li]] = f_bits(lp[li]);
            rows[2 * (int64_t)litem[li] + 1] = hitem[j];
        }
        /* heavies */
        int64_t Js = nh, I = 0;
        int conv = 0;
        OrLeft cv = {0, 0.0f, 0};
        for (int64_t hj = 0; hj < nh; ++hj) {
            if (Eh[hj] > D) {
                Js = hj;
                break;
            }
            while (I < nl && A[I] < Eh[hj]) ++I;
            const u128 A_next = (I < nl) ? A[I] : D;
            const float pr = heavy_row_prob(q_one() + Eh[hj] - A_next);
            if (hj + 1 < nh) {
                rows[2 * (int64_t)hitem[hj]] = f_bits(pr);
                rows[2 * (int64_t)hitem[hj] + 1] = hitem[hj + 1];
            } else {
                const u128 g = ((u128)1 << 16) - 1; /* round up to the 2^-48 grid */
                conv = 1;
                cv.item = hitem[hj];
                cv.prob = pr;
                cv.q = (A_next - Eh[hj] + g) & ~g;
            }
        }
        if (conv) L2[nL2++] = cv;
        for (int64_t li = L0; li < nl; ++li) {
            OrLeft x = {litem[li], lp[li], A[li + 1] - A[li]};
            L2[nL2++] = x;
        }
        for (int64_t hj = Js; hj < nh; ++hj) {
            OrLeft x = {hitem[hj], 0.0f, hj == Js ? Eh[hj] - D : Eh[hj] - Eh[hj - 1]};
            H2[nH2++] = x;
        }
    }
    /* global merge of the leftovers */
    u128 At = 0, Etot = 0;
    for (int64_t i = 0; i < nL2; ++i) At += L2[i].q;
    for (int64_t j = 0; j < nH2; ++j) Etot += H2[j].q;
    const int64_t nfix2 = excess_correction(At, Etot);
    u128* Ap = (u128*)malloc((size_t)(nL2 + 1) * sizeof(u128));
    u128* Ep = (u128*)malloc((size_t)(nH2 + 1) * sizeof(u128));
    u128 run = 0;
    for (int64_t i = 0; i < nL2; ++i) {
        Ap[i] = run;
        run += L2[i].q;
    }
    run = 0;
    for (int64_t j = 0; j < nH2; ++j) {
        run += H2[j].q;
        Ep[j] = q_scale_excess(run, nfix2);
    }
    int64_t i = 0, j = 0;
    while (i < nL2 || j < nH2) {
        if (i < nL2 && (j >= nH2 || Ap[i] < Ep[j])) {
            const uint32_t al = nH2 == 0 ? L2[i].item : (j < nH2 ? H2[j].item : H2[nH2 - 1].item);
            rows[2 * (int64_t)L2[i].item] = f_bits(L2[i].prob);
            rows[2 * (int64_t)L2[i].item + 1] = al;
            ++i;
        } else {
            const u128 A_next = (i < nL2) ? Ap[i] : At;
            const uint32_t al = (j + 1 < nH2) ? H2[j + 1].item : H2[j].item;
            rows[2 * (int64_t)H2[j].item] = f_bits(heavy_row_prob(q_one() + Ep[j] - A_next));
            rows[2 * (int64_t)H2[j].item + 1] = al;
            ++j;
        }
    }
    free(L2); free(H2); free(A); free(Eh); free(lp); free(litem); free(hitem); free(Ap); free(Ep);
    return 0;
}

/* ------------------------------------------------------------------ batched (CSR) */
/* The batched build gives every table the rows of a single-table build of its weights, so
 * its restatement is a loop of or_exact_build (the reference's batches are such loops). */
int or_batched_build(const float* w, const int64_t* off, int64_t num_tables, uint32_t* rows, double* W_out) {
    int bad = 0;
    for (int64_t t = 0; t < num_tables; ++t) {
        const int64_t n = off[t + 1] - off[t];
        if (n <= 0) continue;
        const double W = or_exact_sum_f32(w + off[t], n);
        if (W_out) W_out[t] = W;
        if (!(W > 0.0) || isinf(W)) {
            ++bad;
            continue;
        }
        or_exact_build(w + off[t], n, W, rows + 2 * off[t]);
    }
    return bad;
}


/* ------------------------------------------------------------------ precision comparison builds */
/* The library's all-FP64 / all-FP32 builds (precision_kernels.cuh): the merge of the deficit
 * and excess lines with every quantity in one floating-point type R, in the kernels' summation
 * order. The weight total: tiles of 256 threads x 8 items; a thread sums its items in order,
 * each warp's 32 thread sums in lane order, the 8 warp sums in order; tiles in 1024 chunks of
 * K = ceil(tiles / 1024) consecutive tiles, each chunk in order, the chunk sums in order. The
 * lines: each tile's deficits (excesses) summed in item order, the tile bases in tile order,
 * an item's position = tile base + its tile-local prefix. Bit-exact with the GPU. */
#define PREC_NT 256
#define PREC_IPT 8
#define PREC_TILE (PREC_NT * PREC_IPT)
#define PREC_CHUNKS 1024

#define DEFINE_PREC_BUILD(R, NAME)                                                                           \
    /* exclusive prefixes of v[0..255] in the CTA order; returns the total */                               \
    static R NAME##_block_scan(const R* v, R* ex) {                                                         \
        R wtot[PREC_NT / 32];                                                                               \
        for (int wp = 0; wp < PREC_NT / 32; ++wp) {                                                         \
            R acc = (R)0;                                                                                   \
            for (int l = 0; l < 32; ++l) {                                                                  \
                ex[wp * 32 + l] = acc;                                                                      \
                acc = acc + v[wp * 32 + l];                                                                 \
            }                                                                                               \
            wtot[wp] = acc;                                                                                 \
        }                                                                                                   \
        R base[PREC_NT / 32];                                                                               \
        R acc = (R)0;                                                                                       \
        for (int wp = 0; wp < PREC_NT / 32; ++wp) {                                                         \
            base[wp] = acc;                                                                                 \
            acc = acc + wtot[wp];                                                                           \
        }                                                                                                   \
        for (int t = 0; t < PREC_NT; ++t) ex[t] = base[t / 32] + ex[t];                                     \
        return acc;                                                                                         \
    }                                                                                                       \
    /* exclusive prefixes of per-tile values in the chunked order; returns the total */                    \
    static R NAME##_tile_scan(const R* v, int64_t nt, R* pre) {                                             \
        const int64_t K = (nt + PREC_CHUNKS - 1) / PREC_CHUNKS;                                             \
        R chunk[PREC_CHUNKS];                                                                               \
        for (int c = 0; c < PREC_CHUNKS; ++c) {                                                             \
            R acc = (R)0;                                                                                   \
            for (int64_t t = c * K; t < nt && t < (c + 1) * K; ++t) acc = acc + v[t];                       \
            chunk[c] = acc;                                                                                 \
        }                                                                                                   \
        R b = (R)0;                                                                                         \
        for (int c = 0; c < PREC_CHUNKS; ++c) {                                                             \
            const R t = chunk[c];                                                                           \
            chunk[c] = b;                                                                                   \
            b = b + t;                                                                                      \
        }                                                                                                   \
        if (pre) {                                                                                          \
            for (int c = 0; c < PREC_CHUNKS; ++c) {                                                         \
                R p = chunk[c];                                                                             \
                for (int64_t t = c * K; t < nt && t < (c + 1) * K; ++t) {                                   \
                    pre[t] = p;                                                                             \
                    p = p + v[t];                                                                           \
                }                                                                                           \
            }                                                                                               \
        }                                                                                                   \
        return b;                                                                                           \
    }                                                                                                       \
    static int NAME(const float* w, int64_t n, uint32_t* rows, double* W_out) {                             \
        const int64_t nt = (n + PREC_TILE - 1) / PREC_TILE;                                                 \
        R* tv = (R*)malloc(sizeof(R) * nt);                                                                 \
        R* th = (R*)malloc(sizeof(R) * nt);                                                                 \
        R* pl = (R*)malloc(sizeof(R) * nt);                                                                 \
        R* ph = (R*)malloc(sizeof(R) * nt);                                                                 \
        int64_t* cl = (int64_t*)calloc(nt + 1, sizeof(int64_t));                                            \
        int64_t* ch = (int64_t*)calloc(nt + 1, sizeof(int64_t));                                            \
        R* Lkey = (R*)malloc(sizeof(R) * (n + 1));                                                          \
        R* Hkey = (R*)malloc(sizeof(R) * (n + 1));                                                          \
        uint32_t* Litem = (uint32_t*)malloc(4 * (n + 1));                                                   \
        uint32_t* Hitem = (uint32_t*)malloc(4 * (n + 1));                                                   \
        float* Lprob = (float*)malloc(4 * (n + 1));                                                         \
        R v[PREC_NT], ex[PREC_NT];                                                                          \
        int bad = 0;                                                                                        \
        for (int64_t t = 0; t < nt; ++t) {                                                                  \
            for (int thr = 0; thr < PREC_NT; ++thr) {                                                       \
                R acc = (R)0;                                                                               \
                for (int k = 0; k < PREC_IPT; ++k) {                                                        \
                    const int64_t i = t * PREC_TILE + thr * PREC_IPT + k;                                   \
                    if (i < n) {                                                                            \
                        if (!(w[i] >= 0.0f) || isinf(w[i])) bad = 1;                                        \
                        acc = acc + (R)w[i];                                                                \
                    }                                                                                       \
                }                                                                                           \
                v[thr] = acc;                                                                               \
            }                                                                                               \
            tv[t] = NAME##_block_scan(v, ex);                                                               \
        }                                                                                                   \
        const R W = NAME##_tile_scan(tv, nt, NULL);                                                         \
        if (W_out) *W_out = (double)W;                                                                      \
        if (bad || !(W > (R)0) || isinf((double)W)) {                                                       \
            free(tv); free(th); free(pl); free(ph); free(cl); free(ch);                                     \
            free(Lkey); free(Hkey); free(Litem); free(Hitem); free(Lprob);                                  \
            return 1;                                                                                       \
        }                                                                                                   \
        const R W_N = W / (R)(double)n;                                                                     \
        /* the lines: per tile, sums in item order; tile bases in tile order; positions b + local */       \
        int64_t nL = 0, nH = 0;                                                                             \
        R bl = (R)0, bh = (R)0;                                                                             \
        for (int64_t t = 0; t < nt; ++t) {                                                                  \
            R sl = (R)0, sh = (R)0;                                                                         \
            for (int64_t i = t * PREC_TILE; i < n && i < (t + 1) * PREC_TILE; ++i) {                        \
                const R wr = (R)w[i];                                                                       \
                if (wr > W_N) {                                                                             \
                    sh = sh + (wr - W_N);                                                                   \
                    Hkey[nH] = bh + sh;                                                                     \
                    Hitem[nH] = (uint32_t)i;                                                                \
                    ++nH;                                                                                   \
                } else {                                                                                    \
                    Lkey[nL] = bl + sl;                                                                     \
                    Litem[nL] = (uint32_t)i;                                                                \
                    const R q = wr / W_N;                                                                   \
                    Lprob[nL] = (float)(q < (R)1 ? q : (R)1);                                               \
                    sl = sl + (W_N - wr);                                                                   \
                    ++nL;                                                                                   \
                }                                                                                           \
            }                                                                                               \
            bl = bl + sl;                                                                                   \
            bh = bh + sh;                                                                                   \
        }                                                                                                   \
        const R A_total = bl;                                                                               \
        /* the merge: heavy j before light i iff Hkey[j] <= Lkey[i] */                                      \
        int64_t i = 0, j = 0;                                                                               \
        while (i < nL || j < nH) {                                                                          \
            if (j < nH && (i >= nL || Hkey[j] <= Lkey[i])) {                                                \
                const R A_next = i < nL ? Lkey[i] : A_total;                                                \
                R rr = (W_N + Hkey[j] - A_next) / W_N;                                                      \
                if (rr > (R)1) rr = (R)1;                                                                   \
                if (!(rr > (R)0)) rr = (R)0;                                                                \
                const uint32_t item = Hitem[j];                                                             \
                rows[2 * (int64_t)item] = f_bits((float)rr);                                                \
                rows[2 * (int64_t)item + 1] = Hitem[j + 1 < nH ? j + 1 : j];                                \
                ++j;                                                                                        \
            } else {                                                                                        \
                const uint32_t item = Litem[i];                                                             \
                rows[2 * (int64_t)item] = f_bits(Lprob[i]);                                                 \
                rows[2 * (int64_t)item + 1] = nH ? Hitem[j < nH ? j : nH - 1] : item;                       \
                ++i;                                                                                        \
            }                                                                                               \
        }                                                                                                   \
        free(tv); free(th); free(pl); free(ph); free(cl); free(ch);                                         \
        free(Lkey); free(Hkey); free(Litem); free(Hitem); free(Lprob);                                      \
        return 0;                                                                                           \
    }

DEFINE_PREC_BUILD(double, prec_build_f64)
DEFINE_PREC_BUILD(float, prec_build_f32)

int or_prec_build(const float* w, int64_t n, int fp64, uint32_t* rows, double* W_out) {
    return fp64 ? prec_build_f64(w, n, rows, W_out) : prec_build_f32(w, n, rows, W_out);
}

/* ------------------------------------------------------------------ sampling */
/* doSample (sampling/aliasTable/SamplerGpuBasic.cu:28-69) with frac := coin and
 * weight := prob * W/N: result = coin < prob ? row : alias (a full row keeps itself). */
static inline uint32_t do_sample(const uint32_t* rows, uint32_t row, uint32_t coin_bits) {
    return coin24(coin_bits) < bits_f(rows[2 * (uint64_t)row]) ? row : rows[2 * (uint64_t)row + 1];
}

/* The sampling contract: output position s uses Philox block counter_base + s; the row from
 * the 64-bit uniform x1:x0, the coin from x2. */
void or_sample_plain(const uint32_t* rows, int64_t n, uint64_t m, uint64_t seed, uint64_t cbase, uint32_t* out) {
    for (uint64_t s = 0; s < m; ++s) {
        uint32_t x[4];
        philox_block(cbase + s, 0, 0, seed, x);
        out[s] = do_sample(rows, row_of(x, (uint64_t)n), x[2]);
    }
}

/* The uniforms that make the reference's doSample (SamplerGpuBasic.cu:28-69: rand = u * N,
 * row = (int)rand, frac = rand - row) decide on the contract's (row, coin) of output position
 * s: u = (row + coin) / n in FP64. For power-of-two n <= 2^29, u * n = row + coin exactly
 * (24 + 29 bits fit in 53), so (int)(u * n) = row and u * n - row = coin. rows_out and
 * coins_out (optional) receive the pair itself. */
void or_plain_replay_uniforms(int64_t n, uint64_t m, uint64_t seed, uint64_t cbase, double* u, uint32_t* rows_out,
                              float* coins_out) {
    for (uint64_t s = 0; s < m; ++s) {
        uint32_t x[4];
        philox_block(cbase + s, 0, 0, seed, x);
        const uint32_t row = row_of(x, (uint64_t)n);
        const float c = coin24(x[2]);
        u[s] = ((double)row + (double)c) / (double)n;
        if (rows_out) rows_out[s] = row;
        if (coins_out) coins_out[s] = c;
    }
}

void or_batched_sample(const uint32_t* rows, const int64_t* off, int64_t num_tables, const int64_t* soff,
                       uint64_t seed, uint64_t cbase, uint32_t* out) {
    for (int64_t t = 0; t < num_tables; ++t) {
        const uint64_t n = (uint64_t)(off[t + 1] - off[t]);
        for (int64_t s = soff[t]; s < soff[t + 1]; ++s) {
            uint32_t x[4];
            philox_block(cbase + (uint64_t)s, 0, 0, seed, x);
            if (n == 0) {
                out[s] = 0xffffffffu;
                continue;
            }
            out[s] = do_sample(rows + 2 * off[t], row_of(x, n), x[2]);
        }
    }
}

/* Mixed batch (kinds[t]: 0 alias, 1 rejection, other: skipped). Alias tables get the rows of
 * or_batched_build; rejection table t gets or_rejection_build's slots at A + 2 off[t] (capacity
 * 2 n_t), its acceptances at frac + off[t] and |A_t| in a_size[t]; both with W the exact sum.
 * Returns the number of tables with invalid or all-zero weights. */
int or_batched_mixed_build(const float* w, const int64_t* off, int64_t num_tables, const uint8_t* kinds,
                           uint32_t* rows, uint32_t* A, float* frac, uint64_t* a_size, double* W_out) {
    int bad = 0;
    for (int64_t t = 0; t < num_tables; ++t) {
        const int64_t n = off[t + 1] - off[t];
        if (n <= 0 || kinds[t] > 1) continue;
        const double W = or_exact_sum_f32(w + off[t], n);
        if (W_out) W_out[t] = W;
        if (!(W > 0.0) || isinf(W)) {
            ++bad;
            continue;
        }
        if (kinds[t] == 0) {
            or_exact_build(w + off[t], n, W, rows + 2 * off[t]);
        } else {
            const uint64_t asz = or_rejection_build(w + off[t], n, W, A + 2 * off[t], 2 * (uint64_t)n, frac + off[t]);
            a_size[t] = asz > 2 * (uint64_t)n ? 0 : asz;
        }
    }
    return bad;
}

/* The mixed sampler: alias positions as or_batched_sample, rejection positions as
 * or_rejection_sample over the global position s (b = cbase + s); skipped tables' positions
 * are left as they are. Returns 1 if a rejection sample ran out of tries. */
int or_batched_mixed_sample(const uint32_t* rows, const uint32_t* A, const float* frac, const uint64_t* a_size,
                            const int64_t* off, int64_t num_tables, const uint8_t* kinds, const int64_t* soff,
                            uint64_t seed, uint64_t cbase, uint32_t max_tries, uint32_t* out) {
    int failed = 0;
    const uint32_t tries = max_tries ? max_tries : 64u;
    for (int64_t t = 0; t < num_tables; ++t) {
        const uint64_t n = (uint64_t)(off[t + 1] - off[t]);
        for (int64_t s = soff[t]; s < soff[t + 1]; ++s) {
            uint32_t x[4];
            if (kinds[t] == 0) {
                philox_block(cbase + (uint64_t)s, 0, 0, seed, x);
                out[s] = n == 0 ? 0xffffffffu : do_sample(rows + 2 * off[t], row_of(x, n), x[2]);
            } else if (kinds[t] == 1) {
                const uint64_t asz = n ? a_size[t] : 0;
                if (asz == 0) {
                    out[s] = 0xffffffffu;
                    continue;
                }
                const uint32_t* At = A + 2 * off[t];
                const uint64_t b = cbase + (uint64_t)s;
                uint32_t res = 0xffffffffu;
                for (uint32_t tr = 0; tr < tries; ++tr) {
                    philox_block(b, tr, 0x52454a00u, seed, x);
                    const uint32_t xc = x[2];
                    const uint32_t e = At[slot_of(x[0], x[1], asz)];
                    const uint32_t item = e & 0x7fffffffu;
                    if ((e >> 31) == 0u || coin24(xc) < frac[off[t] + item]) {
                        res = item;
                        break;
                    }
                }
                if (res == 0xffffffffu) failed = 1;
                out[s] = res;
            }
        }
    }
    return failed;
}

double or_sample_plain_timed(const uint32_t* rows, int64_t n, uint64_t m, uint64_t seed, int threads, uint32_t* out) {
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(static)
#endif
    for (int64_t q = 0; q < (int64_t)m; ++q) {
        uint32_t x[4];
        philox_block((uint64_t)q, 0, 0, seed, x);
        out[q] = do_sample(rows, row_of(x, (uint64_t)n), x[2]);
    }
    (void)threads;
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double dt = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    return (double)m / dt;
}

/* ------------------------------------------------------------------ binomial tree */
/* Deterministic natural log: x = m 2^e, m in (sqrt(2)/2, sqrt(2)], log m = 2 atanh(s). */
static double det_2atanh(double s) {
    double z = s * s;
    double p = 1.0 / 25.0;
    p = p * z + 1.0 / 23.0;
    p = p * z + 1.0 / 21.0;
    p = p * z + 1.0 / 19.0;
    p = p * z + 1.0 / 17.0;
    p = p * z + 1.0 / 15.0;
    p = p * z + 1.0 / 13.0;
    p = p * z + 1.0 / 11.0;
    p = p * z + 1.0 / 9.0;
    p = p * z + 1.0 / 7.0;
    p = p * z + 1.0 / 5.0;
    p = p * z + 1.0 / 3.0;
    double s2 = s + s;
    return s2 + (s2 * z) * p;
}
static double det_log(double x) {
    if (!(x > 0.0)) return -HUGE_VAL;
    uint64_t b = dbits(x);
    int e = (int)((b >> 52) & 0x7ff);
    if (e == 0) {
        x = x * 18014398509481984.0;
        b = dbits(x);
        e = (int)((b >> 52) & 0x7ff) - 54;
    }
    int ex = e - 1023;
    uint64_t mb = (b & 0xfffffffffffffull) | (1023ull << 52);
    double m;
    memcpy(&m, &mb, 8);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        ex += 1;
    }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    return (double)ex * 0.6931471805599453094 + det_2atanh(s);
}
static double det_log1m(double p) {
    if (p < 0.25) {
        double s = p / (2.0 - p);
        return -det_2atanh(s);
    }
    return det_log(1.0 - p);
}
static inline double u53(uint32_t hi, uint32_t lo) {
    uint64_t v = (((uint64_t)hi << 21) ^ ((uint64_t)lo >> 11)) & ((1ull << 53) - 1);
    return (double)v * 1.1102230246251565404e-16;
}
static inline double u53_open0(uint32_t hi, uint32_t lo) {
    uint64_t v = (((uint64_t)hi << 21) ^ ((uint64_t)lo >> 11)) & ((1ull << 53) - 1);
    return (double)(v + 1) * 1.1102230246251565404e-16;
}
static double stirling_fc(double k) {
    if (k < 10.0) {
        double f = 1.0;
        for (double i = 2.0; i <= k; i = i + 1.0) f = f * i;
        double k1 = k + 1.0;
        double half_log_2pi = 0.5 * det_log(6.283185307179586477);
        double r = det_log(f);
        r = r - (k + 0.5) * det_log(k1);
        r = r + k1;
        r = r - half_log_2pi;
        return r;
    }
    double k1 = k + 1.0;
    double k1sq = k1 * k1;
    double t = 1.0 / 360.0 - ((1.0 / 1260.0) / k1sq) / 1.0;
    t = 1.0 / 12.0 - t / k1sq;
    return t / k1;
}
typedef struct {
    uint32_t k0, k1, c0, c1, node;
} BStream;
static void bdraw(const BStream* st, uint32_t iter, uint32_t out[4]) {
    uint32_t ctr[4] = {st->c0, st->c1, st->node, (iter << 8) | 0xA5u};
    uint32_t key[2] = {st->k0, st->k1};
    or_philox4x32_10(ctr, key, out);
}
static uint64_t binom_small(uint64_t n, double p, const BStream* st) {
    if (n == 0 || !(p > 0.0)) return 0;
    double l1m = det_log1m(p);
    uint64_t x = 0;
    double pos = 0.0, nd = (double)n;
    for (uint32_t it = 0; it < 4096; ++it) {
        uint32_t r[4];
        bdraw(st, it, r);
        for (int h = 0; h < 2; ++h) {
            double u = u53_open0(r[2 * h], r[2 * h + 1]);
            double g = floor(det_log(u) / l1m) + 1.0;
            pos = pos + g;
            if (pos > nd) return x;
            ++x;
        }
    }
    return x;
}
/* BTRD: W. Hörmann, "The generation of binomial random variates", JSCS 46 (1993). */
static uint64_t binom_btrd(uint64_t n, double p, const BStream* st) {
    double nd = (double)n;
    double q = 1.0 - p;
    double m = floor((nd + 1.0) * p);
    double r = p / q;
    double nr = (nd + 1.0) * r;
    double npq = (nd * p) * q;
    double spq = sqrt(npq);
    double b = 1.15 + 2.53 * spq;
    double a = (-0.0873 + 0.0248 * b) + 0.01 * p;
    double c = nd * p + 0.5;
    double alpha = (2.83 + 5.1 / b) * spq;
    double vr = 0.92 - 4.2 / b;
    double urvr = 0.86 * vr;
    for (uint32_t it = 0; it < 256; ++it) {
        uint32_t wv[4];
        bdraw(st, it, wv);
        double v = u53(wv[0], wv[1]);
        double u;
        if (v <= urvr) {
            u = v / vr - 0.43;
            double au = u < 0.0 ? -u : u;
            double kk = floor(((2.0 * a) / (0.5 - au) + b) * u + c);
            if (kk < 0.0) return 0;
            if (kk > nd) return n;
            return (uint64_t)kk;
        }
        if (v >= vr) {
            u = u53(wv[2], wv[3]) - 0.5;
        } else {
            u = v / vr - 0.93;
            u = (u < 0.0 ? -0.5 : 0.5) - u;
            v = u53(wv[2], wv[3]) * vr;
        }
        double au = u < 0.0 ? -u : u;
        double us = 0.5 - au;
        double kk = floor(((2.0 * a) / us + b) * u + c);
        if (kk < 0.0 || kk > nd) continue;
        v = (v * alpha) / (a / (us * us) + b);
        double km = kk > m ? kk - m : m - kk;
        if (km <= 15.0) {
            double f = 1.0;
            if (m < kk) {
                for (double i = m + 1.0; i <= kk; i = i + 1.0) f = f * (nr / i - r);
            } else if (m > kk) {
                for (double i = kk + 1.0; i <= m; i = i + 1.0) v = v * (nr / i - r);
            }
            if (v <= f) return (uint64_t)kk;
            continue;
        }
        v = det_log(v);
        double rho = (km / npq) * ((((km / 3.0 + 0.625) * km) + 1.0 / 6.0) / npq + 0.5);
        double t = -(km * km) / (2.0 * npq);
        if (v < t - rho) return (uint64_t)kk;
        if (v > t + rho) continue;
        double nm = (nd - m) + 1.0;
        double h = ((m + 0.5) * det_log((m + 1.0) / (r * nm)) + stirling_fc(m)) + stirling_fc(nd - m);
        double nk = (nd - kk) + 1.0;
        double rhs = h + (nd + 1.0) * det_log(nm / nk);
        rhs = rhs + (kk + 0.5) * det_log((nk * r) / (kk + 1.0));
        rhs = rhs - stirling_fc(kk);
        rhs = rhs - stirling_fc(nd - kk);
        if (v <= rhs) return (uint64_t)kk;
    }
    return (uint64_t)m;
}
static uint64_t binomial_st(uint64_t n, double p, const BStream* st) {
    if (n == 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    int flip = p > 0.5;
    double pp = flip ? 1.0 - p : p;
    uint64_t x = ((double)n * pp < 10.0) ? binom_small(n, pp, st) : binom_btrd(n, pp, st);
    return flip ? n - x : x;
}
uint64_t or_binomial(uint64_t n, double p, uint32_t k0, uint32_t k1, uint64_t cbase, uint32_t node) {
    BStream st = {k0, k1, (uint32_t)cbase, (uint32_t)(cbase >> 32), node};
    return binomial_st(n, p, &st);
}
static inline uint64_t section_rows(uint64_t a, uint64_t b, uint64_t S, uint64_t n) {
    uint64_t hi = b * S < n ? b * S : n;
    return hi - a * S;
}
static void tree(uint64_t lo, uint64_t hi, uint64_t cnt, uint32_t node, uint64_t S, uint64_t n, BStream* st,
                 uint64_t* counts) {
    if (hi - lo == 1) {
        counts[lo] = cnt;
        return;
    }
    uint64_t mid = lo + (hi - lo) / 2;
    double pl = (double)section_rows(lo, mid, S, n) / (double)section_rows(lo, hi, S, n);
    st->node = node;
    uint64_t cl = binomial_st(cnt, pl, st);
    tree(lo, mid, cl, 2 * node, S, n, st, counts);
    tree(mid, hi, cnt - cl, 2 * node + 1, S, n, st, counts);
}
void or_section_counts(int64_t n, uint32_t S, uint64_t m, uint64_t seed, uint64_t cbase, uint64_t* counts) {
    uint64_t K = ((uint64_t)n + S - 1) / S;
    BStream st = {(uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)cbase, (uint32_t)(cbase >> 32), 1};
    tree(0, K, m, 1, S, (uint64_t)n, &st, counts);
}
void or_sample_sectioned(const uint32_t* rows, int64_t n, uint64_t m, uint32_t S, uint64_t seed, uint64_t cbase,
                         uint32_t* out, uint64_t* counts) {
    uint64_t K = ((uint64_t)n + S - 1) / S;
    or_section_counts(n, S, m, seed, cbase, counts);
    uint64_t off = 0;
    for (uint64_t k = 0; k < K; ++k) {
        uint32_t start = (uint32_t)(k * S);
        uint32_t len = (uint32_t)section_rows(k, k + 1, S, (uint64_t)n);
        for (uint64_t s = off; s < off + counts[k]; ++s) {
            uint32_t x[4];
            philox_block(cbase + s, 0, 0, seed, x);
            out[s] = do_sample(rows, start + row_of(x, len), x[2]);
        }
        off += counts[k];
    }
}

/* ------------------------------------------------------------------ rejection */
/* RejectionSampling::build (construction/rejectionSampling/RejectionSampling.cu:35-56) with
 * CalcNumOccurrencesOperator (:26-33) and a sequential fillA (RejectionSamplingDirect.cu:12-28). */
uint64_t or_rejection_build(const float* w, int64_t n, double W, uint32_t* A, uint64_t cap, float* frac) {
    double nd = (double)n;
    uint64_t pos = 0;
    for (int64_t i = 0; i < n; ++i) {
        double x = (nd * (double)w[i]) / W;
        double fl = floor(x);
        uint32_t c = (uint32_t)fl + 1u;
        frac[i] = (float)(x - fl);
        for (uint32_t t = 0; t < c; ++t)
            if (pos + t < cap) A[pos + t] = (uint32_t)i | (t == 0 ? 0x80000000u : 0u);
        pos += c;
    }
    return pos;
}

/* SamplerRejection::sample (sampling/rejectionSampling/SamplerRejection.cu:17-35). */
int or_rejection_sample(const uint32_t* A, uint64_t a_size, const float* frac, uint64_t m, uint64_t seed,
                        uint64_t cbase, uint32_t max_tries, uint32_t* out) {
    int failed = 0;
    uint32_t tries = max_tries ? max_tries : 64u;
    for (uint64_t s = 0; s < m; ++s) {
        uint64_t b = cbase + s;
        uint32_t res = 0xffffffffu, x[4];
        for (uint32_t t = 0; t < tries; ++t) {
            philox_block(b, t, 0x52454a00u, seed, x);
            uint32_t xc = x[2];
            uint32_t e = A[slot_of(x[0], x[1], a_size)];
            uint32_t item = e & 0x7fffffffu;
            if ((e >> 31) == 0u || coin24(xc) < frac[item]) {
                res = item;
                break;
            }
        }
        if (res == 0xffffffffu) failed = 1;
        out[s] = res;
    }
    return failed;
}
