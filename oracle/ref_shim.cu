/*
 * ref_shim.cu — C entry points over the reference's own CPU code, compiled together with
 * the reference sources read in place from the reference checkout (see oracle/Makefile).
 *
 * TEST INFRASTRUCTURE ONLY: the compiled reference is the oracle's cross-check and the
 * timed CPU baseline; it never runs inside the library.
 *
 * Weights are injected through the public `weights` member after construction, as the
 * reference itself does in plots/PlotConstruction.cuh:207-224.
 */
#include <chrono>
#include <cstring>
#include <vector>

#include "construction/aliasTable/buildMethod/AliasTableNp.cuh"
#include "construction/aliasTable/buildMethod/AliasTableSplit.cuh"
#include "construction/aliasTable/buildMethod/AliasTableStack.cuh"
#include "construction/aliasTable/buildMethod/AliasTableSweep.cuh"
#include "construction/aliasTable/packMethod/PackMethodSweep.cuh"
#include "construction/aliasTable/splitMethod/SplitMethodBasic.cuh"
#include "sampling/aliasTable/SamplerCpu.cuh"
#include "utils/PrefixSum.cuh"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
template <typename Table>
void export_table(Table& t, int n, double* weight, int* alias) {
    for (int i = 0; i < n; ++i) {
        weight[i] = t.aliasTable.weight(i);
        alias[i] = t.aliasTable.alias(i);
    }
}
}  // namespace

extern "C" {

/* AliasTableSplit<ArrayOfStructs>::build (AliasTableSplit.cu:24-80), 1 core as shipped. */
int ref_split_build(const double* w, int n, int p, double* weight, int* alias, double* W, double* seconds) {
    AliasTableSplit<ArrayOfStructs> t(n, p, weightDistributionSine);
    std::memcpy(t.weights.data, w, sizeof(double) * n);
    auto t0 = std::chrono::steady_clock::now();
    t.build();
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    export_table(t, n, weight, alias);
    if (W) *W = t.W;
    return 0;
}

/* AliasTableSweep::build (AliasTableSweep.cu:12-60). */
int ref_sweep_build(const double* w, int n, double* weight, int* alias, double* W, double* seconds) {
    AliasTableSweep t(n, weightDistributionSine);
    std::memcpy(t.weights.data, w, sizeof(double) * n);
    for (int i = 0; i < n; ++i) {
        t.aliasTable.weight(i) = 0;
        t.aliasTable.alias(i) = -1;
    }
    auto t0 = std::chrono::steady_clock::now();
    t.build();
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    export_table(t, n, weight, alias);
    if (W) *W = t.W;
    return 0;
}

/* AliasTableStack::build (AliasTableStack.cu:11-39). */
int ref_stack_build(const double* w, int n, double* weight, int* alias, double* W, double* seconds) {
    AliasTableStack t(n, weightDistributionSine);
    std::memcpy(t.weights.data, w, sizeof(double) * n);
    for (int i = 0; i < n; ++i) t.aliasTable.alias(i) = -1;
    auto t0 = std::chrono::steady_clock::now();
    t.build();
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    export_table(t, n, weight, alias);
    if (W) *W = t.W;
    return 0;
}

/* AliasTable::verifyTableCorrectness (AliasTable.cu:24-65) on a reference-format table
 * (active only in the debug build of this library; the Release build returns 1). */
int ref_verify(const double* w, int n, const double* weight, const int* alias, double W) {
    AliasTableSweep t(n, weightDistributionSine);
    std::memcpy(t.weights.data, w, sizeof(double) * n);
    t.W = W;
    for (int i = 0; i < n; ++i) {
        t.aliasTable.weight(i) = weight[i];
        t.aliasTable.alias(i) = alias[i];
    }
    return t.verifyTableCorrectness() ? 1 : 0;
}

/* AliasTableNp best / worst case tables (AliasTableNp.cu:24-47) for weights of size n. */
int ref_np_table(int n, int best, double* w_out, double* weight, int* alias, double* W) {
    AliasTableNp<ArrayOfStructs> t(n, best != 0);
    t.build();
    std::memcpy(w_out, t.weights.data, sizeof(double) * n);
    export_table(t, n, weight, alias);
    if (W) *W = t.W;
    return 0;
}

/* The reference's synthetic generators (SamplingAlgorithm.cu:21-71) for the deterministic
 * distributions (Sine, BestWorstCase, Ramp, PowerLaw1, PowerLaw2, OneHeavy, OneLight). */
int ref_generate(int n, int distribution, double* w_out) {
    AliasTableStack t(n, (WeightDistribution)distribution);
    std::memcpy(w_out, t.weights.data, sizeof(double) * n);
    return 0;
}

/* All-core harness over the reference's own split and pack functions: the body of
 * AliasTableSplit::build with its loops over k (disjoint outputs) on `threads` cores. */
int ref_split_build_parallel(const double* w, int n, int p, int threads, double* weight, int* alias, double* W_out,
                             double* seconds) {
    AliasTableSplit<ArrayOfStructs> t(n, p, weightDistributionSine);
    std::memcpy(t.weights.data, w, sizeof(double) * n);
    auto t0 = std::chrono::steady_clock::now();
    const int N = n;
    double W = 0;
    for (int i = 0; i < N; i++) W += t.weights[i];
    t.W = W;
    t.weights[N] = std::numeric_limits<double>::infinity();
    t.weights[N + 1] = 0;
    for (int i = 0; i < N; i++) t.aliasTable.weight(i) = t.weights[i];
    SafeArray<int> pre(N + 2, HOST);
    for (int i = 0; i < N + 2; i++) pre[i] = (t.weights[i] > W / N) ? 1 : 0;
    PrefixSum::exclusivePrefixSum<int>(pre, pre);
    const int numH = pre[N + 1];
    const int numL = (N + 2) - numH;
    SafeArray<LH_TYPE> l(numL, HOST), h(numH, HOST);
    SafeArray<double> pL(numL, HOST), pH(numH, HOST);
    SafeArray<SplitConfig> splits(p + 1, HOST);
    for (int i = 0; i < N + 2; i++) {
        if (t.weights[i] > W / N) {
            h[pre[i]].item = i;
            h[pre[i]].setWeight(t.weights[i]);
            pH[pre[i]] = t.weights[i];
        } else {
            l[i - pre[i]].item = i;
            l[i - pre[i]].setWeight(t.weights[i]);
            pL[i - pre[i]] = t.weights[i];
        }
    }
    PrefixSum::exclusivePrefixSum<double>(pL, pL);
    PrefixSum::exclusivePrefixSum<double>(pH, pH);
    SplitMethodBasic::split(1, splits, N, W, p, t.weights, h, pH, numH, pL, numL);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(dynamic, 8)
#endif
    for (int k = 2; k <= p - 1; k++) SplitMethodBasic::split(k, splits, N, W, p, t.weights, h, pH, numH, pL, numL);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(dynamic, 8)
#endif
    for (int k = 1; k <= p; k++) PackMethodSweep::pack<ArrayOfStructs>(k, splits, W / N, h, l, t.aliasTable, t.weights);
    auto t1 = std::chrono::steady_clock::now();
    (void)threads;
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    export_table(t, n, weight, alias);
    if (W_out) *W_out = W;
    pre.free();
    l.free();
    h.free();
    pL.free();
    pH.free();
    splits.free();
    return 0;
}

/* SamplerCpu::sample() (SamplerCpu.cu:12-18) on a given table, timed; `out` optional. */
double ref_sampler_cpu(const double* weight, const int* alias, int n, double W, long long num_samples, int* out) {
    AliasTableSweep t(n, weightDistributionSine);
    t.W = W;
    for (int i = 0; i < n; ++i) {
        t.aliasTable.weight(i) = weight[i];
        t.aliasTable.alias(i) = alias[i];
    }
    SamplerCpu s(t);
    long long acc = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (long long i = 0; i < num_samples; ++i) {
        int v = s.sample();
        if (out) out[i] = v;
        acc += v;
    }
    auto t1 = std::chrono::steady_clock::now();
    volatile long long sink = acc;
    (void)sink;
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
