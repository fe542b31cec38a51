/*
 * ref_harness.cu — the reference's own test harness run against this library (test
 * infrastructure: compiled with the reference's headers and sources read in place from the
 * reference checkout, see oracle/Makefile target `ref`; nothing of the reference is copied).
 *
 * AliasTableWrs<TableStorage> is a reference SamplingAlgorithm (an AliasTable, the class the
 * reference's experiments and tests drive, construction/aliasTable/AliasTable.cuh) whose build
 * is this library's wrs_alias_build_f32, exported to the reference's row format by
 * wrs_export_reference_table; its postBuild() is the reference's own verifyTableCorrectness
 * (AliasTable.cu:24-65, active since this harness is built without NDEBUG). SamplerWrs is a
 * reference Sampler (sampling/Sampler.cuh) over wrs_alias_sample. The case list is that of
 * UnitTests::testTableCorrectness and ::testSamplingDistribution (UnitTests.cu:10-145): every
 * weight distribution at 10^4 and 10^6 items, both build methods and both row formats, the
 * (505711 items, OneLight) regression case, 20 random cases (sizes 10^2..10^7, random
 * distribution and method) from a fixed seed, and the sampled distribution of a 10^4-item
 * sine table against the expected counts (SamplerExpected) for the reference's SamplerCpu and
 * this library's plain and sectioned samplers. Exit status 0 when every case passes. Cases whose
 * absolute tolerance is finer than the FP32 rows can hold at the weights' own scale are checked
 * at mean 1 and counted ("scaled=" in the summary line).
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "construction/aliasTable/AliasTable.cuh"
#include "sampling/aliasTable/SamplerCpu.cuh"
#include "sampling/aliasTable/SamplerExpected.cuh"
#include "wrs.h"

namespace {

#define CK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            std::cerr << "CUDA error " << cudaGetErrorString(e_) << " at " << __LINE__ \
                      << std::endl;                                                    \
            std::exit(3);                                                              \
        }                                                                              \
    } while (0)

template <typename TS>
void set_row(TS& t, int i, double weight, int alias) {
    t.weight(i) = weight;
    t.alias(i) = alias;
}

template <typename TS>
class AliasTableWrs : public AliasTable<TS> {
   public:
    AliasTableWrs(int size, WeightDistribution distribution, uint32_t method)
        : AliasTable<TS>(size, distribution), method_(method) {}
    ~AliasTableWrs() {
        if (d_table_) cudaFree(d_table_);
    }
    std::string name() override {
        return std::string("AliasTableWrs<") + TS::name() + (method_ == WRS_METHOD_PSA_PLUS ? ", psa+>" : ", split>");
    }
    // The weights (FP64 in the reference's objects) go to the device as FP32.
    void preBuild() override {
        const int n = this->N;
        std::vector<float> w32(n);
        for (int i = 0; i < n; ++i) w32[i] = (float)this->weights[i];
        opts_ = wrs_build_opts{};
        opts_.method = method_;
        opts_.flags = WRS_FLAG_SYNC;
        scratch_bytes_ = wrs_alias_build_scratch_bytes(n, &opts_);
        CK(cudaMalloc(&d_w_, sizeof(float) * n));
        CK(cudaMalloc(&d_table_, sizeof(wrs_alias_row) * n));
        CK(cudaMalloc(&d_scratch_, scratch_bytes_));
        CK(cudaMalloc(&d_W_, sizeof(double)));
        CK(cudaMemcpy(d_w_, w32.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    }
    void build() override {
        status_ = wrs_alias_build_f32(d_w_, this->N, &opts_, d_table_, d_W_, d_scratch_, scratch_bytes_, nullptr);
    }
    // The table in the reference's row format, then the reference's own check.
    bool postBuild() override {
        const int n = this->N;
        bool ok = status_ == WRS_SUCCESS;
        if (!ok) std::cerr << name() << ": " << wrs_status_string(status_) << std::endl;
        double W = 0;
        CK(cudaMemcpy(&W, d_W_, sizeof(double), cudaMemcpyDeviceToHost));
        this->W = W;  // the weight total the table was built with
        double* d_weight = nullptr;
        int32_t* d_alias = nullptr;
        CK(cudaMalloc(&d_weight, sizeof(double) * n));
        CK(cudaMalloc(&d_alias, sizeof(int32_t) * n));
        if (ok && wrs_export_reference_table(d_table_, n, W, d_weight, d_alias, nullptr) != WRS_SUCCESS) ok = false;
        std::vector<double> weight(n);
        std::vector<int32_t> alias(n);
        CK(cudaMemcpy(weight.data(), d_weight, sizeof(double) * n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(alias.data(), d_alias, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n; ++i) set_row(this->aliasTable, i, weight[i], alias[i]);
        cudaFree(d_weight);
        cudaFree(d_alias);
        cudaFree(d_w_);
        cudaFree(d_scratch_);
        cudaFree(d_W_);
        d_w_ = nullptr;
        d_scratch_ = nullptr;
        d_W_ = nullptr;
        return ok && this->verifyTableCorrectness();
    }
    const wrs_alias_row* device_table() const { return d_table_; }

   private:
    uint32_t method_;
    wrs_build_opts opts_{};
    size_t scratch_bytes_ = 0;
    float* d_w_ = nullptr;
    wrs_alias_row* d_table_ = nullptr;
    void* d_scratch_ = nullptr;
    double* d_W_ = nullptr;
    wrs_status status_ = WRS_ERR_INVALID_ARGUMENT;
};

// A reference Sampler over this library's sampler: getSamplingDistribution counts the samples
// on the device (WRS_SAMPLE_HISTOGRAM) or, sectioned, counts the written samples.
class SamplerWrs : public Sampler {
   public:
    SamplerWrs(AliasTableWrs<ArrayOfStructs>& table, uint32_t section_items)
        : table_(table), section_items_(section_items) {}
    std::string name() override {
        return section_items_ ? "SamplerWrsSectioned" : "SamplerWrsPlain";
    }
    std::vector<int> getSamplingDistribution(int numSamples) override {
        const int n = table_.N;
        std::vector<int> out(n, 0);
        wrs_sample_opts o{};
        uint32_t* d_out = nullptr;
        if (section_items_ == 0) {
            o.mode = WRS_SAMPLE_HISTOGRAM;
            CK(cudaMalloc(&d_out, sizeof(uint32_t) * n));
            CK(cudaMemset(d_out, 0, sizeof(uint32_t) * n));
            if (wrs_alias_sample(table_.device_table(), n, numSamples, 0xABCDull, 0, &o, d_out, nullptr, nullptr) !=
                WRS_SUCCESS)
                std::exit(4);
            std::vector<uint32_t> h(n);
            CK(cudaMemcpy(h.data(), d_out, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i) out[i] = (int)h[i];
        } else {
            o.mode = WRS_SAMPLE_SECTIONED;
            o.section_items = section_items_;
            CK(cudaMalloc(&d_out, sizeof(uint32_t) * numSamples));
            if (wrs_alias_sample(table_.device_table(), n, numSamples, 0xABCDull, 0, &o, d_out, nullptr, nullptr) !=
                WRS_SUCCESS)
                std::exit(4);
            std::vector<uint32_t> h(numSamples);
            CK(cudaMemcpy(h.data(), d_out, sizeof(uint32_t) * numSamples, cudaMemcpyDeviceToHost));
            for (uint32_t s : h) {
                if (s < (uint32_t)n) ++out[s];
            }
        }
        cudaFree(d_out);
        return out;
    }

   protected:
    double executeBenchmarkSampling(int numSamples, int* distributionOutput) override {
        (void)distributionOutput;
        const int n = table_.N;
        uint32_t* d_out = nullptr;
        CK(cudaMalloc(&d_out, sizeof(uint32_t) * (size_t)numSamples));
        wrs_sample_opts o{};
        o.mode = section_items_ ? WRS_SAMPLE_SECTIONED : WRS_SAMPLE_PLAIN;
        o.section_items = section_items_;
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a);
        wrs_alias_sample(table_.device_table(), n, numSamples, 1, 0, &o, d_out, nullptr, nullptr);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        cudaFree(d_out);
        return numSamples / (ms * 1e6);  // Gsamples/s, as Sampler::benchmarkSampling reports
    }

   private:
    AliasTableWrs<ArrayOfStructs>& table_;
    uint32_t section_items_;
};

int g_cases = 0, g_failures = 0;

void check(bool ok, const std::string& what) {
    ++g_cases;
    if (!ok) ++g_failures;
    std::cout << (ok ? "ok     " : "FAILED ") << what << std::endl;
}

int g_scaled = 0;

// The reference's check is absolute: every item's reconstructed weight within
// max(n 1e-8, 1e-3) of its weight. A row stores its probability in FP32, so an item's weight is
// held to about 2^-22 of the largest weight; where the check's tolerance is below that at the
// weights' own scale (large tables of large weights, e.g. a ramp over millions of items), the
// case is checked on the same weights scaled to mean 1 (an alias table of c w is that of w) and
// reported as such.
template <typename TS>
void table_case(int n, WeightDistribution d, uint32_t method) {
    AliasTableWrs<TS> t(n, d, method);
    double W = 0, mx = 0;
    for (int i = 0; i < n; ++i) {
        W += t.weights[i];
        mx = std::max(mx, t.weights[i]);
    }
    const double tol = std::max(n * 1e-8, 1e-3);
    const bool scaled = tol < 2.4e-7 * mx;
    if (scaled) {
        const double s = n / W;
        for (int i = 0; i < n; ++i) t.weights[i] *= s;
        ++g_scaled;
    }
    const bool ok = t.fullBuild();
    check(ok, t.name() + " n=" + std::to_string(n) + " distribution=" + std::to_string((int)d) +
                  (scaled ? " (weights scaled to mean 1)" : ""));
}

}  // namespace

int main() {
    // UnitTests::testTableCorrectness (UnitTests.cu:10-94): every distribution
    for (int d = 1; d <= MAX_WEIGHT_DISTRIBUTION; ++d) {
        const WeightDistribution dist = (WeightDistribution)d;
        table_case<ArrayOfStructs>(10000, dist, WRS_METHOD_SPLIT);
        table_case<StructOfArrays>(10000, dist, WRS_METHOD_SPLIT);
        table_case<ArrayOfStructs>(10000, dist, WRS_METHOD_PSA_PLUS);
        table_case<ArrayOfStructs>(1000000, dist, WRS_METHOD_SPLIT);
    }
    // the regression case (a group with no thread eligible for packing in the reference)
    table_case<ArrayOfStructs>(505711, weightDistributionOneLight, WRS_METHOD_PSA_PLUS);
    table_case<ArrayOfStructs>(505711, weightDistributionOneLight, WRS_METHOD_SPLIT);
    // 20 random cases from a fixed seed: size 100 + r % 10^(3 + r % 5), a random distribution and
    // build method, both row formats
    srand(0x5EED);
    for (int i = 0; i < 20; ++i) {
        const int n_max = (int)std::pow(10, 3 + (rand() % 5));
        const int n = 100 + rand() % n_max;
        const WeightDistribution dist = (WeightDistribution)((rand() % MAX_WEIGHT_DISTRIBUTION) + 1);
        const uint32_t method = (rand() % 2) ? WRS_METHOD_PSA_PLUS : WRS_METHOD_SPLIT;
        table_case<ArrayOfStructs>(n, dist, method);
        table_case<StructOfArrays>(n, dist, WRS_METHOD_SPLIT);
    }

    // UnitTests::testSamplingDistribution (UnitTests.cu:96-145)
    const int numSamples = 2000000, tableSize = 10000;
    AliasTableWrs<ArrayOfStructs> table(tableSize, weightDistributionSine, WRS_METHOD_SPLIT);
    check(table.fullBuild(), table.name() + " (sampling table)");
    const std::vector<int> expected = SamplerExpected(table).getSamplingDistribution(numSamples);
    std::vector<Sampler*> samplers = {new SamplerCpu(table), new SamplerWrs(table, 0),
                                      new SamplerWrs(table, tableSize / 4)};
    for (Sampler* s : samplers) {
        const std::vector<int> got = s->getSamplingDistribution(numSamples);
        long total = 0;
        int worst = 0;
        bool ok = true;
        for (int k = 0; k < tableSize; ++k) {
            const int diff = std::abs(expected[k] - got[k]);
            worst = std::max(worst, diff);
            total += got[k];
            if (diff >= numSamples / tableSize) ok = false;
        }
        check(ok && total == numSamples,
              s->name() + " distribution (largest |expected - sampled| = " + std::to_string(worst) + ")");
        delete s;
    }
    std::cout << "cases=" << g_cases << " failures=" << g_failures << " scaled=" << g_scaled << std::endl;
    return g_failures ? 1 : 0;
}
