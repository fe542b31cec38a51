/* wrs.hpp — C++17 shim of the reference's object surface over the C ABI (wrs.h).
 *
 * Code written against the reference's classes keeps its shape: an algorithm object is built
 * with fullBuild() (= preBuild(); build(); return postBuild();) and a sampler bound to it
 * answers name(), benchmarkSampling(n) and getSamplingDistribution(n):
 *
 *   SamplingAlgorithm   <- construction/SamplingAlgorithm.cuh:30-48 (weights, W, N, fullBuild)
 *   AliasTableSplitGpu  <- construction/aliasTable/buildMethod/AliasTableSplitGpu.cuh (split;
 *                          PSA+ with WRS_METHOD_PSA_PLUS)
 *   RejectionSamplingGpu <- construction/rejectionSampling/RejectionSampling.cuh:13-29
 *   Sampler             <- sampling/Sampler.cuh:10-31 (benchmarkSampling in Gsamples/s,
 *                          getSamplingDistribution as per-item counts)
 *   SamplerGpuBasic, SamplerGpuSectioned, SamplerRejection
 *                       <- sampling/aliasTable/SamplerGpuBasic.cuh, SamplerGpuSectioned.cuh,
 *                          sampling/rejectionSampling/SamplerRejection.cuh
 *   BatchedAliasTablesGpu, SamplerBatched
 *                       <- a loop of AliasTableSplitGpu / SamplerGpuBasic objects, one per table
 *                          (the reference has no batched form)
 *
 * Differences, as in the C ABI: weights are FP32 (the reference holds FP64 host weights), the
 * table rows are {float prob, uint32 alias} on the device, and samples are a function of
 * (seed, counter) through Philox4x32-10; each sampler call advances its counter. The shim
 * allocates device memory with cudaMalloc (the C ABI itself never does) and frees it in its
 * destructors; errors throw wrs::Error instead of raising SIGTRAP. Header-only: link with the
 * library (libwrs.so) and the CUDA runtime.
 */
#ifndef WRS_HPP
#define WRS_HPP

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "wrs.h"

namespace wrs {

class Error : public std::runtime_error {
public:
    Error(wrs_status s, const std::string& what)
        : std::runtime_error(what + ": " + wrs_status_string(s)), status(s) {}
    wrs_status status;
};

inline void check(wrs_status s, const char* what) {
    if (s != WRS_SUCCESS) throw Error(s, what);
}
inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(WRS_ERR_CUDA, std::string(what) + " (" + cudaGetErrorString(e) + ")");
}

// Owning device buffer (move-only).
template <class T>
class DeviceArray {
public:
    DeviceArray() = default;
    explicit DeviceArray(size_t count) { resize(count); }
    ~DeviceArray() { release(); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DeviceArray& operator=(DeviceArray&& o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    void resize(size_t count) {
        if (count == n_) return;
        release();
        if (count) check_cuda(cudaMalloc(reinterpret_cast<void**>(&p_), count * sizeof(T)), "cudaMalloc");
        n_ = count;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    size_t bytes() const { return n_ * sizeof(T); }
    std::vector<T> to_host(cudaStream_t s = nullptr) const {
        std::vector<T> h(n_);
        if (n_) {
            check_cuda(cudaMemcpyAsync(h.data(), p_, bytes(), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
            check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        }
        return h;
    }

private:
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* p_ = nullptr;
    size_t n_ = 0;
};

// ---------------------------------------------------------------- algorithms

class SamplingAlgorithm {
public:
    explicit SamplingAlgorithm(std::vector<float> w, cudaStream_t stream = nullptr)
        : weights(std::move(w)), N(static_cast<int64_t>(weights.size())), stream_(stream) {}
    virtual ~SamplingAlgorithm() = default;
    virtual std::string name() = 0;
    virtual void preBuild() = 0;   // device buffers and the weights' upload
    virtual void build() = 0;      // the build itself (stream-ordered)
    virtual bool postBuild() = 0;  // waits, reads the device status and W
    bool fullBuild() {
        preBuild();
        build();
        return postBuild();
    }
    cudaStream_t stream() const { return stream_; }
    const float* deviceWeights() const { return weights_dev_.get(); }

    std::vector<float> weights;  // host copy, FP32
    double W = 0.0;              // weight total the build used (correctly rounded sum)
    int64_t N;

protected:
    void upload() {
        weights_dev_.resize(weights.size());
        if (!weights.empty())
            check_cuda(cudaMemcpyAsync(weights_dev_.get(), weights.data(), weights_dev_.bytes(),
                                       cudaMemcpyHostToDevice, stream_), "weights upload");
    }
    cudaStream_t stream_;
    DeviceArray<float> weights_dev_;
    DeviceArray<double> W_dev_{1};
};

class AliasTableSplitGpu : public SamplingAlgorithm {
public:
    explicit AliasTableSplitGpu(std::vector<float> w, uint32_t method = WRS_METHOD_SPLIT, uint32_t tile_items = 0,
                                cudaStream_t stream = nullptr)
        : SamplingAlgorithm(std::move(w), stream) {
        opts_.method = method;
        opts_.tile_items = tile_items;
        opts_.flags = 0;
        opts_.small_table_items = 0;
    }
    std::string name() override {
        return opts_.method == WRS_METHOD_PSA_PLUS ? "AliasTableSplitGpu<PsaPlus>" : "AliasTableSplitGpu";
    }
    void preBuild() override {
        upload();
        table_.resize((size_t)N);
        scratch_.resize(wrs_alias_build_scratch_bytes(N, &opts_));
    }
    void build() override {
        check(wrs_alias_build_f32(deviceWeights(), N, &opts_, table_.get(), W_dev_.get(), scratch_.get(),
                                  scratch_.bytes(), stream_), "alias build");
    }
    bool postBuild() override {
        check(wrs_scratch_status(scratch_.get(), stream_), "alias build (device)");
        W = W_dev_.to_host(stream_)[0];
        return true;
    }
    const wrs_alias_row* deviceTable() const { return table_.get(); }
    std::vector<wrs_alias_row> hostTable() const { return table_.to_host(stream_); }

private:
    wrs_build_opts opts_{};
    DeviceArray<wrs_alias_row> table_;
    DeviceArray<unsigned char> scratch_;
};

class RejectionSamplingGpu : public SamplingAlgorithm {
public:
    explicit RejectionSamplingGpu(std::vector<float> w, cudaStream_t stream = nullptr)
        : SamplingAlgorithm(std::move(w), stream) {}
    std::string name() override { return "RejectionSamplingGpu"; }
    void preBuild() override {
        upload();
        A_.resize(2 * (size_t)N);
        frac_.resize((size_t)N);
        scratch_.resize(wrs_rejection_build_scratch_bytes(N));
    }
    void build() override {
        check(wrs_rejection_build_f32(deviceWeights(), N, A_.get(), A_.size(), frac_.get(), a_size_.get(),
                                      W_dev_.get(), scratch_.get(), scratch_.bytes(), 0u, stream_),
              "rejection build");
    }
    bool postBuild() override {
        check(wrs_scratch_status(scratch_.get(), stream_), "rejection build (device)");
        W = W_dev_.to_host(stream_)[0];
        slots = a_size_.to_host(stream_)[0];
        // the slots packed with the first slots' fractions: one gather per try when sampling
        packed_.resize(slots ? (size_t)slots : 1);
        check(wrs_rejection_pack(A_.get(), a_size_.get(), frac_.get(), N, packed_.size(), packed_.get(), stream_),
              "rejection pack");
        return true;
    }
    const uint32_t* deviceA() const { return A_.get(); }
    const float* deviceFrac() const { return frac_.get(); }
    const uint64_t* deviceASize() const { return a_size_.get(); }
    const uint64_t* devicePacked() const { return packed_.get(); }
    uint64_t packedCapacity() const { return packed_.size(); }
    uint64_t slots = 0;  // |A|

private:
    DeviceArray<uint64_t> packed_;
    DeviceArray<uint32_t> A_;
    DeviceArray<float> frac_;
    DeviceArray<uint64_t> a_size_{1};
    DeviceArray<unsigned char> scratch_;
};

// ---------------------------------------------------------------- samplers

class Sampler {
public:
    explicit Sampler(uint64_t seed) : seed_(seed) {}
    virtual ~Sampler() = default;
    virtual std::string name() = 0;
    // numSamples samples into d_out (device, u32), stream-ordered; advances the counter.
    virtual void sample(uint64_t numSamples, uint32_t* d_out) = 0;
    // Per-item counts of numSamples samples.
    virtual std::vector<int64_t> getSamplingDistribution(uint64_t numSamples) {
        DeviceArray<uint32_t> out(numSamples);
        sample(numSamples, out.get());
        const std::vector<uint32_t> h = out.to_host(stream());
        std::vector<int64_t> counts((size_t)items(), 0);
        for (uint32_t v : h)
            if (v < counts.size()) ++counts[v];
        return counts;
    }
    // Samples per second (in 10^9), device-timed with CUDA events around one call.
    double benchmarkSampling(uint64_t numSamples) {
        DeviceArray<uint32_t> out(numSamples);
        sample(numSamples, out.get());  // warm-up
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        check_cuda(cudaEventRecord(e0, stream()), "cudaEventRecord");
        sample(numSamples, out.get());
        check_cuda(cudaEventRecord(e1, stream()), "cudaEventRecord");
        check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return (double)numSamples / ((double)ms * 1e-3) / 1e9;
    }
    uint64_t counter = 0;  // the next call's Philox counter base

protected:
    virtual cudaStream_t stream() const = 0;
    virtual int64_t items() const = 0;
    uint64_t seed_;
};

class SamplerGpuBasic : public Sampler {
public:
    explicit SamplerGpuBasic(AliasTableSplitGpu& a, uint64_t seed = 0x5EED) : Sampler(seed), a_(a) {}
    std::string name() override { return "SamplerGpuBasic"; }
    void sample(uint64_t numSamples, uint32_t* d_out) override {
        wrs_sample_opts o{WRS_SAMPLE_PLAIN, 0u, 0u, 0u};
        check(wrs_alias_sample(a_.deviceTable(), a_.N, numSamples, seed_, counter, &o, d_out, nullptr, a_.stream()),
              "plain sample");
        counter += numSamples;
    }
    // counted on the device (the histogram mode), without a sample list
    std::vector<int64_t> getSamplingDistribution(uint64_t numSamples) override {
        DeviceArray<uint32_t> counts((size_t)a_.N);
        check_cuda(cudaMemsetAsync(counts.get(), 0, counts.bytes(), a_.stream()), "cudaMemsetAsync");
        wrs_sample_opts o{WRS_SAMPLE_HISTOGRAM, 0u, 0u, 0u};
        check(wrs_alias_sample(a_.deviceTable(), a_.N, numSamples, seed_, counter, &o, counts.get(), nullptr,
                               a_.stream()), "plain histogram");
        counter += numSamples;
        const std::vector<uint32_t> h = counts.to_host(a_.stream());
        return std::vector<int64_t>(h.begin(), h.end());
    }

protected:
    cudaStream_t stream() const override { return a_.stream(); }
    int64_t items() const override { return a_.N; }
    AliasTableSplitGpu& a_;
};

class SamplerGpuSectioned : public Sampler {
public:
    explicit SamplerGpuSectioned(AliasTableSplitGpu& a, uint32_t itemsPerSection = 0, uint64_t seed = 0x5EED)
        : Sampler(seed), a_(a), section_(itemsPerSection) {}
    std::string name() override { return "SamplerGpuSectioned"; }
    void sample(uint64_t numSamples, uint32_t* d_out) override {
        wrs_sample_opts o{WRS_SAMPLE_SECTIONED, section_, 0u, 0u};
        check(wrs_alias_sample(a_.deviceTable(), a_.N, numSamples, seed_, counter, &o, d_out, nullptr, a_.stream()),
              "sectioned sample");
        counter += numSamples;
    }

protected:
    cudaStream_t stream() const override { return a_.stream(); }
    int64_t items() const override { return a_.N; }
    AliasTableSplitGpu& a_;
    uint32_t section_;
};

// SamplerGpuSectionedShared (sampling/aliasTable/SamplerGpuSectionedShared.cu:3-111): each section is
// staged in shared memory before it is sampled. wrs_alias_sample stages every section of at most
// 12,288 rows (96 KiB), so this is the sectioned sampler with the reference's default of 3000 rows
// per section; a section too large to stage is an error, as the reference asserts.
class SamplerGpuSectionedShared : public SamplerGpuSectioned {
public:
    static constexpr uint32_t kMaxStagedRows = 12288;
    explicit SamplerGpuSectionedShared(AliasTableSplitGpu& a, uint32_t itemsPerSection = 3000, uint64_t seed = 0x5EED)
        : SamplerGpuSectioned(a, itemsPerSection, seed) {
        if (itemsPerSection < 2 || itemsPerSection > kMaxStagedRows || (itemsPerSection & 1u))
            throw Error(WRS_ERR_INVALID_ARGUMENT, "SamplerGpuSectionedShared: itemsPerSection must be even, in [2, 12288]");
    }
    std::string name() override { return "SamplerGpuSectionedShared"; }
};

class SamplerRejection : public Sampler {
public:
    explicit SamplerRejection(RejectionSamplingGpu& r, uint64_t seed = 0x5EED, uint32_t maxTries = 0)
        : Sampler(seed), r_(r), tries_(maxTries) {}
    std::string name() override { return "SamplerRejection"; }
    void sample(uint64_t numSamples, uint32_t* d_out) override {
        check(wrs_rejection_sample_packed(r_.devicePacked(), r_.packedCapacity(), r_.deviceASize(), r_.N, numSamples,
                                          seed_, counter, tries_, d_out, nullptr, 0u, r_.stream()),
              "rejection sample");
        counter += numSamples;
    }

protected:
    cudaStream_t stream() const override { return r_.stream(); }
    int64_t items() const override { return r_.N; }
    RejectionSamplingGpu& r_;
    uint32_t tries_;
};

// SamplerRejectionGiveUp (sampling/rejectionSampling/SamplerRejectionGiveUp.cu:17-37,
// MAX_TRIES 8 in SamplerRejectionGiveUp.cuh): at most 8 tries per sample; a sample that runs
// out of tries is written as 0xFFFFFFFF (the reference gives up on it the same way).
class SamplerRejectionGiveUp : public SamplerRejection {
public:
    explicit SamplerRejectionGiveUp(RejectionSamplingGpu& r, uint64_t seed = 0x5EED) : SamplerRejection(r, seed, 8u) {}
    std::string name() override { return "SamplerRejectionGiveUp"; }
};

// ---------------------------------------------------------------- batches

// Many alias tables at once (CSR offsets into one weight array): the batched form of
// AliasTableSplitGpu (the reference builds one object per table). autotune() picks the
// launch shape on this batch; the table's rows land at their items with table-local aliases.
class BatchedAliasTablesGpu {
public:
    BatchedAliasTablesGpu(std::vector<float> w, std::vector<int64_t> offsets, cudaStream_t stream = nullptr)
        : weights(std::move(w)), offsets(std::move(offsets)), stream_(stream) {
        opts_.method = WRS_METHOD_SPLIT;
        opts_.tile_items = 0;
        opts_.flags = 0;
        opts_.small_table_items = 0;
    }
    std::string name() { return "BatchedAliasTablesGpu"; }
    int64_t numTables() const { return (int64_t)offsets.size() - 1; }
    void preBuild() {
        w_dev_.resize(weights.size());
        if (!weights.empty())
            check_cuda(cudaMemcpyAsync(w_dev_.get(), weights.data(), w_dev_.bytes(), cudaMemcpyHostToDevice, stream_),
                       "weights upload");
        off_dev_.resize(offsets.size());
        check_cuda(cudaMemcpyAsync(off_dev_.get(), offsets.data(), off_dev_.bytes(), cudaMemcpyHostToDevice, stream_),
                   "offsets upload");
        table_.resize(weights.empty() ? 1 : weights.size());
        W_dev_.resize((size_t)numTables());
        scratch_.resize(wrs_batched_build_scratch_bytes(offsets.data(), numTables(), nullptr));
    }
    void autotune() {
        check(wrs_batched_autotune(w_dev_.get(), off_dev_.get(), offsets.data(), numTables(), table_.get(),
                                   scratch_.get(), scratch_.bytes(), &opts_, stream_), "batched autotune");
    }
    void build() {
        check(wrs_batched_build_f32(w_dev_.get(), off_dev_.get(), offsets.data(), numTables(), &opts_, table_.get(),
                                    W_dev_.get(), scratch_.get(), scratch_.bytes(), stream_), "batched build");
    }
    bool postBuild() {
        check(wrs_scratch_status(scratch_.get(), stream_), "batched build (device)");
        W = W_dev_.to_host(stream_);
        return true;
    }
    bool fullBuild() {
        preBuild();
        build();
        return postBuild();
    }
    const wrs_alias_row* deviceTable() const { return table_.get(); }
    const int64_t* deviceOffsets() const { return off_dev_.get(); }
    std::vector<wrs_alias_row> hostTable() const { return table_.to_host(stream_); }
    cudaStream_t stream() const { return stream_; }

    std::vector<float> weights;
    std::vector<int64_t> offsets;
    std::vector<double> W;  // per-table weight totals

private:
    cudaStream_t stream_;
    wrs_build_opts opts_{};
    DeviceArray<float> w_dev_;
    DeviceArray<int64_t> off_dev_;
    DeviceArray<wrs_alias_row> table_;
    DeviceArray<double> W_dev_;
    DeviceArray<unsigned char> scratch_;
};

// Per-table sample counts over a batch: table t's table-local samples at
// [sampleOffsets[t], sampleOffsets[t + 1]) of the output.
class SamplerBatched {
public:
    explicit SamplerBatched(BatchedAliasTablesGpu& b, uint64_t seed = 0x5EED) : b_(b), seed_(seed) {}
    std::string name() { return "SamplerBatched"; }
    // counts (host, one per table) -> samples (host); sampleOffsets receives the CSR offsets
    std::vector<uint32_t> sample(const std::vector<int64_t>& counts, std::vector<int64_t>* sampleOffsets = nullptr) {
        std::vector<int64_t> soff(counts.size() + 1, 0);
        for (size_t t = 0; t < counts.size(); ++t) soff[t + 1] = soff[t] + counts[t];
        const uint64_t total = (uint64_t)soff.back();
        DeviceArray<int64_t> d_soff(soff.size());
        check_cuda(cudaMemcpyAsync(d_soff.get(), soff.data(), d_soff.bytes(), cudaMemcpyHostToDevice, b_.stream()),
                   "sample offsets upload");
        DeviceArray<uint32_t> out(total ? total : 1);
        check(wrs_batched_sample(b_.deviceTable(), b_.deviceOffsets(), b_.numTables(), d_soff.get(), total, seed_,
                                 counter, out.get(), b_.stream()), "batched sample");
        counter += total;
        std::vector<uint32_t> h = out.to_host(b_.stream());
        h.resize(total);
        if (sampleOffsets) *sampleOffsets = soff;
        return h;
    }
    uint64_t counter = 0;

private:
    BatchedAliasTablesGpu& b_;
    uint64_t seed_;
};

}  // namespace wrs

#endif /* WRS_HPP */
