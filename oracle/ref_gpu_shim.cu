/*
 * ref_gpu_shim.cu — C entry points over the reference's own GPU code (sm_100a), compiled
 * together with the reference sources read in place from the reference checkout (see
 * oracle/Makefile, target `ref`; nothing of the reference is copied into this repository).
 *
 * TEST INFRASTRUCTURE ONLY: the GPU parity tests feed this library's tables, weights and
 * Philox-derived uniforms to the reference's own device code and compare its answers with
 * the library's. The library never links or calls it.
 *
 *  - ref_gpu_do_sample_{aos,soa}: the reference's sampling decision, doSample<TableStorage>
 *    (sampling/aliasTable/SamplerGpuBasic.cu:28-69), one call per given uniform. The
 *    reference's samplers draw u from cuRAND; a replay of u = (row + coin) / n in FP64 gives
 *    u * n = row + coin exactly for power-of-two n <= 2^29, so the reference decides on the
 *    same (row, coin) pair as the library's Philox contract.
 *  - ref_gpu_rejection_build: RejectionSampling::build's slot-count scan
 *    (construction/rejectionSampling/RejectionSampling.cu:26-56: CalcNumOccurrencesOperator
 *    through cub::DeviceScan::InclusiveSum) and fillABinarySearch
 *    (RejectionSamplingBinarySearch.cu:12-37), with the weight total W given by the caller
 *    (the reference's build() sums it on the host first, SamplingAlgorithm.cu:14-19).
 *  - ref_gpu_sample_timed: the reference's plain GPU sampling as its benchmark kernel draws it
 *    (sampleBenchmarkBasic, SamplerGpuBasic.cu:77-101): a curand XORWOW generator per thread
 *    (XorWowPrng, utils/Prng.cuh:58-94, seeded with a fixed seed and the thread number) and
 *    doSample<ArrayOfStructs> on the reference's 16-byte rows, in a harness loop of a fixed
 *    trip count. The benchmark kernel itself is not run: its closing `while (dummy == 0)` loop
 *    never ends in a thread that drew no sample once the asserts are compiled out.
 *  - ref_gpu_rejection_fraction: the first-slot acceptance expression of
 *    SamplerRejection::sample (sampling/rejectionSampling/SamplerRejection.cu:27), with the
 *    reference's own fracf, for every item; the sampler itself (an unbounded retry loop) is
 *    never run.
 *
 * Every entry point checks its sizes on the host before a launch (the reference's device
 * asserts are compiled out), returns 0 on success and a CUDA error code otherwise, and
 * synchronises before returning.
 */
#include <cstdint>

#include "construction/rejectionSampling/RejectionSampling.cu"
#include "construction/rejectionSampling/RejectionSamplingBinarySearch.cu"
#include "sampling/aliasTable/SamplerGpuBasic.cu"
#include "sampling/rejectionSampling/SamplerRejection.cu"

namespace {

template <typename TableStorage>
__global__ void replay_do_sample(TableStorage table, double W_N, int N, const double* __restrict__ u,
                                 int* __restrict__ out, int m) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = doSample<TableStorage>(table, W_N, N, u[i]);
}

__global__ void fill_aos(ArrayOfStructs table, const double* __restrict__ weight, const int* __restrict__ alias,
                         int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        ArrayOfStructs::TableRow r;
        r.weight = weight[i];
        r.alias = alias[i];
        table.setBoth(i, r);
    }
}

__global__ void rejection_fraction(const double* __restrict__ weights, int N, double W, float* __restrict__ out,
                                   int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        // SamplerRejection.cu:26-27, as written there: the FP64 weight read into a float,
        // N * weight formed in FP32, divided by W in FP64, and fracf in FP32.
        float weight = weights[i];
        out[i] = fracf((double)(N * weight) / (double)W);
    }
}

int blocks_for(int count, int threads) { return count / threads + 1; }

__global__ void harness_sample(ArrayOfStructs table, int N, double W_N, long long per_thread,
                               unsigned long long seed, unsigned int* sink) {
    XorWowPrng random;
    random.initGpu(blockIdx.x * blockDim.x + threadIdx.x, (long)seed);
    unsigned int acc = 0;
    for (long long i = 0; i < per_thread; ++i)
        acc ^= (unsigned int)doSample<ArrayOfStructs>(table, W_N, N, random.next());
    atomicXor(sink, acc);
}

}  // namespace

extern "C" {

/* doSample<ArrayOfStructs> over a table given as device arrays (weight = absolute row weight,
 * alias), rows packed into the reference's 16-byte AoS rows first. */
int ref_gpu_do_sample_aos(const double* d_weight, const int* d_alias, int n, double W_N, const double* d_u,
                          int* d_out, int m) {
    if (n < 1 || m < 0) return (int)cudaErrorInvalidValue;
    ArrayOfStructs table(DEVICE);
    table.malloc((size_t)n);
    fill_aos<<<blocks_for(n, 256), 256>>>(table, d_weight, d_alias, n);
    if (m > 0) replay_do_sample<ArrayOfStructs><<<blocks_for(m, 256), 256>>>(table, W_N, n, d_u, d_out, m);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    table.free();
    return (int)e;
}

/* The reference's plain GPU sampling (see above) of blocks x threads x per_thread samples on a
 * table given as device arrays (absolute row weight, alias; packed into its 16-byte AoS rows
 * first), timed with CUDA events around the sampling kernel alone (generator set-up included, as
 * in the reference's benchmark). *ms gets the time, *checksum the XOR of all samples. */
int ref_gpu_sample_timed(const double* d_weight, const int* d_alias, int n, double W_N, int blocks, int threads,
                         long long per_thread, unsigned long long seed, float* ms, unsigned int* checksum) {
    if (n < 1 || blocks < 1 || threads < 1 || threads > 1024 || per_thread < 0 || !ms || !checksum)
        return (int)cudaErrorInvalidValue;
    ArrayOfStructs table(DEVICE);
    table.malloc((size_t)n);
    fill_aos<<<blocks_for(n, 256), 256>>>(table, d_weight, d_alias, n);
    unsigned int* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(sink, 0, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        cudaEventRecord(e0);
        harness_sample<<<blocks, threads>>>(table, n, W_N, per_thread, seed, sink);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    if (e == cudaSuccess) e = cudaMemcpy(checksum, sink, sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (sink) cudaFree(sink);
    table.free();
    return (int)e;
}

/* doSample<StructOfArrays> over the caller's device arrays (no copy). */
int ref_gpu_do_sample_soa(double* d_weight, int* d_alias, int n, double W_N, const double* d_u, int* d_out, int m) {
    if (n < 1 || m < 0) return (int)cudaErrorInvalidValue;
    StructOfArrays table(DEVICE);
    table.weights.usePreInitialized(d_weight, n);
    table.aliases.usePreInitialized(d_alias, n);
    table.size = n;
    if (m > 0) replay_do_sample<StructOfArrays><<<blocks_for(m, 256), 256>>>(table, W_N, n, d_u, d_out, m);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return (int)e;
}

/* RejectionSampling::build's scan (CalcNumOccurrencesOperator, cub InclusiveSum) and
 * fillABinarySearch, with the given W. *a_size receives |A|; d_A (a_capacity ints) receives
 * A when |A| <= a_capacity (else nothing is filled and the return value is
 * cudaErrorInvalidValue with *a_size set). */
int ref_gpu_rejection_build(double* d_w, int n, double W, int* d_A, long long a_capacity, long long* a_size) {
    if (n < 1 || !(W > 0.0)) return (int)cudaErrorInvalidValue;
    SafeArray<double> weights(DEVICE);
    weights.usePreInitialized(d_w, n);
    SafeArray<int> elementsPerItem(DEVICE);
    elementsPerItem.malloc((size_t)n);

    CalcNumOccurrencesOperator op = {};
    op.N = n;
    op.W = W;
    cub::TransformInputIterator<int, CalcNumOccurrencesOperator, double*> it(weights.data, op);
    void* temp = nullptr;
    size_t temp_bytes = 0;
    cudaError_t e = cub::DeviceScan::InclusiveSum(temp, temp_bytes, it, elementsPerItem.data, elementsPerItem.size);
    if (e == cudaSuccess) e = cudaMalloc(&temp, temp_bytes);
    if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(temp, temp_bytes, it, elementsPerItem.data, elementsPerItem.size);
    int total = 0;
    if (e == cudaSuccess)
        e = cudaMemcpy(&total, &elementsPerItem.data[elementsPerItem.size - 1], sizeof(int), cudaMemcpyDeviceToHost);
    if (temp) cudaFree(temp);
    if (e != cudaSuccess) {
        elementsPerItem.free();
        return (int)e;
    }
    *a_size = total;
    if (total < 1 || (long long)total > a_capacity) {
        elementsPerItem.free();
        return (int)cudaErrorInvalidValue;
    }
    SafeArray<int> A(DEVICE);
    A.usePreInitialized(d_A, total);
    fillABinarySearch<<<dim3(A.size / REJECTION_THREADS_PER_BLOCK + 1), dim3(REJECTION_THREADS_PER_BLOCK)>>>(
        A, elementsPerItem);
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    elementsPerItem.free();
    return (int)e;
}

/* fracf((double)(N * weight) / W) of SamplerRejection.cu:27 for every item. */
int ref_gpu_rejection_fraction(const double* d_w, int n, double W, float* d_out) {
    if (n < 1) return (int)cudaErrorInvalidValue;
    rejection_fraction<<<blocks_for(n, 256), 256>>>(d_w, n, W, d_out, n);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return (int)e;
}

}  // extern "C"
