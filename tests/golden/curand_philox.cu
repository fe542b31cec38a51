// Prints cuRAND Philox4_32_10 outputs (curand_init + curand4) as JSON lines, to pin the
// oracle's Philox4x32-10 against an independent implementation. Built and run by
// tests/golden/make_philox_golden.py on a CUDA machine.
#include <cstdio>
#include <curand_kernel.h>

__global__ void draw(unsigned long long seed, unsigned long long subseq, unsigned long long offset, uint4* out, int k) {
    curandStatePhilox4_32_10_t st;
    curand_init(seed, subseq, offset, &st);
    for (int i = 0; i < k; ++i) out[i] = curand4(&st);
}

int main() {
    const unsigned long long cases[][3] = {{0ull, 0ull, 0ull}, {0x5EEDull, 0ull, 0ull},
                                           {0x123456789abcdef0ull, 7ull, 0ull}, {42ull, 0ull, 8ull},
                                           {42ull, 1ull << 40, 4ull * 1000003ull}, {0xffffffffffffffffull, 3ull, 0ull}};
    const int k = 3;
    uint4* d;
    cudaMalloc(&d, sizeof(uint4) * k);
    uint4 h[k];
    for (const auto& c : cases) {
        draw<<<1, 1>>>(c[0], c[1], c[2], d, k);
        cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
        printf("{\"seed\": %llu, \"subsequence\": %llu, \"offset\": %llu, \"outputs\": [", c[0], c[1], c[2]);
        for (int i = 0; i < k; ++i)
            printf("%s[%u, %u, %u, %u]", i ? ", " : "", h[i].x, h[i].y, h[i].z, h[i].w);
        printf("]}\n");
    }
    cudaFree(d);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
