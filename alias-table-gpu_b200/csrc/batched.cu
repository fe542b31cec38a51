// batched.cu — C ABI of the batched (CSR) alias build and sampler.
#include <cuda_runtime.h>

#include "host_util.h"

extern "C" size_t wrs_batched_build_scratch_bytes(const int64_t* h_offsets, int64_t num_tables,
                                                  const wrs_build_opts* opts) {
    (void)h_offsets;
    (void)num_tables;
    (void)opts;
    return 0;
}

extern "C" wrs_status wrs_batched_build_f32(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                            int64_t num_tables, const wrs_build_opts* opts, wrs_alias_row* d_table,
                                            double* d_W, void* d_scratch, size_t scratch_bytes, void* stream) {
    (void)d_w; (void)d_offsets; (void)h_offsets; (void)num_tables; (void)opts; (void)d_table; (void)d_W;
    (void)d_scratch; (void)scratch_bytes; (void)stream;
    return WRS_ERR_UNSUPPORTED;
}

extern "C" wrs_status wrs_batched_sample(const wrs_alias_row* d_table, const int64_t* d_offsets, int64_t num_tables,
                                         const int64_t* d_sample_offsets, uint64_t total_samples, uint64_t seed,
                                         uint64_t counter_base, uint32_t* d_out, void* stream) {
    (void)d_table; (void)d_offsets; (void)num_tables; (void)d_sample_offsets; (void)total_samples; (void)seed;
    (void)counter_base; (void)d_out; (void)stream;
    return WRS_ERR_UNSUPPORTED;
}
