/*
 * wrs_oracle.h — CPU oracle of the weighted-random-sampling hot path.
 *
 * TEST INFRASTRUCTURE ONLY. The library never links, loads or calls anything here; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm use it, and only as the
 * checker or the timed CPU reference — never as the thing measured on the GPU.
 *
 * Contents (each function cites the reference file:line it restates):
 *   - or_sweep_build / or_split_build: the reference's sequential CPU alias builds in FP64
 *     (AliasTableSweep::build, AliasTableSplit::build + PackMethodSweep::pack);
 *   - or_check_table / or_check_ref_table: per-item probability reconstruction against
 *     w_i / W with W summed exactly (AliasTable::verifyTableCorrectness, tightened to a
 *     relative per-item error);
 *   - or_exact_build: a sequential restatement of the library's exact merge build (bit-exact
 *     reference for the GPU tables);
 *   - or_philox4x32_10 / or_sample_plain / or_sample_sectioned: the sampling-input contract
 *     and the reference's doSample decision (SamplerGpuBasic.cu:28-69);
 *   - or_rejection_build / or_rejection_sample: RejectionSampling::build + fillA and
 *     SamplerRejection::sample;
 *   - or_binomial / or_section_counts: the sectioned sampler's binomial tree.
 */
#ifndef WRS_ORACLE_H
#define WRS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* exact (correctly rounded) sum of FP32 weights (Shewchuk expansion, as math.fsum) */
double or_exact_sum_f32(const float* w, int64_t n);

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* reference-format tables: weight (absolute, FP64) + alias (int32) */
int or_sweep_build(const double* w, int64_t n, double* weight, int32_t* alias, double* W_out);
/* the same sweep with every quantity in FP32; W_out gets the FP32 total */
int or_sweep_build_f32(const float* w, int64_t n, double* weight, int32_t* alias, double* W_out);
int or_split_build(const double* w, int64_t n, int64_t p, double* weight, int32_t* alias, double* W_out,
                   int threads);

/* per-item check of a {f32 prob, u32 alias} table (rows interleaved: prob bits, alias).
 * stats[0] = max relative error over items with w > 0, stats[1] = p99.99 relative error,
 * stats[2] = index of the worst item, stats[3] = number of zero-weight items that got mass,
 * stats[4] = number of rows with prob outside [0, 1] or alias >= n. W_used = the sum. */
int or_check_table(const float* w, int64_t n, const uint32_t* rows, double* stats, double* W_used);
/* same for a reference-format table, prob = weight / (W/N), alias ignored when weight >= W/N */
int or_check_ref_table(const double* w, int64_t n, const double* weight, const int32_t* alias, double W,
                       double* stats);
/* a reference-format table on its own scale W_N_table, against n w_i / W_exact */
int or_check_ref_table_w(const float* w, int64_t n, const double* weight, const int32_t* alias, double W_N_table,
                         double W_exact, double* stats);

/* the library's exact merge build, sequentially; W = the weight total the build uses */
int or_exact_build(const float* w, int64_t n, double W, uint32_t* rows);
/* The library's all-FP64 (fp64 = 1) or all-FP32 (fp64 = 0) comparison build
 * (precision_kernels.cuh), bit-exact; returns 1 for invalid weights or a zero total. */
int or_prec_build(const float* w, int64_t n, int fp64, uint32_t* rows, double* W_out);

/* sampling contract */
void or_sample_plain(const uint32_t* rows, int64_t n, uint64_t m, uint64_t seed, uint64_t cbase, uint32_t* out);
void or_plain_replay_uniforms(int64_t n, uint64_t m, uint64_t seed, uint64_t cbase, double* u, uint32_t* rows_out,
                              float* coins_out);
uint64_t or_binomial(uint64_t n, double p, uint32_t k0, uint32_t k1, uint64_t cbase, uint32_t node);
void or_section_counts(int64_t n, uint32_t S, uint64_t m, uint64_t seed, uint64_t cbase, uint64_t* counts);
void or_sample_sectioned(const uint32_t* rows, int64_t n, uint64_t m, uint32_t S, uint64_t seed, uint64_t cbase,
                         uint32_t* out, uint64_t* counts);

/* PSA+: tile-local pre-pack over tiles of T items, then the exact merge of the leftovers */
int or_psa_plus_build(const float* w, int64_t n, double W, int64_t T, uint32_t* rows);

/* batched (CSR): table t owns items [off[t], off[t+1]); its rows (table-local aliases) are
 * or_exact_build of its weights with W = their exact sum (empty tables: no rows). W_out
 * (optional) gets the totals. Returns the number of tables with a zero or invalid total
 * (left unwritten). */
int or_batched_build(const float* w, const int64_t* off, int64_t num_tables, uint32_t* rows, double* W_out);
/* output position s of the batch belongs to table t with soff[t] <= s < soff[t+1] and follows
 * the plain contract over the global position s (table-local rows) */
void or_batched_sample(const uint32_t* rows, const int64_t* off, int64_t num_tables, const int64_t* soff,
                       uint64_t seed, uint64_t cbase, uint32_t* out);

/* rejection: A holds item | 0x80000000 on first slots; returns |A| (or 0 on capacity error) */
uint64_t or_rejection_build(const float* w, int64_t n, double W, uint32_t* A, uint64_t a_capacity, float* frac);
int or_rejection_sample(const uint32_t* A, uint64_t a_size, const float* frac, uint64_t m, uint64_t seed,
                        uint64_t cbase, uint32_t max_tries, uint32_t* out);
/* mixed batch (kinds: 0 alias, 1 rejection, else skipped); rejection slots at A + 2 off[t] */
int or_batched_mixed_build(const float* w, const int64_t* off, int64_t num_tables, const uint8_t* kinds,
                           uint32_t* rows, uint32_t* A, float* frac, uint64_t* a_size, double* W_out);
int or_batched_mixed_sample(const uint32_t* rows, const uint32_t* A, const float* frac, const uint64_t* a_size,
                            const int64_t* off, int64_t num_tables, const uint8_t* kinds, const int64_t* soff,
                            uint64_t seed, uint64_t cbase, uint32_t max_tries, uint32_t* out);

/* reference CPU sampler restatement with the Philox contract, all cores; returns samples/s */
double or_sample_plain_timed(const uint32_t* rows, int64_t n, uint64_t m, uint64_t seed, int threads,
                             uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif
