/*
 * wrs.h — C ABI of the B200 (sm_100a) weighted-random-sampling library.
 *
 * The library builds alias tables and rejection-sampling structures from FP32
 * weights that already live in device memory, and draws samples from them with
 * a counter-based Philox4x32-10 stream. Every entry point is stream-ordered,
 * allocates no device memory itself (the caller passes a scratch buffer sized by
 * the matching *_scratch_bytes query), never traps, and returns a wrs_status.
 *
 * Errors found on the device while a launch runs (an invalid weight, a bounded
 * device wait that gave up, a rejection sample that ran out of tries) are
 * written into a status word inside the scratch buffer (or the sampler's
 * d_status argument) and read back with wrs_scratch_status(); passing
 * WRS_FLAG_SYNC in the options makes the call itself synchronise and return it.
 *
 * Each entry point replaces one interface of ByteHamster/alias-table-gpu:
 *   wrs_alias_build_f32   <- AliasTableSplitGpu<TableStorage>::build()
 *                            (construction/aliasTable/buildMethod/AliasTableSplitGpu.cu:388-468),
 *                            with psaPlus() (:342-386) selected by WRS_METHOD_PSA_PLUS
 *   wrs_alias_sample      <- SamplerGpuBasic::executeBenchmarkSampling
 *                            (sampling/aliasTable/SamplerGpuBasic.cu:109-133) and
 *                            SamplerGpuSectioned[Shared]::executeBenchmarkSampling
 *                            (sampling/aliasTable/SamplerGpuSectioned.cu:138-166,
 *                             SamplerGpuSectionedShared.cu:90-111)
 *   wrs_rejection_build_f32 <- RejectionSampling::build() + fillA()
 *                            (construction/rejectionSampling/RejectionSampling.cu:35-56,
 *                             RejectionSamplingBinarySearch.cu:12-37)
 *   wrs_rejection_sample  <- SamplerRejection / SamplerRejectionGiveUp
 *                            (sampling/rejectionSampling/SamplerRejection.cu:17-72,
 *                             SamplerRejectionGiveUp.cu:17-79)
 *   wrs_batched_*         <- a loop of AliasTableSplitGpu objects (one per table) in the
 *                            reference's experiment drivers; the reference has no batched form
 *                            (and no autotuner: its launch shapes are compile-time constants,
 *                            AliasTableSplitGpu.cuh:60-94)
 *   wrs_sum_f32           <- Adder::addGpuCub (utils/Adder.cu:144-157)
 */
#ifndef WRS_H
#define WRS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define WRS_API __attribute__((visibility("default")))
#else
#define WRS_API
#endif

#define WRS_VERSION_MAJOR 0
#define WRS_VERSION_MINOR 2

typedef enum wrs_status {
    WRS_SUCCESS = 0,
    WRS_ERR_INVALID_ARGUMENT = 1,  /* null pointer, size out of range, unknown option */
    WRS_ERR_INVALID_WEIGHT = 2,    /* a weight is NaN, negative or infinite */
    WRS_ERR_ZERO_TOTAL = 3,        /* all weights are zero: no distribution */
    WRS_ERR_SCRATCH_TOO_SMALL = 4, /* scratch_bytes below the *_scratch_bytes query */
    WRS_ERR_CUDA = 5,              /* a CUDA runtime call failed */
    WRS_ERR_DEVICE_TIMEOUT = 6,    /* a bounded device-side wait gave up */
    WRS_ERR_TOO_MANY_TRIES = 7,    /* a rejection sample exhausted max_tries */
    WRS_ERR_UNSUPPORTED = 8,       /* the device is not an sm_100 part */
    WRS_ERR_CAPACITY = 9           /* an output buffer is too small (rejection array) */
} wrs_status;

/* One alias-table row: the row keeps itself with probability `prob`, else
 * yields `alias`. Item i's probability is
 *   (prob_i + sum_{r : alias_r = i, r != i} (1 - prob_r)) / n.
 * The reference stores {double weight (absolute, in [0, W/N]); int alias}
 * (construction/aliasTable/TableStorage.cuh:8-11); prob = weight / (W/N). */
typedef struct wrs_alias_row {
    float prob;
    uint32_t alias;
} wrs_alias_row;

typedef enum wrs_build_method {
    WRS_METHOD_SPLIT = 0,     /* split/pack over light/heavy residual prefix sums ("PSA") */
    WRS_METHOD_PSA_PLUS = 1   /* tile-local pre-pack, leftovers through split/pack (more scratch:
                                 query wrs_alias_build_scratch_bytes with the method set) */
} wrs_build_method;

#define WRS_FLAG_SYNC 1u      /* synchronise the stream and return the device status */

/* Arithmetic of the split build's deficit and excess lines. MIXED (the default) keeps them in
 * exact fixed point with a compensated weight total, and only the stored probabilities in
 * FP32: per-item probability error about 2^-23. FP64 and FP32 are comparison builds that run
 * the same merge with every quantity (weight total, W/N, deficits, excesses and their prefix
 * sums) rounded to that type at each operation, as the reference's build does in FP64
 * (AliasTableSplitGpu.cu:406-432); their error grows with n and the weights' spread. */
typedef enum wrs_precision {
    WRS_PRECISION_MIXED = 0,
    WRS_PRECISION_FP64 = 1,
    WRS_PRECISION_FP32 = 2
} wrs_precision;

typedef struct wrs_build_opts {
    uint32_t method;            /* wrs_build_method */
    uint32_t tile_items;        /* 0 = default (2048; 1024 for PSA+); 1024, 2048 or 4096 */
    uint32_t flags;             /* WRS_FLAG_* */
    uint32_t small_table_items; /* batched builds: tables of at most this many items are built
                                   one per warp (0 = default 128; 32, 64, 128, 256 or 512) */
    uint32_t precision;         /* wrs_precision (single-table split builds only; 0 = MIXED) */
} wrs_build_opts;

typedef enum wrs_sample_mode {
    WRS_SAMPLE_PLAIN = 0,     /* sample s at output position s, any row */
    WRS_SAMPLE_SECTIONED = 1, /* rows cut into sections; per-section counts from an exact
                                 binomial tree; output grouped by section */
    WRS_SAMPLE_HISTOGRAM = 2, /* the PLAIN samples counted instead of written: d_out holds n u32
                                 counters that the call adds to (the caller zeroes them); the
                                 reference's samplers write no samples, and its
                                 getSamplingDistribution returns these counts */
    WRS_SAMPLE_DISCARD = 3    /* the PLAIN samples drawn and folded into d_out[0] ^= (the XOR of
                                 all of them): the like-for-like timing of the reference's
                                 samplers, which keep nothing (SamplerGpuBasic.cu:77-107) */
} wrs_sample_mode;

typedef struct wrs_sample_opts {
    uint32_t mode;            /* wrs_sample_mode */
    uint32_t section_items;   /* SECTIONED: rows per section (0 = 65536) */
    uint32_t flags;           /* WRS_FLAG_* */
    uint32_t threads;         /* 0 = default launch shape */
} wrs_sample_opts;

/* ---- weight total ------------------------------------------------------- */

/* Compensated (double-double) sum of n FP32 weights. Writes the correctly rounded
 * total to *d_total (device). Rejects NaN / negative / infinite weights. */
WRS_API size_t     wrs_sum_scratch_bytes(int64_t n);
WRS_API wrs_status wrs_sum_f32(const float* d_w, int64_t n, double* d_total,
                       void* d_scratch, size_t scratch_bytes, void* stream);

/* ---- alias tables ------------------------------------------------------- */

WRS_API size_t     wrs_alias_build_scratch_bytes(int64_t n, const wrs_build_opts* opts);
/* Builds an n-row table in d_table from n FP32 weights d_w (1 <= n <= 2^31-1).
 * d_W (optional, device) receives the weight total used. opts may be NULL. */
WRS_API wrs_status wrs_alias_build_f32(const float* d_w, int64_t n, const wrs_build_opts* opts,
                               wrs_alias_row* d_table, double* d_W,
                               void* d_scratch, size_t scratch_bytes, void* stream);

/* The same build for callers that cannot allocate device memory (code under an allocator
 * that forbids cudaMalloc, plugins that must not touch the host process's memory pools,
 * paths that may not block on an allocation). No counterpart in the reference. Its scratch
 * is a fixed 8 MiB device array inside this library, so it takes n <= 262,144 (2^18) items
 * (about 190,000 with WRS_METHOD_PSA_PLUS, which needs more scratch) and rejects larger n
 * with WRS_ERR_INVALID_ARGUMENT. It calls no allocating routine itself, but the driver
 * reserves the array on a device when it loads this library's device code there: with lazy
 * module loading (the CUDA default) that is the first call of any wrs_* entry point on that
 * device, so make one warm-up call (or set CUDA_MODULE_LOADING=EAGER) before entering a
 * region that must not allocate or a stream capture. The array stays reserved on every GPU
 * that loaded it until the process exits. The first call on each device (and the first after
 * a device reset, which makes a new context) looks up the array's device address. All calls
 * on a device share the array, so calls that overlap on the GPU race: serialise them.
 * Device-side errors are returned when opts->flags has WRS_FLAG_SYNC; without it,
 * wrs_static_scratch_status reads them afterwards. */
WRS_API wrs_status wrs_alias_build_f32_static_scratch(const float* d_w, int64_t n, const wrs_build_opts* opts,
                                                      wrs_alias_row* d_table, double* d_W, void* stream);
/* Reads (synchronising `stream`) the device status word of the current device's static
 * scratch array: the status of the last wrs_alias_build_f32_static_scratch call on this
 * device, valid until the next such call. No counterpart in the reference. */
WRS_API wrs_status wrs_static_scratch_status(void* stream);

/* Sampling-input contract (bit-exact, see the oracle):
 *   output position s uses Philox4x32-10 with key (lo32(seed), hi32(seed)) and counter
 *   (lo32(b), hi32(b), 0, 0), b = counter_base + s, giving words x0..x3.
 *   row = floor(u * len / 2^64) + offset for the 64-bit uniform u = x1 * 2^32 + x0 (PLAIN:
 *   len = n, offset = 0; SECTIONED: the section of s), coin = (x2 >> 8) * 2^-24,
 *   result = coin < prob[row] ? row : alias[row]. x3 is unused.
 *   Every row's share of the 2^64 values of u is within len / 2^64 (relative) of 1 / len.
 * SECTIONED derives the per-section counts from a binomial tree keyed by the same
 * (seed, counter_base). d_section_counts (optional, device, ceil(n/section_items) u64)
 * receives them. */
WRS_API wrs_status wrs_alias_sample(const wrs_alias_row* d_table, int64_t n, uint64_t num_samples,
                            uint64_t seed, uint64_t counter_base, const wrs_sample_opts* opts,
                            uint32_t* d_out, uint64_t* d_section_counts, void* stream);
/* Plain sampling with the samples delivered to host memory: the samples of wrs_alias_sample
 * (PLAIN, same seed and counter_base) are produced chunk by chunk into d_out on `stream`, and
 * an internal copy stream of the library moves each finished chunk to h_out (num_samples u32;
 * pinned host memory, or the copies do not overlap), so the transfer overlaps the sampling
 * of the next chunk. Work enqueued on `stream` after the call waits for every copy.
 * chunk_samples: 0 = 2^25. The copy stream is created on the
 * first call on a device: make that call outside stream capture. The reference's samplers
 * keep no output (SamplerGpuBasic.cu:77-133); this is the transfer a caller of its
 * getSamplingDistribution pays for, overlapped. */
WRS_API wrs_status wrs_alias_sample_to_host(const wrs_alias_row* d_table, int64_t n, uint64_t num_samples,
                                            uint64_t seed, uint64_t counter_base, uint64_t chunk_samples,
                                            uint32_t* d_out, uint32_t* h_out, void* stream);

/* Diagnostic: num_gathers random 8-byte row gathers from the table (rows from an integer hash
 * of seed and position; the plain sampler's load form, eight in flight per thread), XOR-folded
 * into *d_sink (device u32). Its rate is the random-access ceiling of the plain sampler on that
 * table. No counterpart in the reference. */
WRS_API wrs_status wrs_random_gather_probe(const wrs_alias_row* d_table, int64_t n, uint64_t num_gathers,
                                           uint64_t seed, uint32_t* d_sink, void* stream);

/* ---- rejection sampling ------------------------------------------------- */

WRS_API size_t     wrs_rejection_build_scratch_bytes(int64_t n);
/* Slot array A: item i owns c_i = floor(n*w_i/W) + 1 consecutive slots (|A| <= 2n);
 * d_A[s] = item | 0x80000000 on the item's first slot. d_frac[i] = frac(n*w_i/W) as FP32,
 * the acceptance probability of the first slot. d_A_size (device u64) receives |A|.
 * a_capacity is the number of u32 entries d_A can hold (2n always suffices). */
WRS_API wrs_status wrs_rejection_build_f32(const float* d_w, int64_t n, uint32_t* d_A, uint64_t a_capacity,
                                   float* d_frac, uint64_t* d_A_size, double* d_W,
                                   void* d_scratch, size_t scratch_bytes, uint32_t flags,
                                   void* stream);
/* Sample s, try t uses Philox counter (lo32(b), hi32(b), t, 0x52454a00) with
 * b = counter_base + s: slot = floor(u * |A| / 2^64) for the 64-bit uniform u = x1:x0 (every
 * slot's share is exact to |A| / 2^64); a first slot is accepted iff
 * (x2 >> 8) * 2^-24 < frac[item]; other slots always accept.
 * After max_tries (0 = 64) failed tries the output is 0xFFFFFFFF and *d_status
 * (optional, device u32) gets WRS_ERR_TOO_MANY_TRIES. */
WRS_API wrs_status wrs_rejection_sample(const uint32_t* d_A, const uint64_t* d_A_size, const float* d_frac,
                                int64_t n, uint64_t num_samples, uint64_t seed,
                                uint64_t counter_base, uint32_t max_tries, uint32_t* d_out,
                                uint32_t* d_status, uint32_t flags, void* stream);

/* The slot array packed with the first slots' acceptance fractions: d_slots[s] (u64, 8-byte
 * aligned, a_capacity entries) = d_A[s] in the low 32 bits and, on an item's first slot, the
 * FP32 bits of d_frac[item] in the high 32 bits (0 elsewhere), for s < |A| (read from
 * d_A_size). Asynchronous. No counterpart in the reference: it is a layout of this library's
 * rejection structure, for wrs_rejection_sample_packed. */
WRS_API wrs_status wrs_rejection_pack(const uint32_t* d_A, const uint64_t* d_A_size, const float* d_frac,
                                      int64_t n, uint64_t a_capacity, uint64_t* d_slots, void* stream);
/* wrs_rejection_sample over packed slots: the same tries, slots and decisions, so the same
 * samples and status, with one random 8-byte gather per try instead of a slot gather and, on a
 * first slot, a second gather for the item's fraction. slot_capacity is the number of entries
 * d_slots holds: a |A| above it samples nothing (outputs 0xFFFFFFFF, *d_status gets
 * WRS_ERR_CAPACITY). The sampling side of SamplerRejection::sample
 * (sampling/rejectionSampling/SamplerRejection.cu:17-35). */
WRS_API wrs_status wrs_rejection_sample_packed(const uint64_t* d_slots, uint64_t slot_capacity,
                                               const uint64_t* d_A_size, int64_t n,
                                               uint64_t num_samples, uint64_t seed, uint64_t counter_base,
                                               uint32_t max_tries, uint32_t* d_out, uint32_t* d_status,
                                               uint32_t flags, void* stream);

/* ---- batched (CSR) ------------------------------------------------------ */

/* Tables t = 0..num_tables-1 own weights d_w[d_offsets[t] .. d_offsets[t+1]); their rows are
 * written at the same positions of d_table, with table-local aliases: every table's rows are
 * exactly those wrs_alias_build_f32 gives for its weights. Empty tables get no rows. The
 * offsets are int64, non-decreasing, with d_offsets[0] = 0 and tables of at most 2^31 - 8193
 * items. h_offsets is the same array in host memory: the call reads it to size the launches
 * (and only during the call); the plan itself is made on the device from d_offsets, so the
 * call issues kernels and one memset only and can be captured in a CUDA graph. If the two
 * arrays disagree, the large tables are not built and the status is WRS_ERR_INVALID_ARGUMENT.
 * d_W (optional, device, num_tables doubles) receives the per-table weight totals.
 * opts->small_table_items and opts->tile_items pick the launch shape (see
 * wrs_batched_autotune). The scratch query with opts == NULL covers every shape. */
WRS_API size_t     wrs_batched_build_scratch_bytes(const int64_t* h_offsets, int64_t num_tables,
                                           const wrs_build_opts* opts);
WRS_API wrs_status wrs_batched_build_f32(const float* d_w, const int64_t* d_offsets,
                                 const int64_t* h_offsets, int64_t num_tables,
                                 const wrs_build_opts* opts, wrs_alias_row* d_table,
                                 double* d_W /* num_tables, optional */,
                                 void* d_scratch, size_t scratch_bytes, void* stream);
/* Table t draws d_sample_offsets[t+1] - d_sample_offsets[t] samples, written (as table-local
 * row indices) at d_out[d_sample_offsets[t] ...]. Output position s of table t uses the
 * plain contract with b = counter_base + s over the global position s. */
WRS_API wrs_status wrs_batched_sample(const wrs_alias_row* d_table, const int64_t* d_offsets,
                              int64_t num_tables, const int64_t* d_sample_offsets,
                              uint64_t total_samples, uint64_t seed, uint64_t counter_base,
                              uint32_t* d_out, void* stream);
/* The batched build and the batched sampler in one call, with the same rows and the same
 * samples as wrs_batched_build_f32 followed by wrs_batched_sample. The samples of each table of
 * at most 8192 items (with at most 2048 samples) are drawn as soon as its size class is built,
 * on the side stream that built it, while the larger tables are still being built; the other
 * tables' samples follow the last build. d_sample_offsets must start at 0 and end at
 * total_samples; an empty table with samples gets 0xFFFFFFFF at its positions and the status
 * WRS_ERR_INVALID_ARGUMENT. Can be captured in a CUDA graph. */
WRS_API size_t     wrs_batched_build_sample_scratch_bytes(const int64_t* h_offsets, int64_t num_tables,
                                                  const wrs_build_opts* opts);
WRS_API wrs_status wrs_batched_build_sample(const float* d_w, const int64_t* d_offsets,
                                    const int64_t* h_offsets, int64_t num_tables,
                                    const wrs_build_opts* opts, wrs_alias_row* d_table,
                                    double* d_W /* num_tables, optional */,
                                    const int64_t* d_sample_offsets, uint64_t total_samples,
                                    uint64_t seed, uint64_t counter_base, uint32_t* d_out,
                                    void* d_scratch, size_t scratch_bytes, void* stream);
/* The one-table-per-launch form of a batch, for comparison with the batched calls: for each
 * table t in h_tables[0 .. num_ids), one wrs_alias_build_f32 of its weights into its rows and
 * one wrs_alias_sample of its h_sample_offsets[t+1] - h_sample_offsets[t] samples with
 * counter_base + h_sample_offsets[t] (the same samples as the batched sampler), in order on
 * `stream`. d_scratch must hold the single-table scratch of the largest of these tables. */
WRS_API wrs_status wrs_batched_per_table(const float* d_w, const int64_t* h_offsets,
                                 const int64_t* h_sample_offsets, const int64_t* h_tables,
                                 int64_t num_ids, const wrs_build_opts* opts, wrs_alias_row* d_table,
                                 uint64_t seed, uint64_t counter_base, uint32_t* d_out,
                                 void* d_scratch, size_t scratch_bytes, void* stream);
/* Times the batched build of this batch for every launch shape (small_table_items in
 * {32, 64, 128, 256, 512} x tile_items in {1024, 2048, 4096}) and writes the fastest into
 * *opts (method and flags are kept). Synchronous; it builds into d_table (the same rows every
 * time). d_scratch must hold the opts == NULL scratch query. */
WRS_API wrs_status wrs_batched_autotune(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                int64_t num_tables, wrs_alias_row* d_table, void* d_scratch,
                                size_t scratch_bytes, wrs_build_opts* opts, void* stream);

/* The same search for wrs_batched_build_sample: every shape's build and sample call is timed
 * (samples with seed 0 into d_out). d_scratch must hold the opts == NULL scratch query of
 * wrs_batched_build_sample_scratch_bytes. */
WRS_API wrs_status wrs_batched_autotune_build_sample(const float* d_w, const int64_t* d_offsets,
                                             const int64_t* h_offsets, int64_t num_tables,
                                             wrs_alias_row* d_table, const int64_t* d_sample_offsets,
                                             uint64_t total_samples, uint32_t* d_out, void* d_scratch,
                                             size_t scratch_bytes, wrs_build_opts* opts, void* stream);

/* ---- mixed batches: alias or rejection per table ----------------------- */

/* Method of each table of a mixed batch, one byte per table (d_kinds in device memory,
 * h_kinds the same array in host memory). A table of any other kind is skipped: it gets no
 * rows and no slots, and its sample positions are left as they are. */
#define WRS_TABLE_ALIAS 0u
#define WRS_TABLE_REJECTION 1u
#define WRS_TABLE_SKIP 2u

/* Builds every table by its kind. Alias tables as wrs_batched_build_f32 does (their rows in
 * d_table at the table's items, table-local aliases). Rejection tables as
 * wrs_rejection_build_f32 does for their weights: c_i = floor(n w_i / W) + 1 slots per item,
 * the table's slots at d_A[2 * offsets[t] ...] (|A_t| <= 2 n_t, in d_a_size[t]), first-slot
 * acceptances at d_frac[offsets[t] ...], table-local items. d_A holds 2 * offsets[num_tables]
 * slots, d_frac offsets[num_tables] floats, d_a_size num_tables u64 (written for rejection
 * tables only). h_kinds sizes the launches, as h_offsets does; a NULL kinds pair makes every
 * table an alias table. The scratch query with h_kinds = NULL covers every choice of kinds.
 * Replaces a loop of AliasTableSplitGpu and RejectionSampling objects, one per table
 * (AliasTableSplitGpu.cu:388-468, RejectionSampling.cu:35-56). */
WRS_API size_t     wrs_batched_mixed_build_scratch_bytes(const int64_t* h_offsets, const uint8_t* h_kinds,
                                                         int64_t num_tables, const wrs_build_opts* opts);
WRS_API wrs_status wrs_batched_mixed_build_f32(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                               const uint8_t* d_kinds, const uint8_t* h_kinds, int64_t num_tables,
                                               const wrs_build_opts* opts, wrs_alias_row* d_table, uint32_t* d_A,
                                               float* d_frac, uint64_t* d_a_size, double* d_W /* optional */,
                                               void* d_scratch, size_t scratch_bytes, void* stream);
/* One launch for the whole batch: output position s of table t follows table t's kind.
 * Alias tables: the contract of wrs_batched_sample. Rejection tables: the contract of
 * wrs_rejection_sample over the global position s (b = counter_base + s, at most max_tries
 * tries, 0 = 64), the result a table-local item. A table without items (or without slots)
 * and a rejection sample that runs out of tries write 0xFFFFFFFF and record the error in
 * *d_status (optional, device). */
WRS_API wrs_status wrs_batched_mixed_sample(const wrs_alias_row* d_table, const uint32_t* d_A, const float* d_frac,
                                            const uint64_t* d_a_size, const int64_t* d_offsets,
                                            const uint8_t* d_kinds, int64_t num_tables,
                                            const int64_t* d_sample_offsets, uint64_t total_samples, uint64_t seed,
                                            uint64_t counter_base, uint32_t max_tries, uint32_t* d_out,
                                            uint32_t* d_status, void* stream);
/* The autotuner's choice of method per size class; class c holds the tables with
 * 2^(c-1) < n <= 2^c (class 0: n = 1). For every class present it times the mixed build and
 * the mixed sample of that class's tables alone (every other table skipped), once as alias
 * and once as rejection tables, with the batch's sample counts (h_sample_offsets is the host
 * copy of d_sample_offsets). A class takes rejection where that took under 0.95 of alias's
 * time, else alias. It writes each table's kind into h_kinds_out (empty tables:
 * WRS_TABLE_SKIP) and, if class_kinds is not NULL, the choice per class into
 * class_kinds[0..32] (WRS_TABLE_SKIP for absent classes), and if class_ms is not NULL the
 * timings behind the choice into class_ms[0..65] (class c: [2c] as alias, [2c+1] as rejection,
 * in ms; 0 for absent classes). Synchronous. d_kinds_tmp (num_tables
 * bytes) and d_out (the batch's samples) are working buffers on the device; the other buffers
 * are those of wrs_batched_mixed_build_f32, with the scratch of its query for h_kinds = NULL.
 * This replaces the reference's compile-time choice of one method for every table. */
WRS_API wrs_status wrs_batched_autotune_kinds(const float* d_w, const int64_t* d_offsets, const int64_t* h_offsets,
                                              int64_t num_tables, const int64_t* d_sample_offsets,
                                              const int64_t* h_sample_offsets, const wrs_build_opts* opts,
                                              wrs_alias_row* d_table, uint32_t* d_A, float* d_frac,
                                              uint64_t* d_a_size, uint8_t* d_kinds_tmp, uint32_t* d_out,
                                              void* d_scratch, size_t scratch_bytes, uint8_t* h_kinds_out,
                                              uint8_t* class_kinds, float* class_ms, void* stream);

/* ---- autotuning of the single-table build and the sectioned sampler --- */

/* Times the split build of these weights at every tile size (1024, 2048, 4096; those whose
 * scratch fits scratch_bytes) and writes the fastest into opts->tile_items (method SPLIT,
 * precision MIXED). Synchronous; it builds into d_table. Replaces the reference's compile-time
 * launch shapes and its fixed rule for the split count (AliasTableSplitGpu.cuh:60-94,
 * AliasTableSplitGpu.cu:53-75). The choice is recorded for this GPU and ceil(log2 n). */
WRS_API wrs_status wrs_autotune_build(const float* d_w, int64_t n, wrs_alias_row* d_table, void* d_scratch,
                                      size_t scratch_bytes, wrs_build_opts* opts, void* stream);
/* Times WRS_SAMPLE_SECTIONED sampling of num_samples from this table at section sizes 512 ..
 * 65536 and writes the fastest into *section_items (recorded like wrs_autotune_build's choice).
 * Synchronous; d_out holds num_samples. The reference takes the section size as an argument
 * (SamplerGpuSectioned.cu:7-9). */
WRS_API wrs_status wrs_autotune_sections(const wrs_alias_row* d_table, int64_t n, uint64_t num_samples,
                                         uint32_t* d_out, uint32_t* section_items, void* stream);
/* The recorded choices for this GPU and ceil(log2 n) (0 where not tuned); WRS_ERR_INVALID_ARGUMENT
 * when nothing is recorded for that size. */
WRS_API wrs_status wrs_autotune_lookup(int64_t n, uint32_t* tile_items, uint32_t* section_items);
/* The recorded choices as JSON, {"entries": [{"gpu", "log2n", "tile_items", "section_items"}]},
 * written to / merged from a file. */
WRS_API wrs_status wrs_autotune_cache_save(const char* path);
WRS_API wrs_status wrs_autotune_cache_load(const char* path);

/* ---- reference table format -------------------------------------------- */

/* Writes the table in the reference's format (TableStorage, construction/aliasTable/
 * TableStorage.cuh:6-128, structure of arrays): d_weight[i] = prob_i * W / n (absolute FP64
 * weight in [0, W/n]) and d_alias[i] = alias_i, for code written against the reference
 * (verifyTableCorrectness, doSample). W is the weight total the build used (its d_W). */
WRS_API wrs_status wrs_export_reference_table(const wrs_alias_row* d_table, int64_t n, double W,
                                              double* d_weight, int32_t* d_alias, void* stream);

/* ---- table files -------------------------------------------------------- */

/* A table saved to a file and read back, so that a table built once is sampled later by another
 * process or on another device (the reference keeps its tables in memory only,
 * construction/aliasTable/TableStorage.cuh:6-128). The file holds a 64-byte header (magic
 * "WRSTABLE", version, row size, n, number of tables, W, an FNV-1a checksum of offsets and rows),
 * the CSR offsets (num_tables + 1 int64) and the n rows. The calls copy through host memory in
 * chunks, synchronising `stream`. */
WRS_API wrs_status wrs_table_file_write(const char* path, const wrs_alias_row* d_table, int64_t n, double W,
                                        void* stream);
WRS_API wrs_status wrs_batched_table_file_write(const char* path, const wrs_alias_row* d_table,
                                                const int64_t* h_offsets, int64_t num_tables, void* stream);
/* Rows, tables and W (0 for a batch) of a table file; WRS_ERR_INVALID_ARGUMENT if it is not one. */
WRS_API wrs_status wrs_table_file_info(const char* path, int64_t* n, int64_t* num_tables, double* W);
/* Reads the rows into d_table (n rows; n and num_tables must match the file, else
 * WRS_ERR_CAPACITY) and the offsets into h_offsets (optional, num_tables + 1); a checksum
 * mismatch gives WRS_ERR_INVALID_ARGUMENT. */
WRS_API wrs_status wrs_table_file_read(const char* path, wrs_alias_row* d_table, int64_t n, int64_t* h_offsets,
                                       int64_t num_tables, void* stream);

/* ---- sharding a batch over devices ------------------------------------- */

/* Tables are independent, so a batch spreads over devices by contiguous table ranges with no
 * exchange between them: shard s builds and samples tables [h_bounds[s], h_bounds[s+1]) with
 * the batched calls on its own device. The ranges balance items + table_cost per table
 * (table_cost: the items one table's fixed costs are worth, e.g. 16). Host only; no counterpart
 * in the reference (one GPU). */
WRS_API wrs_status wrs_shard_tables(const int64_t* h_offsets, int64_t num_tables, int32_t num_shards,
                                    int64_t table_cost, int64_t* h_bounds);

/* ---- status / misc ------------------------------------------------------ */

/* Bounded device waits. Every device-side wait of the library (the decoupled look-back scans
 * of the builds) gives up after a time limit, records WRS_ERR_DEVICE_TIMEOUT in the status
 * word and returns, so a wait never hangs the GPU. This sets the limit for launches this
 * process makes from now on: limit_ns = 0 restores the default (2 s); at most 60 s. No
 * counterpart in the reference (its kernels never wait on one another). */
WRS_API wrs_status wrs_set_device_wait_limit(uint64_t limit_ns);
/* For failure-detection tests: look-back block or tile `block` (its index in launch order) of
 * the builds launched from now on publishes nothing, so that the waits of the blocks after it
 * run out at the limit and the build reports WRS_ERR_DEVICE_TIMEOUT (its outputs are then
 * invalid); block = -1 turns this off. No counterpart in the reference. */
WRS_API wrs_status wrs_debug_hold_lookback(int64_t block);

/* Reads (synchronising `stream`) the device status word of a build scratch buffer. */
WRS_API wrs_status wrs_scratch_status(const void* d_scratch, void* stream);
WRS_API const char* wrs_status_string(wrs_status status);
/* Returns WRS_SUCCESS when the current device is an sm_100 part the kernels were built for. */
WRS_API wrs_status wrs_check_device(void);
WRS_API int        wrs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WRS_H */
