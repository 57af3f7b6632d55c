/* dvgpu C-ABI: BN254 prover operators on NVIDIA B200 (sm_100a).
 *
 * Drop-in for the reference's native ABI, native/include/dynaverse_gpu.h,
 * whose symbols the Rust crate binds in crates/gpu/src/icicle.rs:35-57,
 * crates/gpu/src/setup.rs:47-52 and crates/gpu/src/g2_validation.rs:84-93.
 * Every entry point of the reference that this library implements keeps its
 * exact signature, argument meaning and status codes:
 *
 *    0  success (outputs written)
 *   -1  invalid argument; nothing written, owner unchanged
 *   -2  CUDA failure; the owner is retired
 *   -3  unknown native exception; the owner is retired
 *   -4  owner already retired (create a new owner to recover)
 *   -5  G2 content rejected; only the report is published
 *
 * Wire formats (crates/gpu/src/codec.rs:25-111, crates/gpu/src/resident.rs:419-431):
 * Fr and Fq elements are 32-byte little-endian canonical integers (NOT
 * Montgomery), G1 points 64 bytes x||y, G2 points 128 bytes
 * x.c0||x.c1||y.c0||y.c1, infinity all zero.  Host-buffer calls are
 * synchronous and retain no caller pointer.  Error text is NUL-terminated
 * into (error, error_capacity) when capacity > 0.
 *
 * Differences from the reference, all additive:
 *  - size caps are lifted: MSM up to DVGPU_MAX_MSM_SIZE points, NTT up to
 *    DVGPU_MAX_NTT_SIZE, fixed base and G2 validation up to
 *    DVGPU_MAX_SETUP_SIZE per call (the reference stops at 2^20 / 2^20 /
 *    4096);
 *  - owners share the device's primary context, so the *_device entry points
 *    accept device pointers from any runtime user on the same device;
 *  - new entry points below the reference set are marked "additive".
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

enum { DVGPU_MAX_MSM_SIZE = 1 << 26 };
enum { DVGPU_MAX_NTT_SIZE = 1 << 26 };
enum { DVGPU_MAX_SETUP_SIZE = 1 << 26 };
enum { DVGPU_MAX_MSM_BATCH_SIZE = 1 << 20 };
enum { DVGPU_MAX_LARGE_BUCKET_FACTOR = 100 };

#ifdef __cplusplus
extern "C" {
#endif

/* ---- owner lifecycle (native/include/dynaverse_gpu.h:15-27) ------------ */
int dvgpu_backend_create(void** backend, char* error, size_t error_capacity);
/* factor 0..100 is validated and recorded; bucket load balancing is always on
 * in this engine, so the value does not change results or the algorithm. */
int dvgpu_backend_create_with_large_bucket_factor(uint32_t factor, void** backend, char* error,
                                                  size_t error_capacity);
void dvgpu_backend_destroy(void* backend);
int dvgpu_backend_device_identity(void* backend, char* output, size_t output_capacity, char* error,
                                  size_t error_capacity);

/* ---- MSM (native/include/dynaverse_gpu.h:28-38, 46-52) ----------------- */
int dvgpu_bn254_msm(void* backend, const uint8_t* points, const uint8_t* scalars, size_t length, uint8_t* result,
                    char* error, size_t error_capacity);
int dvgpu_bn254_g2_msm(void* backend, const uint8_t* points, const uint8_t* scalars, size_t length, uint8_t* result,
                       char* error, size_t error_capacity);
/* count sets, each padded to `length` points (points_size = length * count). */
int dvgpu_bn254_msm_batch(void* backend, const uint8_t* points, const uint8_t* scalars, size_t length, size_t count,
                          uint8_t* results, char* error, size_t error_capacity);

/* ---- NTT (native/include/dynaverse_gpu.h:39-45) ------------------------ */
/* root: the canonical primitive 2^20-th root of unity of the CPU reference
 * (Fr::get_root_of_unity(2^20), icicle.rs:442-443); checked to have order
 * exactly 2^20 and to equal that root (the reference fixes whichever root of
 * order 2^20 an owner sees first; this library fixes arkworks' one, since
 * another root defines a different, conjugate, transform).  length: a power
 * of two up to 2^20, the longest transform such a root defines; longer ones
 * go through dvgpu_bn254_ntt_ex. */
int dvgpu_bn254_ntt(void* backend, const uint8_t* values, size_t length, int inverse, const uint8_t* root,
                    uint8_t* result, char* error, size_t error_capacity);

typedef struct DvgpuBatchStats {
    uint64_t icicle_calls; /* native batch launches */
    uint64_t buffer_grows;
    uint64_t max_batch_size;
    uint64_t input_capacity;
} DvgpuBatchStats;
typedef struct DvgpuSetupStats {
    uint64_t table_builds[2], calls[2], points[2], table_bytes;
    uint64_t device_ns[5], native_wall_ns;
} DvgpuSetupStats;
/* native/include/dynaverse_gpu.h:59-66: mode 0..2 is validated and recorded;
 * this engine always uses the table + batch-normalise path (mode 2). */
int dvgpu_setup_mode(void* backend, int mode);
int dvgpu_setup_stats(void* backend, DvgpuSetupStats* stats);

/* ---- G2 validation (native/include/dynaverse_gpu.h:67-89) -------------- */
typedef struct DvgpuG2ValidationReport {
    uint64_t checked_points, invalid_points, first_invalid;
    uint32_t failure_mask, algorithm;
} DvgpuG2ValidationReport;
typedef struct DvgpuG2ValidationStats {
    uint64_t parse_curve_device_ns, subgroup_device_ns, reduce_device_ns;
    uint64_t h2d_device_ns, d2h_device_ns, native_wall_ns;
    uint64_t checked_points, accepted_points;
} DvgpuG2ValidationStats;
/* masks: 1 encoding, 2 off-curve, 4 outside the subgroup; algorithm 1/2/3. */
int dvgpu_bn254_g2_validation_inspect(void* owner, const uint8_t* wire, size_t n, uint32_t algorithm,
                                      uint32_t* point_masks, DvgpuG2ValidationReport* report, char* error,
                                      size_t error_capacity);
int dvgpu_g2_validation_stats(void* owner, DvgpuG2ValidationStats* stats);
typedef struct DvgpuG2ValidationTraffic {
    uint64_t scalar_h2d_bytes, point_h2d_bytes, point_d2h_bytes, status_d2h_bytes;
} DvgpuG2ValidationTraffic;
int dvgpu_g2_validation_traffic(void* owner, DvgpuG2ValidationTraffic* stats);
/* Fixed-base G2 generation validated on the device; -5 publishes only the report. */
int dvgpu_bn254_fixed_base_g2_checked(void* owner, const uint8_t* scalars, size_t n, uint32_t algorithm,
                                      uint8_t* output, DvgpuG2ValidationReport* report, char* error,
                                      size_t error_capacity);
/* G2 check kernel diagnostics (native/include/dynaverse_g2_experiments.h:6-17,
 * bound by crates/gpu/src/g2_validation.rs:91-94).  config: threads 64, 128
 * or 256 is the check kernel's block size; schedule, layout and fused (0 or
 * 1) name the reference's experimental variants and are accepted and kept
 * without effect (this library has one check kernel, with the fixed-base
 * normalisation always fused).  resources: the check kernel's attributes and
 * theoretical occupancy at the configured block size, and those of the
 * checked G2 fixed-base generation.  experiment stats: no repacking
 * (repack fields 0); subgroup_kernel_ns sums the check kernel's device time. */
typedef struct DvgpuG2KernelConfig {
    uint32_t threads, schedule, layout, fused;
} DvgpuG2KernelConfig;
typedef struct DvgpuG2ExperimentStats {
    uint64_t repack_device_ns, subgroup_kernel_ns, logical_repack_bytes;
} DvgpuG2ExperimentStats;
typedef struct DvgpuG2KernelResources {
    uint32_t registers, block_threads, active_blocks, max_threads_per_sm;
    uint64_t local_bytes, shared_bytes;
    uint32_t normalize_registers, normalize_active_blocks;
    uint64_t normalize_local_bytes, normalize_shared_bytes;
} DvgpuG2KernelResources;
int dvgpu_g2_kernel_config_set(void* owner, const DvgpuG2KernelConfig* config);
int dvgpu_g2_kernel_config_get(void* owner, DvgpuG2KernelConfig* config);
int dvgpu_g2_kernel_resources(void* owner, uint32_t algorithm, DvgpuG2KernelResources* output);
int dvgpu_g2_experiment_stats(void* owner, DvgpuG2ExperimentStats* output);
int dvgpu_backend_batch_stats(void* backend, DvgpuBatchStats* stats);
typedef struct DvgpuMemoryInfo {
    uint64_t free_bytes;
    uint64_t total_bytes;
} DvgpuMemoryInfo;
int dvgpu_backend_memory_info(void* backend, DvgpuMemoryInfo* info, char* error, size_t error_capacity);

/* ---- fixed base (crates/gpu/src/setup.rs:47-52; icicle_msm.cu:494-521) --- */
/* [s_i] G for the standard G1 (g2 = 0) or G2 (g2 = 1) generator. */
int dvgpu_bn254_fixed_base(void* backend, const uint8_t* scalars, size_t length, int g2, uint8_t* output, char* error,
                           size_t error_capacity);
int dvgpu_reserve_batch(void* backend, size_t points, char* error, size_t error_capacity);

/* ---- diagnostics (native/include/dynaverse_gpu.h:159-168) -------------- */
typedef struct DvgpuMsmTimings {
    uint64_t conversion_ns; /* host-side argument handling */
    uint64_t icicle_ns;     /* device work incl. transfers and synchronisation */
    uint64_t output_ns;     /* host-side window combination and normalisation */
} DvgpuMsmTimings;
int dvgpu_bn254_msm_profiled(void* backend, const uint8_t* points, const uint8_t* scalars, size_t length,
                             uint8_t* result, DvgpuMsmTimings* timings, char* error, size_t error_capacity);
/* One MSM with its phase timeline (native/include/dynaverse_gpu.h:169-192,
 * bound by crates/gpu/src/icicle.rs:54, used at :250).  Phases: 0
 * allocation_preparation, 1 point_h2d, 2 scalar_h2d, 3 kernel_submission
 * (point conversion, digit sort, accumulation, reduction, window
 * combination), 4 synchronization, 5 output_d2h, 6 remaining_overhead, 7
 * metadata_d2h (the point-validation word), 8 free (nothing is freed: the
 * workspaces grow only).  wall_ns is the host clock, event_ns CUDA events on
 * the owner's stream: different clocks, not additive.  Kernel slots: 0
 * digit histogram, 1 offsets scan, 2 scatter, 6 bucket accumulation with its
 * split-bucket merges, 7 bucket reduction, 8 window combination (host), 9
 * point conversion (not timed alone: 0).  label names the call in the
 * reference's NVTX ranges and is unused here. */
enum { DVGPU_TIMELINE_PHASES = 9, DVGPU_TIMELINE_KERNELS = 10 };
typedef struct DvgpuMsmTimeline {
    uint64_t wall_ns[DVGPU_TIMELINE_PHASES];
    uint64_t event_ns[DVGPU_TIMELINE_PHASES];
    uint64_t calls[DVGPU_TIMELINE_PHASES];
    uint64_t event_calls[DVGPU_TIMELINE_PHASES];
    uint64_t bytes[DVGPU_TIMELINE_PHASES];
    uint64_t kernel_ns[DVGPU_TIMELINE_KERNELS];
    uint64_t kernel_calls[DVGPU_TIMELINE_KERNELS];
    uint64_t instrumentation_inclusive_ns;
    uint64_t instrumentation_total_ns;
    uint64_t c;
    uint64_t bitsize;
    uint64_t windows;
    uint64_t buckets;
} DvgpuMsmTimeline;
int dvgpu_bn254_msm_timeline(void* backend, const uint8_t* points, const uint8_t* scalars, size_t length,
                             uint8_t* result, const char* label, DvgpuMsmTimings* timings, DvgpuMsmTimeline* timeline,
                             char* error, size_t error_capacity);

/* ---- research probes: declared so the crate's extern blocks link --------
 * The reference's tower, line and Miller-loop inspectors and G2 psi probe
 * (crates/gpu/src/bn254_tower.rs:40, bn254_lines.rs:24, bn254_miller.rs:38,
 * g2_validation/tests.rs:273) and its test-only corruption hook
 * (g2_validation/tuning_tests.rs:7) are diagnostics outside the compute
 * path; here each returns -1 with "not provided" in the error text and
 * writes no output.  The pairing checks they were built towards are
 * dvgpu_bn254_pairing_check and friends. */
int dvgpu_bn254_tower_inspect(void* owner, uint32_t degree, uint32_t operation, uint32_t power, const uint8_t* left,
                              size_t left_bytes, const uint8_t* right, size_t right_bytes, uint8_t* output,
                              size_t output_bytes, uint32_t* statuses, size_t statuses_count, char* error,
                              size_t error_capacity);
int dvgpu_bn254_lines_inspect(void* owner, const uint8_t* points, size_t points_bytes, uint8_t* output,
                              size_t output_bytes, uint32_t* counts, size_t counts_count, uint32_t* statuses,
                              size_t statuses_count, char* error, size_t error_capacity);
int dvgpu_bn254_miller_inspect(void* owner, const uint8_t* p, size_t p_bytes, const uint8_t* q, size_t q_bytes,
                               uint8_t* output, size_t output_bytes, uint32_t* metadata, size_t metadata_count,
                               char* error, size_t error_capacity);
int dvgpu_g2_psi_probe(void* owner, const uint8_t* points, size_t n, uint8_t* output, char* error,
                       size_t error_capacity);
int dvgpu_g2_test_corrupt_next(void* owner, uint64_t index);

/* ======================= additive entry points ========================= */

/* NTT of any kind: 0 forward, 1 inverse, 2 coset forward, 3 coset inverse
 * (coset offset g = 5, the Fr multiplicative generator).  The domain root is
 * the arkworks one (GENERATOR^((r-1)/2^28) squared down to order length). */
int dvgpu_bn254_ntt_ex(void* backend, const uint8_t* values, size_t length, int kind, uint8_t* result, char* error,
                       size_t error_capacity);

/* count independent G1 MSMs of uneven sizes in one launch sequence:
 * set k uses points/scalars [set_offsets[k], set_offsets[k+1]). */
int dvgpu_bn254_msm_batch_uneven(void* backend, const uint8_t* points, const uint8_t* scalars,
                                 const uint64_t* set_offsets, size_t count, uint8_t* results, char* error,
                                 size_t error_capacity);

/* Resident MSM bases (an SRS table kept in HBM across calls).  points are
 * validated (canonical, on curve) and converted once.  g2 selects G2. */
int dvgpu_bases_register(void* backend, const uint8_t* points, size_t n, int g2, uint64_t* handle, char* error,
                         size_t error_capacity);
int dvgpu_bases_release(void* backend, uint64_t handle);
/* Precomputed window multiples for registered bases: stores 2^(c w) P_i for
 * every base and window (windows = ceil(255 / c) entries per base, e.g. 13 x
 * 64 B per G1 base at c = 20).  dvgpu_bn254_msm_resident then adds every
 * window into one shared bucket set and skips the window combination.
 * c = 0 picks the width by cost model; c_used (may be NULL) receives it. */
int dvgpu_bases_precompute(void* backend, uint64_t handle, int c, int* c_used, char* error, size_t error_capacity);

/* Sparse-index G1 MSM over resident bases (OperatorBackend::msm_sparse_batch,
 * crates/protocol/src/types.rs:262-345): request k sums
 * values[j] * bases[indices[j]] for j in [request_offsets[k], request_offsets[k+1]).
 * Order, repeated indices and zero values are preserved; an index >= n of
 * the registered table is rejected (-1) before any result is written. */
int dvgpu_bn254_msm_sparse_batch(void* backend, uint64_t bases_handle, const uint64_t* indices, const uint8_t* values,
                                 const uint64_t* request_offsets, size_t count, uint8_t* results, char* error,
                                 size_t error_capacity);

/* The same over device-resident indices and values (request_offsets and the
 * results stay in host memory).  Indices are checked on the device; an index
 * out of range returns -1 and writes no result. */
int dvgpu_bn254_msm_sparse_device(void* backend, uint64_t bases_handle, const uint64_t* d_indices,
                                  const uint8_t* d_values, const uint64_t* request_offsets, size_t count,
                                  uint8_t* results_host, void* stream, char* error, size_t error_capacity);

/* Device-pointer forms (inputs already in HBM, canonical wire layout).
 * stream: a cudaStream_t, or NULL for the owner's stream.  The call returns
 * after the device work on `stream` completed.  result_host: host memory. */
int dvgpu_bn254_msm_device(void* backend, const uint8_t* d_points, const uint8_t* d_scalars, size_t length, int g2,
                           uint8_t* result_host, void* stream, char* error, size_t error_capacity);
/* MSM over a registered base table (first `length` bases) with device scalars. */
int dvgpu_bn254_msm_resident(void* backend, uint64_t bases_handle, const uint8_t* d_scalars, size_t length,
                             uint8_t* result_host, void* stream, char* error, size_t error_capacity);
/* The resident-bases MSM with scalars in host memory (synchronous, like
 * dvgpu_bn254_msm): the per-request call of a prover whose SRS is resident. */
int dvgpu_bn254_msm_resident_host(void* backend, uint64_t bases_handle, const uint8_t* scalars, size_t length,
                                  uint8_t* result, char* error, size_t error_capacity);
int dvgpu_bn254_ntt_device(void* backend, const uint8_t* d_values, size_t length, int kind, uint8_t* d_result,
                           void* stream, char* error, size_t error_capacity);
int dvgpu_bn254_fixed_base_device(void* backend, const uint8_t* d_scalars, size_t length, int g2, uint8_t* d_output,
                                  void* stream, char* error, size_t error_capacity);
int dvgpu_bn254_g2_check_device(void* backend, const uint8_t* d_wire, size_t n, uint32_t algorithm,
                                uint32_t* d_masks, DvgpuG2ValidationReport* report_host, void* stream, char* error,
                                size_t error_capacity);

/* Autotuner: times candidate window widths on seeded synthetic data of n
 * points (G1 or G2) on this owner, stores the fastest for n's size class
 * (ceil(log2 n)) and returns it; later MSMs of that class use it.  log_json
 * receives the measured candidates as one JSON object. */
int dvgpu_msm_autotune(void* backend, size_t n, int g2, int* best_c, char* log_json, size_t log_capacity,
                       char* error, size_t error_capacity);
/* Allocation-free NTT (no counterpart in the reference).  For callers that
 * must not allocate device memory when they need a transform -- code that
 * runs while a caching allocator or memory pool owns device memory, a
 * latency-critical path that cannot afford the device synchronisation
 * cudaMalloc/cudaFree may cause, or a host with a device-memory budget fixed
 * at start-up.  The caller passes canonical input and output device buffers
 * and a stream (NULL = legacy default stream); no owner is needed, and the
 * call allocates nothing: its working memory is a static device array of
 * about 3.1 MB reserved on each device that loads the library, held until
 * process exit.  length is a power of two up to 65536 (larger is rejected
 * with -1); kind as in dvgpu_bn254_ntt_ex.  Calls share that array: calls
 * whose device work overlaps (unordered streams) race and must be
 * serialised by the caller.  The first call on a device looks up the
 * array's address and should come before any stream capture.  Returns after
 * the transform on `stream` has completed. */
int dvgpu_bn254_ntt_noalloc(const uint8_t* d_values, size_t length, int kind, uint8_t* d_result, void* stream,
                            char* error, size_t error_capacity);

/* Tuning: force the Pippenger window width c (0 = autotuned / cost-model choice). */
int dvgpu_msm_set_window(void* backend, int c);
int dvgpu_msm_get_window(void* backend, size_t points_per_set, int* c);

/* Integer-multiply roofline probe: runs a dependent-chain-free kernel of
 * mad.lo.cc / madc.hi.cc pairs on every SM and reports the achieved
 * 32x32->64-bit multiply-accumulate rate (MAC/s). */
int dvgpu_probe_imad_rate(void* backend, double* macs_per_second, char* error, size_t error_capacity);

/* Diagnostics: kernel launches of this library since load (all owners). */
uint64_t dvgpu_launch_count(void);
/* Per-phase MSM device time, accumulated over calls while enabled (CUDA
 * events on the launching stream).  ms[]: 0 digit histogram, 1 offsets scan,
 * 2 scatter, 3 bucket accumulation, 4 split-bucket merges, 5 bucket
 * reduction, 6 unused, 7 tail (window D2H + host Horner).  enable = 1
 * resets and starts, 0 stops; out (may be NULL) receives the totals so far. */
typedef struct DvgpuMsmPhaseTimes {
    double ms[8];
    uint64_t calls;
    uint64_t accum_mixed_adds; /* points x windows accumulated while enabled */
} DvgpuMsmPhaseTimes;
int dvgpu_msm_timeline(void* backend, int enable, DvgpuMsmPhaseTimes* out);

/* Seeded synthetic inputs on the device: n uniform Fr scalars (canonical),
 * and the powers tau^0..tau^(n-1) of a canonical device scalar. */
int dvgpu_random_fr_device(void* backend, uint64_t seed, size_t n, uint8_t* d_out, void* stream, char* error,
                           size_t error_capacity);
int dvgpu_fr_powers_device(void* backend, const uint8_t* d_tau, size_t n, uint8_t* d_out, void* stream, char* error,
                           size_t error_capacity);
/* n seeded random points of the G2 twist curve, 128-byte wire form, with no
 * cofactor clearing: on the curve but (with overwhelming probability) not in
 * the order-r subgroup -- the invalid half of a subgroup-check corpus, as
 * built by crates/gpu/src/g2_validation/tests.rs:24-31. */
int dvgpu_g2_random_twist_device(void* backend, uint64_t seed, size_t n, uint8_t* d_out, void* stream, char* error,
                                 size_t error_capacity);

/* G1 transform (EC-NTT) of `rows` rows of row_len = 2^k points (wire form,
 * 64 bytes each, k <= 20, at most 2^24 points in all): per row
 * out_i = sum_j w^(ij) P_j in natural order, w the arkworks root of order
 * row_len; inverse = 1 uses w^-1 and scales by 1/row_len; results are
 * canonical affine (RebuildBackend::transform_rows with kind G1,
 * crates/protocol/src/incremental_rebuild/operators.rs:413-440; ICICLE's
 * dvgpu_ecntt_rows, native/src/icicle_ntt.cu:90-95).  Invalid points: -1. */
int dvgpu_bn254_g1_ntt_rows(void* backend, const uint8_t* points, size_t row_len, size_t rows, int inverse,
                            uint8_t* results, char* error, size_t error_capacity);
int dvgpu_bn254_g1_ntt_rows_device(void* backend, const uint8_t* d_points, size_t row_len, size_t rows, int inverse,
                                   uint8_t* d_results, void* stream, char* error, size_t error_capacity);

/* ---------------------------------------------------------------- pairing checks
 * The verifier's pairing-product checks (crates/protocol/src/verification.rs
 * :37-144, PairingChecks::equal / equal_prepared / product_equal over
 * Bn254::multi_miller_loop + final_exponentiation).  Terms are (G1 64 B,
 * G2 128 B) wire points, canonical, on their curves (all zero = infinity,
 * which contributes one); the caller negates right-hand G1 points as
 * product_equal does.  Equation e holds iff the product over terms
 * [offsets[e], offsets[e+1]) of e(P_k, Q_k) is one; verdicts[e] = 1 / 0.
 * offsets has equations + 1 entries, offsets[0] = 0; at most 2^24 terms and
 * equations.  An invalid point: -1 naming the term. */
int dvgpu_bn254_pairing_check(void* backend, const uint8_t* g1, const uint8_t* g2, const uint64_t* offsets,
                              size_t equations, uint8_t* verdicts, char* error, size_t error_capacity);
/* e(P_i, Q_i) for n pairs: 384-byte GT elements, Fq12 in tower order
 * (c0.c0.c0, c0.c0.c1, c0.c1.c0, ..., c1.c2.c1; Fq12 = Fq6 + Fq6 w,
 * Fq6 = Fq2 + Fq2 v + Fq2 v^2), canonical 32-byte LE Fq.  The final
 * exponent is (q^12 - 1)/r times 2z(6z^2 + 3z + 1). */
int dvgpu_bn254_pairing(void* backend, const uint8_t* g1, const uint8_t* g2, size_t n, uint8_t* gt, char* error,
                        size_t error_capacity);
/* Prepared G2 points (arkworks G2Prepared; the verifier caches one per
 * distinct G2 point, crates/protocol/src/verification.rs:105-126, and the
 * rebuild checks use fixed preparations, :55-77): the 88 lines of each
 * point's Miller loop are computed once and kept on the device under a
 * handle (at most 2^17 points, 17 KB each).  dvgpu_bn254_pairing_check
 * prepares the distinct G2 points of a call by itself when some repeat;
 * these entry points keep preparations across calls.  In
 * dvgpu_bn254_pairing_check_prepared term k pairs g1[k] with prepared point
 * q_index[k]; equations and verdicts as dvgpu_bn254_pairing_check. */
int dvgpu_bn254_g2_prepare(void* backend, const uint8_t* g2, size_t n, uint64_t* prepared, char* error,
                           size_t error_capacity);
int dvgpu_bn254_g2_prepared_release(void* backend, uint64_t prepared, char* error, size_t error_capacity);
int dvgpu_bn254_pairing_check_prepared(void* backend, const uint8_t* g1, uint64_t prepared, const uint32_t* q_index,
                                       const uint64_t* offsets, size_t equations, uint8_t* verdicts, char* error,
                                       size_t error_capacity);

/* ---------------------------------------------------------------- polynomial toolkit
 * The field work of a sparse update (crates/protocol/src/domain/fast.rs,
 * called from crates/protocol/src/dynaverse/sparse.rs:125-236), which the
 * reference runs on the host with every product routed through
 * OperatorBackend::ntt.  Polynomials are canonical Fr coefficient vectors,
 * lowest degree first; results are trimmed as the reference's trim()
 * (crates/protocol/src/domain.rs:339-346): no trailing zero coefficient,
 * at least one entry.  Non-canonical inputs and the reference's error
 * conditions return -1 with the reference's message. */

/* fft_multiply_with_backend (domain/fast.rs:213-234): result_capacity >=
 * max(1, left_len + right_len - 1) <= 2^24; an empty operand gives [0]. */
int dvgpu_bn254_poly_multiply(void* backend, const uint8_t* left, size_t left_len, const uint8_t* right,
                              size_t right_len, uint8_t* result, size_t result_capacity, size_t* result_len,
                              char* error, size_t error_capacity);
/* newton_divide_exact_with_backend (domain/fast.rs:236-240, div_rem_impl
 * :163-202): the quotient of an exact division; quotient_capacity >=
 * max(1, numerator_len).  Errors: "cannot divide by zero polynomial",
 * "polynomial division has a nonzero remainder". */
int dvgpu_bn254_poly_divide_exact(void* backend, const uint8_t* numerator, size_t numerator_len,
                                  const uint8_t* denominator, size_t denominator_len, uint8_t* quotient,
                                  size_t quotient_capacity, size_t* quotient_len, char* error, size_t error_capacity);
/* SubproductTree::new_with_backend (domain/fast.rs:18-62) over `count`
 * <= 2^20 distinct points, kept on the device under a handle.  A repeated
 * point: -1 "duplicate interpolation point". */
int dvgpu_bn254_tree_create(void* backend, const uint8_t* points, size_t count, uint64_t* tree, char* error,
                            size_t error_capacity);
int dvgpu_bn254_tree_destroy(void* backend, uint64_t tree, char* error, size_t error_capacity);
/* vanishing() (fast.rs:64): prod (X - x_i), count + 1 coefficients. */
int dvgpu_bn254_tree_vanishing(void* backend, uint64_t tree, uint8_t* coefficients, size_t capacity, size_t* length,
                               char* error, size_t error_capacity);
/* inverse_derivatives() (fast.rs:67): 1 / A'(x_i) in point order. */
int dvgpu_bn254_tree_inverse_derivatives(void* backend, uint64_t tree, uint8_t* values, size_t capacity, char* error,
                                         size_t error_capacity);
/* multipoint_eval_with_backend (fast.rs:22-24, 73-84) of `rows` (<= 65535)
 * polynomials of `length` coefficients each: rows x count values. */
int dvgpu_bn254_tree_evaluate(void* backend, uint64_t tree, const uint8_t* polynomials, size_t length, size_t rows,
                              uint8_t* values, char* error, size_t error_capacity);
/* interpolate_with_backend (fast.rs:26-28, 90-116) of `rows` value vectors
 * of `count` (= the tree's points) entries: row r's coefficients at
 * coefficients + 32 * r * max(1, count), its trimmed length in lengths[r]. */
int dvgpu_bn254_tree_interpolate(void* backend, uint64_t tree, const uint8_t* values, size_t count, size_t rows,
                                 uint8_t* coefficients, size_t* lengths, char* error, size_t error_capacity);
/* cauchy_sums_with_backend (fast.rs:30-32, 118-139): sum_{j != i}
 * w_j / (x_i - x_j) for `rows` weight vectors of `count` entries. */
int dvgpu_bn254_tree_cauchy_sums(void* backend, uint64_t tree, const uint8_t* weights, size_t count, size_t rows,
                                 uint8_t* sums, char* error, size_t error_capacity);

/* ---------------------------------------------------------------- resident buffers
 * The reference's resident ABI (native/include/dynaverse_gpu.h:100-160,
 * bound by crates/gpu/src/resident.rs:81-92; semantics of
 * CpuRebuildBackend, crates/protocol/src/incremental_rebuild/operators.rs):
 * owner-local buffers of Fr (kind 0) or G1 (kind 1) elements, allocated
 * zero / infinity before dvgpu_resident_seal; after sealing only writable
 * buffers (ALLOC flags bit 0) accept writes.  ALLOC_BASES registers
 * immutable affine MSM bases (kind 2), accepted only by READ and MSM_G1.
 * BEGIN opens a transaction; the first write to an element saves its old
 * value in the device journal (journal_bytes, 144 bytes per saved element);
 * ROLLBACK restores every saved element; dvgpu_resident_commit publishes.
 * Field use per opcode, as the reference binding sets them:
 *   ALLOC kind,length,flags -> handle | LENGTH a | KIND a
 *   WRITE/READ kind,a,a_offset,length,input/output (READ flags: 0 or 1)
 *   COPY a,a_offset -> c,c_offset,length | REVERSE kind, same fields
 *   TRANSPOSE kind,a -> c,rows,cols,a_offset = start,length,flags bit 0 with
 *     input = root: element i -> (i % cols) rows + i / cols, times root^(row col)
 *   TRANSFORM kind,a -> c,cols = row length,rows,a_offset = first row,
 *     flags bit 0 = inverse (Fr NTT rows or G1 transform rows)
 *   TRANSFORM_PACKET kind,a -> c (b scratch),length <= 4096,flags = inverse
 *   ZIP flags 0 add / 1 sub / 2 mul, a,a_offset,b,b_offset -> c,c_offset,length
 *   SCALE a points,a_offset x b scalars,b_offset -> c,c_offset,length
 *   MSM_G1 a points,a_offset, b scalars,b_offset,length -> output 64 bytes
 *   MSM_G2 input = length host G2 bases, b scalars,b_offset -> output 128 bytes
 * Handles carry an owner tag; handles of other owners are rejected.
 * configure: memory_limit_bytes caps device bytes (journal included); root
 * must have multiplicative order exactly 2^20. */
enum DvgpuResidentOpcode {
    DVGPU_RESIDENT_ALLOC = 1, DVGPU_RESIDENT_LENGTH, DVGPU_RESIDENT_KIND,
    DVGPU_RESIDENT_BEGIN, DVGPU_RESIDENT_ROLLBACK, DVGPU_RESIDENT_WRITE,
    DVGPU_RESIDENT_READ, DVGPU_RESIDENT_COPY, DVGPU_RESIDENT_REVERSE,
    DVGPU_RESIDENT_TRANSPOSE, DVGPU_RESIDENT_TRANSFORM, DVGPU_RESIDENT_ZIP,
    DVGPU_RESIDENT_SCALE, DVGPU_RESIDENT_MSM_G1, DVGPU_RESIDENT_MSM_G2,
    DVGPU_RESIDENT_ALLOC_BASES, DVGPU_RESIDENT_TRANSFORM_PACKET
};
typedef struct DvgpuResidentOp {
    uint32_t opcode, kind, flags, reserved;
    uint64_t a, b, c;
    uint64_t a_offset, b_offset, c_offset, length, rows, cols;
    const uint8_t* input;
    uint8_t* output;
} DvgpuResidentOp;
typedef struct DvgpuResidentStats {
    uint64_t h2d_bytes, d2h_bytes, bytes_allocated;
    uint64_t fr_transform_elements, g1_transform_elements;
    uint64_t msm_g1_points, msm_g2_points, calls;
} DvgpuResidentStats;
typedef struct DvgpuResidentDiagnostics {
    uint64_t resident_allocations, temporary_allocations, temporary_peak_bytes;
    uint64_t journal_saved_bytes, journal_saved_ranges, journal_peak_bytes;
    uint64_t device_operation_ns, device_operations;
    uint64_t physical_h2d_bytes, physical_d2h_bytes, explicit_d2d_bytes;
    uint64_t journal_metadata_capacity_bytes;
} DvgpuResidentDiagnostics;
int dvgpu_resident_configure(void* backend, uint64_t memory_limit_bytes, uint64_t journal_bytes, const uint8_t* root,
                             char* error, size_t error_capacity);
int dvgpu_resident_call(void* backend, const DvgpuResidentOp* operation, uint64_t* result, char* error,
                        size_t error_capacity);
void dvgpu_resident_seal(void* backend);
void dvgpu_resident_commit(void* backend);
int dvgpu_resident_stats(void* backend, DvgpuResidentStats* stats);
int dvgpu_resident_diagnostics(void* backend, DvgpuResidentDiagnostics* stats);
/* dvgpu_resident_call with its costs (native/include/dynaverse_gpu.h:147-158,
 * bound by crates/gpu/src/resident_profile.rs:40).  native_wall_ns and
 * operation_host_ns: host clock around the call; wait_host_ns: the closing
 * stream synchronisation; journal and conversion host times are inside the
 * operation (0); event_total_ns: CUDA events around the call on the owner's
 * stream (event_mask 4, total only); h2d / d2h / d2d bytes: this call's
 * change in the owner's resident counters. */
typedef struct DvgpuResidentProfile {
    uint64_t native_wall_ns, journal_host_ns, conversion_host_ns;
    uint64_t operation_host_ns, wait_host_ns;
    uint64_t event_total_ns, event_journal_ns, event_operation_ns, event_mask;
    uint64_t h2d_bytes, d2h_bytes, d2d_bytes;
} DvgpuResidentProfile;
int dvgpu_resident_call_profiled(void* backend, const DvgpuResidentOp* operation, uint64_t* result,
                                 DvgpuResidentProfile* profile, char* error, size_t error_capacity);

/* ---------------------------------------------------------------- batching
 * No counterpart in the reference ABI (its batch path is
 * dvgpu_bn254_msm_batch with next-pow2 padding, icicle_msm.cu:810-880, and
 * one dvgpu_bn254_ntt call per vector, icicle.rs:429-456).
 *
 * dvgpu_bn254_ntt_batch: count transforms of sizes 2^log_sizes[i]
 * (1 <= log <= 24) in ONE persistent launch.  values / results: the
 * transforms' canonical elements concatenated in order (may alias);
 * kinds[i] as in dvgpu_bn254_ntt_ex (NULL = all forward).  The _device form
 * takes device buffers and returns after `stream` has completed. */
int dvgpu_bn254_ntt_batch(void* backend, const uint8_t* values, const uint32_t* log_sizes, const int32_t* kinds,
                          size_t count, uint8_t* results, char* error, size_t error_capacity);
int dvgpu_bn254_ntt_batch_device(void* backend, const uint8_t* d_values, const uint32_t* log_sizes,
                                 const int32_t* kinds, size_t count, uint8_t* d_results, void* stream, char* error,
                                 size_t error_capacity);

/* Batch plans: a fixed workload of G1 MSMs over prefixes of one registered
 * G1 base set (MSM i uses bases [0, msm_sizes[i]) and scalars
 * msm_sizes[0] + ... + msm_sizes[i-1] onwards) plus NTTs of fixed sizes and
 * kinds, captured once into a CUDA graph and replayed per run.  At creation
 * the MSMs are grouped into size classes; the autotuner times candidate
 * window widths per class on random scalars, keeps a table of precomputed
 * window multiples for the best one, then times the bucket partition of the
 * reduction (segment lengths around the default rule; log keys
 * seg_candidates, best_seg) and writes its log (JSON) to log_json.
 * It also times the persistent NTT launch for every pair of tile (2^10,
 * 2^11, 2^12 elements) and register round (radix 2, 4, 8) on the plan's
 * own transforms, requires every candidate's output to equal the first's
 * (a mismatch fails the call) and keeps the fastest (log keys
 * ntt.candidates, ntt.best_tile, ntt.best_radix).  Each class is one launch sequence
 * over all its MSMs; the NTTs are one persistent launch on a parallel
 * branch of the graph.
 *
 * dvgpu_batch_plan_buffers: the plan's device buffers (inputs in request
 * order, outputs in request order: 64-byte affine G1 results, canonical NTT
 * elements).  dvgpu_batch_plan_launch: enqueue one replay on `stream` (NULL:
 * the plan's own stream) and return; dvgpu_batch_plan_check: wait for it and
 * report invalid inputs (-1) of the last replay.  dvgpu_batch_plan_run: host
 * inputs and outputs, copies included, synchronous. */
typedef struct DvgpuBatchPlanBuffers {
    uint8_t* scalars;      /* sum(msm_sizes) x 32 bytes */
    uint8_t* ntt_values;   /* sum(2^ntt_log_sizes) x 32 bytes */
    uint8_t* msm_results;  /* msm_count x 64 bytes */
    uint8_t* ntt_results;  /* sum(2^ntt_log_sizes) x 32 bytes */
    uint64_t scalar_bytes, ntt_bytes, msm_result_bytes;
    uint32_t msm_classes, graph_nodes, graph_kernels, reserved;
} DvgpuBatchPlanBuffers;
int dvgpu_batch_plan_create(void* backend, uint64_t bases_handle, const uint64_t* msm_sizes, size_t msm_count,
                            const uint32_t* ntt_log_sizes, const int32_t* ntt_kinds, size_t ntt_count,
                            uint64_t* plan, char* log_json, size_t log_capacity, char* error, size_t error_capacity);
int dvgpu_batch_plan_buffers(void* backend, uint64_t plan, DvgpuBatchPlanBuffers* out, char* error,
                             size_t error_capacity);
int dvgpu_batch_plan_launch(void* backend, uint64_t plan, void* stream, char* error, size_t error_capacity);
int dvgpu_batch_plan_check(void* backend, uint64_t plan, char* error, size_t error_capacity);
int dvgpu_batch_plan_run(void* backend, uint64_t plan, const uint8_t* scalars, const uint8_t* ntt_values,
                         uint8_t* msm_results, uint8_t* ntt_results, char* error, size_t error_capacity);
int dvgpu_batch_plan_destroy(void* backend, uint64_t plan, char* error, size_t error_capacity);

/* ---------------------------------------------------------------- serving
 * No counterpart in the reference ABI: the reference serves updates one
 * call at a time per session (crates/protocol/src/session.rs:51-142).
 *
 * A server keeps sessions resident -- SRS bases (G1 wire form in), the
 * committed vector of canonical Fr values, its commitment C = sum v_i G_i
 * and a table of 32 precomputed window multiples per base -- and admits a
 * session only while the resident bytes (n x (64 x 33 + 32) + 64 per
 * session) stay within hbm_budget_bytes (-1 otherwise).
 * dvgpu_serve_submit queues a commitment update of a session: the entries
 * at `indices` (distinct, < n) take the new `values`; the result is the new
 * commitment C' = C + sum (v'_i - v_i) G_i.  One engine thread merges the
 * pending requests of up to max_batch sessions into shared launches (one
 * per session per batch; a session's requests complete in order), and
 * requests arriving meanwhile form the next batch.  max_batch = 1 is the
 * per-call form.  dvgpu_serve_wait blocks until a ticket completes and
 * returns its commitment and timings (steady-clock nanoseconds).  The
 * server uses device 0 and its own stream and workspaces. */
typedef struct DvgpuServeResult {
    uint64_t submit_ns, start_ns, done_ns;
    uint32_t batch_requests, batch_id;
} DvgpuServeResult;
typedef struct DvgpuServeStats {
    uint64_t requests, batches, sessions, resident_bytes, budget_bytes;
    uint64_t max_batch, largest_batch, busy_ns, pending;
} DvgpuServeStats;
int dvgpu_serve_create(uint64_t hbm_budget_bytes, uint32_t max_batch, void** server, char* error,
                       size_t error_capacity);
void dvgpu_serve_destroy(void* server);
int dvgpu_serve_open_session(void* server, const uint8_t* srs_g1, const uint8_t* values, size_t n, uint64_t* session,
                             uint8_t* commitment, char* error, size_t error_capacity);
int dvgpu_serve_close_session(void* server, uint64_t session, char* error, size_t error_capacity);
int dvgpu_serve_submit(void* server, uint64_t session, const uint64_t* indices, const uint8_t* values, size_t k,
                       uint64_t* ticket, char* error, size_t error_capacity);
int dvgpu_serve_wait(void* server, uint64_t ticket, uint8_t* commitment, DvgpuServeResult* result, char* error,
                     size_t error_capacity);
int dvgpu_serve_set_max_batch(void* server, uint32_t max_batch);
int dvgpu_serve_stats(void* server, DvgpuServeStats* out);

/* ---------------------------------------------------------------- Dynaverse update proofs
 * The prover of crates/protocol/src/dynaverse: DynaverseParams (setup from
 * the two trapdoors, dynaverse.rs:104-147 over srs.rs:147-197),
 * UpdateSession (dynaverse/session.rs:17-142: start_update_session,
 * update_with_public_inputs, including the synchronous re-anchor of
 * update_proof_backend, dynaverse.rs:379-470), and
 * DynaverseVerifyingKey::verify (dynaverse.rs:978-1016), with the whole
 * proof composed on the device.  In the reference this is Rust host code
 * that calls OperatorBackend once per MSM (about 70 calls per sparse
 * update); these entry points replace that loop.
 *
 * Values are 32-byte canonical little-endian Fr; a witness holds 6n wires,
 * an instance n public inputs (ToyCircuit, toy_circuit.rs).  A proof is
 * DVGPU_DYNAVERSE_PROOF_BYTES: the AnchorProof fields (3968 B), the
 * DeltaProof fields (5312 B, zero when absent), then u64 has_delta,
 * anchor_generation, generation (little-endian); every field in the
 * declaration order of types.rs:64-172, G1 64 B and G2 128 B in the wire
 * format (infinity all zero).
 *
 * An engine owns a worker thread, a stream and workspaces on the calling
 * thread's current device.  Parameters and sessions are admitted against
 * its HBM budget (-1 when they do not fit).  dvgpu_dynaverse_submit queues
 * an update (witness edits and public-input edits, session.rs:39-41) and
 * returns a ticket; the worker merges the pending updates of up to
 * max_batch sessions (one per session per batch, in submission order) into
 * shared launches and verifies every proof on the device before it is
 * published; requests arriving meanwhile form the next batch.
 * dvgpu_dynaverse_wait returns the proof, or -1 with the reference's error
 * text for an invalid update (the session is then unchanged).
 * dvgpu_dynaverse_update is submit + wait (with max_batch = 1, the per-call
 * form).  n: a power of two in 1..2^17. */
#define DVGPU_DYNAVERSE_PROOF_BYTES 9304
typedef struct DvgpuDynaverseParamsInfo {
    uint64_t n, m, rebuild_interval, resident_bytes;
    uint8_t g1_generator[64];
    uint8_t multiplication_vanishing_g1[64];
    /* the verifying key's G2 points: u, [x^m - 1], x, 1/m, [y^m - 1], y^m,
     * x^m, x^2, [1], z_in of the six slices, x - y, x - y^(m/n), I_x, x^n - 1 */
    uint8_t vk_g2[19][128];
} DvgpuDynaverseParamsInfo;
typedef struct DvgpuDynaverseResult {
    uint64_t submit_ns, start_ns, done_ns; /* steady-clock nanoseconds */
    uint32_t batch_requests, batch_id;
    uint32_t rebuilt; /* 1: the update re-anchored (delta reached ceil(sqrt(n))) */
    uint32_t pad;
} DvgpuDynaverseResult;
typedef struct DvgpuDynaverseStats {
    uint64_t requests, batches, sessions, resident_bytes, budget_bytes;
    uint64_t max_batch, largest_batch, busy_ns, pending;
    uint64_t sparse_proofs, rebuilds, launches;
    /* algorithmic G1 field multiplications of every MSM run (min over c of
     * ceil(254/c) (10 k + 14 2^c) per k-term set, x3 for G2 sets) */
    uint64_t msm_fme;
    /* of busy_ns: host time (staging, checks, publishing) and time blocked
     * on the device */
    uint64_t host_ns, device_wait_ns;
    /* the bucket accumulation of the dense MSMs (anchor openings and
     * re-anchor quotients), timed by CUDA events on its stream, and its
     * XYZZ mixed additions (terms x 16 windows) */
    uint64_t dense_accum_ns, dense_accum_adds;
    /* device and pinned-host allocations made while serving (growth of the
     * engine's grow-only workspaces) */
    uint64_t allocations, allocation_ns;
    /* host time from a batch's first launch to its synchronisation (the
     * enqueue phase, which allocation inside it lengthens) */
    uint64_t enqueue_ns;
    /* the slowest single allocation of the library so far: nanoseconds,
     * bytes, 1 if pinned host memory */
    uint64_t slowest_alloc_ns, slowest_alloc_bytes, slowest_alloc_pinned;
} DvgpuDynaverseStats;
int dvgpu_dynaverse_create(uint64_t hbm_budget_bytes, uint32_t max_batch, void** engine, char* error,
                           size_t error_capacity);
void dvgpu_dynaverse_destroy(void* engine);
/* SRS, window tables and verifying key of ToyCircuit(n) from the trapdoors
 * tau_x, tau_y (canonical Fr; rejected as in srs.rs:158-178). */
int dvgpu_dynaverse_params_create(void* engine, size_t n, const uint8_t* tau_x, const uint8_t* tau_y,
                                  uint64_t* params, char* error, size_t error_capacity);
int dvgpu_dynaverse_params_destroy(void* engine, uint64_t params, char* error, size_t error_capacity);
int dvgpu_dynaverse_params_info(void* engine, uint64_t params, DvgpuDynaverseParamsInfo* info, char* error,
                                size_t error_capacity);
/* start_update_session: the anchor proof of (public_inputs, witness),
 * verified, written to proof. */
int dvgpu_dynaverse_session_open(void* engine, uint64_t params, const uint8_t* public_inputs, const uint8_t* witness,
                                 uint64_t* session, uint8_t* proof, char* error, size_t error_capacity);
int dvgpu_dynaverse_session_close(void* engine, uint64_t session, char* error, size_t error_capacity);
/* The session's current witness (6n), instance (n), proof and anchor
 * distance (UpdateSession::current_witness / current_instance / proof /
 * anchor_distance); any output may be NULL. */
int dvgpu_dynaverse_session_state(void* engine, uint64_t session, uint8_t* witness, uint8_t* public_inputs,
                                  uint8_t* proof, uint64_t* anchor_distance, char* error, size_t error_capacity);
int dvgpu_dynaverse_submit(void* engine, uint64_t session, const uint64_t* indices, const uint8_t* values,
                           size_t count, const uint64_t* public_indices, const uint8_t* public_values,
                           size_t public_count, uint64_t* ticket, char* error, size_t error_capacity);
int dvgpu_dynaverse_wait(void* engine, uint64_t ticket, uint8_t* proof, DvgpuDynaverseResult* result, char* error,
                         size_t error_capacity);
int dvgpu_dynaverse_update(void* engine, uint64_t session, const uint64_t* indices, const uint8_t* values,
                           size_t count, const uint64_t* public_indices, const uint8_t* public_values,
                           size_t public_count, uint8_t* proof, char* error, size_t error_capacity);
/* accepted = 1 iff the proof parses and passes every check of verify. */
int dvgpu_dynaverse_verify(void* engine, uint64_t params, const uint8_t* public_inputs, const uint8_t* proof,
                           uint8_t* accepted, char* error, size_t error_capacity);
int dvgpu_dynaverse_set_max_batch(void* engine, uint32_t max_batch);
int dvgpu_dynaverse_stats(void* engine, DvgpuDynaverseStats* out);

#ifdef __cplusplus
}
#endif
