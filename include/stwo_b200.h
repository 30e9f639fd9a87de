/*
 * stwo_b200 — Blackwell-native (sm_100a) CUDA backend for the Stwo circle-STARK
 * prover's hot path: M31 circle FFT, FRI folds, DEEP quotients, batch inverse,
 * Blake2s Merkle commitment, accumulation and the wide-Fibonacci composition.
 *
 * Two tiers of `extern "C"` entry points are exported by libstwo_b200.so:
 *
 *  1. Reference-compatible entry points. Their names, argument order and
 *     argument meaning are exactly those the reference's Rust FFI binds
 *     (NethermindEth/stwo-gpu, stwo_gpu_backend/src/cuda/bindings.rs:75-271), so
 *     the reference's trait impls link against this library unchanged. Like the
 *     reference they run on the legacy default stream and return after the work
 *     is done. Failures are recorded for stwo_last_error() instead of printed.
 *
 *  2. Native entry points (stwo_*): asynchronous on a caller-supplied CUDA stream
 *     (a cudaStream_t passed as void*, NULL = legacy default stream), returning a
 *     status code (STWO_OK = 0). They take host arrays of device column pointers
 *     (passed to the kernels by value, so the calls are CUDA-graph capturable),
 *     accept columns of mixed power-of-two sizes where the reference assumed one
 *     size, and fuse steps the reference ran as separate passes.
 *
 * Conventions. An M31 element is a uint32_t in [0, 2^31 - 1). A QM31 value is
 * stwo_qm31 {a, b, c, d} = (a + b i) + (c + d i) u, the reference's repr(C)
 * CudaSecureField (bindings.rs:8-14). "SoA QM31 columns" are four M31 device
 * arrays (SecureColumnByCoords); "AoS QM31" is 16 contiguous bytes per element
 * (SecureFieldVec). Evaluations are in bit-reversed order. Twiddle trees are the
 * layout PolyOps::precompute_twiddles produces (twiddles.cu:29-73): the layers
 * of the root coset's doublings, concatenated, followed by a single 1.
 */
#ifndef STWO_B200_H
#define STWO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- types */
typedef struct { uint32_t x, y; } stwo_point;          /* CirclePointBaseField, bindings.rs:45-58 */
typedef struct { uint32_t a, b, c, d; } stwo_qm31;      /* CudaSecureField, bindings.rs:8-14 */
typedef struct { stwo_qm31 x, y; } stwo_spoint;         /* CirclePointSecureField, bindings.rs:60-73 */
typedef struct { uint32_t s[8]; } stwo_blake2s_hash;    /* Blake2sHash, cuda/include/utils.cuh:7-9 */

enum {
    STWO_OK = 0,
    STWO_ERR_INVALID_ARGUMENT = 1,
    STWO_ERR_UNSUPPORTED_SIZE = 2,
    STWO_ERR_OUT_OF_MEMORY = 3,
    STWO_ERR_CUDA = 4,
    STWO_ERR_CANCELLED = 5,  /* a queued server job removed by stwo_server_cancel */
    STWO_ERR_TIMEOUT = 6,    /* a server job that waited in the queue past its limit */
};

/* =====================================================================
 * Tier 1: reference-compatible entry points (bindings.rs:75-271)
 * ===================================================================== */

/* Device memory and copies. Replaces cuda/src/utils.cu:14-80 (bindings.rs:77-99,196-216). */
void copy_uint32_t_vec_from_device_to_host(const uint32_t *device_ptr, uint32_t *host_ptr, uint32_t size);
uint32_t *copy_uint32_t_vec_from_host_to_device(const uint32_t *host_ptr, uint32_t size);
uint32_t *copy_uint32_t_vec_from_device_to_device(const uint32_t *from, uint32_t *dst, uint32_t size);
uint32_t *cuda_malloc_uint32_t(uint32_t size);
stwo_blake2s_hash *cuda_malloc_blake_2s_hash(size_t size);
uint32_t *cuda_alloc_zeroes_uint32_t(uint32_t size);
stwo_blake2s_hash *cuda_alloc_zeroes_blake_2s_hash(size_t size);
void cuda_free_memory(void *device_ptr);
stwo_blake2s_hash *copy_blake_2s_hash_vec_from_host_to_device(const stwo_blake2s_hash *from, size_t size);
void copy_blake_2s_hash_vec_from_device_to_host(const stwo_blake2s_hash *from, stwo_blake2s_hash *to, size_t size);
void copy_blake_2s_hash_vec_from_device_to_device(const stwo_blake2s_hash *from, stwo_blake2s_hash *dst, size_t size);
uint32_t **copy_device_pointer_vec_from_host_to_device(uint32_t *const *from, size_t size);

/* ColumnOps::bit_reverse_column. Replaces cuda/src/bit_reverse.cu:18-33 (bindings.rs:101-103). */
void bit_reverse_base_field(uint32_t *array, size_t size);
void bit_reverse_secure_field(uint32_t *array, size_t size);

/* FieldOps::batch_inverse. Replaces cuda/src/batch_inverse.cu:157-177 (bindings.rs:105-107). */
void batch_inverse_base_field(const uint32_t *from, uint32_t *dst, size_t size);
void batch_inverse_secure_field(const uint32_t *from, uint32_t *dst, size_t size);

/* PolyOps::new_canonical_ordered. Replaces cuda/src/poly/twiddles.cu:17-27 (bindings.rs:109-112).
 * Returns a new device buffer owned by the caller (free with cuda_free_memory). */
uint32_t *sort_values_and_permute_with_bit_reverse_order(const uint32_t *from, size_t size);

/* PolyOps::precompute_twiddles. Replaces cuda/src/poly/twiddles.cu:50-73 (bindings.rs:114-118).
 * Returns a new device buffer of total_size twiddles owned by the caller. */
uint32_t *precompute_twiddles(stwo_point initial, stwo_point step, size_t total_size);

/* PolyOps::interpolate / interpolate_columns / evaluate / evaluate_polynomials.
 * Replace cuda/src/poly/ifft.cu:41-163 and rfft.cu:45-141 (bindings.rs:120-152).
 * eval_domain_size is the domain's half-coset size; values are in place. In
 * interpolate_columns `values` is a host array of `values_size` device column
 * pointers of `number_of_rows` elements; evaluate_columns accepts per-column sizes. */
void interpolate(uint32_t eval_domain_size, uint32_t *values, const uint32_t *inverse_twiddles_tree,
                 uint32_t inverse_twiddle_tree_size, uint32_t values_size);
void interpolate_columns(uint32_t eval_domain_size, uint32_t *const *values, const uint32_t *inverse_twiddles_tree,
                         uint32_t inverse_twiddle_tree_size, uint32_t values_size, uint32_t number_of_rows);
void evaluate(uint32_t eval_domain_size, uint32_t *values, const uint32_t *twiddles_tree,
              uint32_t twiddle_tree_size, uint32_t values_size);
void evaluate_columns(const uint32_t *eval_domain_sizes, uint32_t *const *values, const uint32_t *twiddles_tree,
                      uint32_t twiddle_tree_size, uint32_t number_of_columns, const uint32_t *column_sizes);

/* PolyOps::eval_at_point. Replaces cuda/src/poly/eval_at_point.cu:99-155 (bindings.rs:154-159). */
stwo_qm31 eval_at_point(const uint32_t *coeffs, uint32_t coeffs_size, stwo_qm31 point_x, stwo_qm31 point_y);

/* FriOps::fold_line / fold_circle_into_line. Replace cuda/src/fri/fold_line.cu:36-53 and
 * fold_circle_into_line.cu:48-69 (bindings.rs:161-177). gpu_domain is the itwiddles tree,
 * eval_values / folded_values are host arrays of the 4 SoA coordinate columns. */
void fold_line(const uint32_t *gpu_domain, size_t twiddle_offset, size_t n, uint32_t *const *eval_values,
               stwo_qm31 alpha, uint32_t *const *folded_values);
void fold_circle_into_line(const uint32_t *gpu_domain, size_t twiddle_offset, size_t n, uint32_t *const *eval_values,
                           stwo_qm31 alpha, uint32_t *const *folded_values);

/* AccumulationOps::accumulate. Replaces cuda/src/accumulate.cu:15-26 (bindings.rs:179). */
void accumulate(uint32_t size, uint32_t *const *left_columns, uint32_t *const *right_columns);

/* MerkleOps<Blake2sMerkleHasher>::commit_on_layer. Replaces cuda/src/blake2s.cu:157-170
 * (bindings.rs:181-194). `columns` is a DEVICE array of device column pointers. */
void commit_on_first_layer(size_t size, size_t amount_of_columns, uint32_t *const *columns, stwo_blake2s_hash *result);
void commit_on_layer_with_previous(size_t size, size_t amount_of_columns, uint32_t *const *columns,
                                   const stwo_blake2s_hash *previous_layer, stwo_blake2s_hash *result);

/* QuotientOps::accumulate_quotients. Replaces cuda/src/quotients.cu:180-270
 * (bindings.rs:218-236). `columns` is a DEVICE array of device column pointers;
 * sample arrays are host memory; batches may have different sizes. */
void accumulate_quotients(uint32_t half_coset_initial_index, uint32_t half_coset_step_size, uint32_t domain_size,
                          uint32_t *const *columns, size_t number_of_columns, stwo_qm31 random_coeff,
                          const uint32_t *sample_points, const uint32_t *sample_columns_indexes,
                          uint32_t sample_columns_indexes_size, const stwo_qm31 *sample_column_values,
                          const uint32_t *sample_column_and_values_sizes, uint32_t sample_size,
                          uint32_t *result_column_0, uint32_t *result_column_1, uint32_t *result_column_2,
                          uint32_t *result_column_3, uint32_t flattened_line_coeffs_size);

/* Wide-Fibonacci composition (ComponentProver::evaluate_constraint_quotients_on_domain).
 * Replaces cuda/src/examples/wide_fibonacci.cu:40-66 (bindings.rs:260-270).
 * trace_evaluations is a host array of device pointers; random_coeff_powers is a device
 * AoS QM31 array; denominator_inverses a device M31 array (bit-reversed order). */
void evaluate_wide_fibonacci_constraint_quotients_on_domain(
    uint32_t *quotients_0, uint32_t *quotients_1, uint32_t *quotients_2, uint32_t *quotients_3,
    uint32_t *const *trace_evaluations, const uint32_t *random_coeff_powers, const uint32_t *denominator_inverses,
    uint32_t extended_domain_size, uint32_t number_of_columns);

/* =====================================================================
 * Tier 2: native asynchronous entry points
 * ===================================================================== */

/* Message of the last failure on the calling thread ("" if none); the record is
 * sticky until stwo_clear_last_error(). The void reference-compatible entry points
 * report failures only through this record. */
const char *stwo_last_error(void);
void stwo_clear_last_error(void);
/* Grows the library's device memory pool (which keeps what it holds) to at least
 * `bytes`, so allocations up to that total map no new memory later. */
int stwo_reserve_device_memory(uint64_t bytes);
/* Measures the library's launch-parameter variants on the current device (FFT elements
 * per thread per pass kind and size, Merkle layers per launch and bottom-level nodes
 * per thread) and keeps the fastest
 * for this process; every variant computes the same values. Writes a JSON summary of
 * the timings and choices into report (NUL-terminated, at most report_cap bytes) if
 * it is not NULL. Takes well under a second. */
int stwo_autotune(char *report, size_t report_cap);
/* Sets one tunable by name: fft_ept_contig_small / fft_ept_contig_large /
 * fft_ept_strided (5 or 6), merkle_sub_threads (128, 256 or 512), merkle_sub_spread
 * (0..5: log2 of the bottom-level nodes each thread hashes), eval_at_point_groups_log
 * (2..4: log2 of the 8192-coefficient groups each eval_at_point CTA folds; 0, the
 * default, chooses per launch), quotients_tensor_cores (0, 1 = the default, 2) and
 * composition_tensor_cores (0 = the default, 1). */
int stwo_set_tunable(const char *name, int value);
/* Diagnostics (no counterpart in the reference): the integer ceiling of the FFT. One
 * launch runs the FFT passes' own forward butterfly on register-resident operands
 * (16 independent chains a thread, 2048 threads an SM) for `iters` rounds and reports
 * in *butterflies how many it executes; time it on `stream` to get the device's
 * butterfly rate. `sink` is device memory of at least 2048 x SM-count words. */
int stwo_probe_m31_butterflies(uint32_t iters, uint32_t *sink, uint64_t sink_words, uint64_t *butterflies,
                               void *stream);
/* Number of kernel launches the library has made in this process (all threads). */
uint64_t stwo_kernel_launches(void);
/* Waits for all work on `stream`; returns STWO_ERR_CUDA if any of it failed. */
int stwo_stream_synchronize(void *stream);

/* Twiddle tree of the coset {root_initial_index, root_step_size, 2^root_log_size}
 * into twiddles[2^root_log_size] and its element-wise inverse into itwiddles
 * (either output may be NULL). Replaces twiddles.cu:29-73 plus the batch_inverse
 * call of poly.rs:181-186. */
int stwo_precompute_twiddles(uint32_t root_initial_index, uint32_t root_step_size, uint32_t root_log_size,
                             uint32_t *twiddles, uint32_t *itwiddles, void *stream);

/* In-place circle FFTs over columns of mixed sizes; column i has 2^log_sizes[i]
 * elements and its domain's half coset is a doubling of the tree's root coset.
 * Inverse FFTs include the 2^-log rescale.
 * Up to 64 columns travel in the launch parameters. Beyond that, these three
 * calls copy the column table into a pool buffer with a stream-ordered copy from
 * pageable host memory. Such a call may not be recorded into a CUDA graph; the
 * prover's own calls pass a prebuilt device table and stay graph-capturable. */
int stwo_interpolate_columns(uint32_t *const *columns, const uint32_t *log_sizes, uint32_t n_columns,
                             const uint32_t *itwiddles, uint64_t tree_size, void *stream);
int stwo_evaluate_columns(uint32_t *const *columns, const uint32_t *log_sizes, uint32_t n_columns,
                          const uint32_t *twiddles, uint64_t tree_size, void *stream);
/* Fused PolyOps::extend + evaluate: reads 2^coeff_log_sizes[i] coefficients from coeffs[i]
 * and writes the 2^(coeff_log_sizes[i] + log_blowup) evaluations to outputs[i] (distinct
 * buffers); the zero padding is never materialised. */
int stwo_extend_evaluate_columns(const uint32_t *const *coeffs, const uint32_t *coeff_log_sizes,
                                 uint32_t *const *outputs, uint32_t log_blowup, uint32_t n_columns,
                                 const uint32_t *twiddles, uint64_t tree_size, void *stream);

/* ColumnOps / FieldOps. qm31 arrays are AoS. */
int stwo_bit_reverse_m31(uint32_t *column, uint64_t n, void *stream);
int stwo_bit_reverse_qm31(uint32_t *column, uint64_t n, void *stream);
int stwo_new_canonical_ordered(const uint32_t *src, uint32_t *dst, uint32_t log_size, void *stream);
int stwo_batch_inverse_m31(const uint32_t *src, uint32_t *dst, uint64_t n, void *stream);
int stwo_batch_inverse_qm31(const uint32_t *src, uint32_t *dst, uint64_t n, void *stream);
/* (the batch inverses accept src == dst) */

/* PolyOps::eval_at_point for n_polys polynomials, each at its own point; results
 * (device, AoS QM31) in results[i]. `scratch` is caller-owned device memory of at
 * least stwo_eval_at_points_scratch_bytes() bytes (per-block partial sums and
 * completion tickets); concurrent calls need distinct scratch. */
size_t stwo_eval_at_points_scratch_bytes(const uint32_t *log_sizes, uint32_t n_polys);
int stwo_eval_at_points(const uint32_t *const *coeffs, const uint32_t *log_sizes, uint32_t n_polys,
                        const stwo_spoint *points, stwo_qm31 *results, void *scratch, size_t scratch_bytes,
                        void *stream);

/* PolyOps::eval_at_point that allocates nothing. It has no counterpart in the
 * reference (whose eval_at_point mallocs and frees scratch on every call); it is
 * for callers that cannot call cudaMalloc, for example a server whose device memory
 * all belongs to its own pool, or a loop that cannot afford cudaMalloc/cudaFree's
 * implicit synchronisation. The scratch is a fixed 32.5 KiB array inside the library,
 * held on every GPU that loads it until the process exits, so polynomials are
 * limited to 2^26 coefficients (larger sizes return STWO_ERR_UNSUPPORTED_SIZE).
 * result is a device pointer to one QM31; the call is asynchronous on `stream`.
 * The first call on each device looks the array's device address up (make it
 * before any stream capture); after a device reset the first call in the new
 * context looks it up again. All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller. */
int stwo_eval_at_point_no_alloc(const uint32_t *coeffs, uint32_t log_size, stwo_qm31 point_x, stwo_qm31 point_y,
                                stwo_qm31 *result, void *stream);

/* FriOps on SoA QM31 columns; itwiddles + twiddle_offset as in fri.rs:24-26,56. */
int stwo_fold_line(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha, const uint32_t *itwiddles,
                   uint64_t twiddle_offset, uint32_t *const *dst4, void *stream);
int stwo_fold_circle_into_line(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha, const uint32_t *itwiddles,
                               uint64_t twiddle_offset, uint32_t *const *dst4, void *stream);

/* AccumulationOps::accumulate on SoA QM31 columns: left += right. */
int stwo_accumulate(uint32_t *const *left4, const uint32_t *const *right4, uint64_t n, void *stream);

/* One Merkle layer of 2^log_size Blake2s nodes (32 bytes each). prev_layer (2^(log_size+1)
 * nodes) may be NULL for the leaf layer; columns is a host array of device pointers to
 * columns of 2^log_size elements. */
int stwo_merkle_commit_layer(uint32_t log_size, const uint32_t *prev_layer, const uint32_t *const *columns,
                             uint32_t n_columns, uint32_t *out, void *stream);
/* A whole Merkle tree (MerkleProver::commit, blake2s.rs:19-97 driven layer by layer)
 * over columns of mixed power-of-two sizes in one launch instead of one per layer.
 * columns / log_sizes: host arrays of n_columns device column pointers and their log
 * sizes (at most max_log); a layer's columns are hashed in their order in `columns`.
 * layers: host array of max_log + 1 device buffers, layers[l] receiving the 2^l nodes
 * of layer l (16-byte aligned); layers[0] is the root. The column tables and the
 * kernel's tickets are staged through the library's pool with a copy from pageable
 * memory, so the call may not be recorded into a CUDA graph. */
int stwo_merkle_commit_tree(const uint32_t *const *columns, const uint32_t *log_sizes, uint32_t n_columns,
                            uint32_t max_log, uint32_t *const *layers, void *stream);

/* DEEP quotient accumulation over the circle domain with half coset
 * {initial_index, step_size, 2^(domain_log_size-1)}. Batch b samples batch_sizes[b]
 * columns (indices in column_indices, values in sampled_values, flattened) at
 * sample_points[b]. Host arrays; columns is a host array of device pointers; out4 are
 * the four SoA result columns. */
int stwo_accumulate_quotients(uint32_t half_coset_initial_index, uint32_t half_coset_step_size,
                              uint32_t domain_log_size, const uint32_t *const *columns, uint32_t n_columns,
                              stwo_qm31 random_coeff, const stwo_spoint *sample_points, const uint32_t *batch_sizes,
                              const uint32_t *column_indices, const stwo_qm31 *sampled_values, uint32_t n_batches,
                              uint32_t *const *out4, void *stream);
/* Calls of 2..4 batches over at least 2^16 rows (and 64 * n_batches * n_columns <=
 * 65536, columns rounded up to a multiple of 8) are computed on the tensor cores: the
 * batches' column sums as an 8-bit integer matrix product (column bytes x coefficient
 * bytes, 32-bit accumulators in TMEM); other calls on the CUDA cores.
 * stwo_set_tunable("quotients_tensor_cores", v) moves the line: 0 for the CUDA cores
 * always, 2 for the tensor cores wherever the form applies (one batch, and domains
 * down to 2^8 rows). Every choice gives the same values. The tensor-core kernel's
 * barrier waits give up after one second; *count receives how many CTAs gave up since
 * the last reset (0 unless the device misbehaved; their rows are then not written).
 * Synchronises the device. */
int stwo_quotients_tc_faults(uint32_t *count, int reset);

/* Wide-Fibonacci composition: out = den_inv * sum_i (c_i^2 + c_{i+1}^2 - c_{i+2}) * powers[N-3-i].
 * With stwo_set_tunable("composition_tensor_cores", 1), domains of at least 2^7 rows
 * with 3..1024 columns run on the tensor cores (the constraint values' bytes times the
 * weights' bytes, an 8-bit integer matrix product), with the same values; by default
 * (0) all run on the CUDA cores. stwo_composition_tc_faults reports the tensor-core kernel's
 * CTAs that gave up a barrier wait after one second, as stwo_quotients_tc_faults
 * does. */
int stwo_wide_fib_composition(const uint32_t *const *trace, uint32_t n_columns, uint32_t ext_log_size,
                              const stwo_qm31 *coeff_powers, const uint32_t *den_inv, uint32_t *const *out4,
                              void *stream);
int stwo_composition_tc_faults(uint32_t *count, int reset);

/* =====================================================================
 * Tier 3: the wide-Fibonacci STARK prover and the proof server. The reference has
 * no C entry point for these: its prover is stwo's Rust prove() driving CudaBackend
 * (stwo_gpu_backend/src/examples/wide_fibonacci.rs:205-250).
 * ===================================================================== */

/* One wide-Fibonacci proof: the trace has 2^log_n_rows rows of n_columns columns
 * (row r: a0[r], a1[r], then a_{j+2} = a_j^2 + a_{j+1}^2), proved with
 * PcsConfig{pow_bits, FriConfig{log_last_layer_degree_bound = 0, log_blowup, n_queries}}
 * and a Blake2s channel starting from the zero digest. Limits: 3 <= n_columns <= 1024,
 * 1 <= log_blowup <= 4, 2 <= log_n_rows, log_n_rows + 1 + log_blowup <= 27,
 * 1 <= n_queries <= 1024, pow_bits <= 32 (the search gives up after 2^(pow_bits+6) nonces). */
typedef struct {
    uint32_t log_n_rows;
    uint32_t n_columns;
    uint32_t log_blowup;
    uint32_t n_queries;
    uint32_t pow_bits;
} stwo_wide_fib_job;

/* Per-phase host wall-clock times of one proof (each phase ends on a device
 * synchronisation, so device work is included), and what the proof used. */
typedef struct {
    double trace_ms;        /* trace generation, interpolation, evaluation, tree */
    double composition_ms;  /* composition polynomial and its tree */
    double oods_ms;         /* out-of-domain sampling and the constraint check */
    double fri_ms;          /* DEEP quotients and the FRI commitment */
    double decommit_ms;     /* proof of work, queries, decommitments, serialisation */
    double total_ms;
    uint64_t device_bytes;    /* device memory the proof allocated */
    uint64_t kernel_launches; /* kernels it launched */
    uint64_t proof_bytes;
} stwo_prove_stats;

/* Upper bound of the device bytes stwo_wide_fib_prove allocates for `job` (0 if the
 * job is unsupported); with_own_twiddles: the call builds its own twiddle tree. */
uint64_t stwo_wide_fib_prove_device_bytes(const stwo_wide_fib_job *job, int with_own_twiddles);

/* Proves one job on `stream`. a0, a1: the first two trace columns, 2^log_n_rows M31
 * values each, in host or device memory. twiddles/itwiddles: NULL, or a tree of
 * tree_size entries for the half coset of a canonic domain of log size at least
 * log_n_rows + 1 + log_blowup (stwo_precompute_twiddles). On success *proof is a
 * malloc'd buffer of *proof_len bytes (free with stwo_free_proof): the
 * CommitmentSchemeProof fields in declaration order, little endian, vectors prefixed
 * by a u64 length. stats may be NULL. Blocks the calling thread until the proof is
 * done; calls on distinct streams from distinct threads run concurrently. */
int stwo_wide_fib_prove(const stwo_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1,
                        const uint32_t *twiddles, const uint32_t *itwiddles, uint64_t tree_size, uint8_t **proof,
                        uint64_t *proof_len, stwo_prove_stats *stats, void *stream);
void stwo_free_proof(uint8_t *proof);

/* n_jobs proofs of one job shape in one launch sequence (no counterpart in the
 * reference): every kernel of the proof is launched once for all of them, job k's
 * device memory being job 0's moved by one job's bound. a0[k], a1[k]: job k's first
 * two trace columns (host or device). Needs the caller's twiddle tree; n_jobs <= 256,
 * and the device memory of n_jobs jobs (n_jobs x stwo_wide_fib_prove_device_bytes).
 * proofs[k] / proof_lens[k] receive job k's malloc'd proof (free with
 * stwo_free_proof; NULL for a job that failed) and job_status[k] its status; the
 * call's own status reports the launch sequence. The proofs are byte for byte those
 * of stwo_wide_fib_prove. stats (may be NULL) describes the whole sequence. */
int stwo_wide_fib_prove_batch(const stwo_wide_fib_job *job, uint32_t n_jobs, const uint32_t *const *a0,
                              const uint32_t *const *a1, const uint32_t *twiddles, const uint32_t *itwiddles,
                              uint64_t tree_size, uint8_t **proofs, uint64_t *proof_lens, int *job_status,
                              stwo_prove_stats *stats, void *stream);

/* Repeated proofs of one job shape (no counterpart in the reference). A cache keeps
 * the device memory of its last proof; the next stwo_wide_fib_prove_cached call with
 * the same shape, twiddle tree and device reuses it, every buffer at the same address,
 * so the proof's launch sequence (trace to query words) is captured as a CUDA graph on
 * that second call and replayed with one launch from the third on. A call with a
 * different shape, or after any stwo_set_tunable / stwo_autotune, frees the memory
 * first and starts over. Needs the caller's twiddle tree; jobs with
 * log_n_rows < 3 are proved without reuse, and on the legacy default stream (NULL) the
 * memory is reused but no graph is captured. A cache serves one thread and one stream
 * at a time; it holds up to stwo_wide_fib_prove_device_bytes(job, 0) bytes between
 * calls (stwo_prove_cache_stats). destroy frees them, stream-ordered on `stream`. */
typedef struct stwo_prove_cache stwo_prove_cache;
stwo_prove_cache *stwo_prove_cache_create(void);
int stwo_wide_fib_prove_cached(stwo_prove_cache *cache, const stwo_wide_fib_job *job, const uint32_t *a0,
                               const uint32_t *a1, const uint32_t *twiddles, const uint32_t *itwiddles,
                               uint64_t tree_size, uint8_t **proof, uint64_t *proof_len, stwo_prove_stats *stats,
                               void *stream);
void stwo_prove_cache_stats(const stwo_prove_cache *cache, uint64_t *device_bytes, uint64_t *graph_replays);
void stwo_prove_cache_destroy(stwo_prove_cache *cache, void *stream);

/* Proof server on the current device: n_workers jobs in flight at most, admitted in
 * arrival order while their device bound fits device_budget_bytes (smaller later jobs
 * pass a job that does not fit), each on its own stream; one shared twiddle tree for
 * domains up to log size max_domain_log. */
typedef struct stwo_prover_server stwo_prover_server;

typedef struct {
    uint64_t job_id;
    int status;          /* STWO_OK or the prover's error status */
    char error[256];     /* the error message when status != STWO_OK */
    uint8_t *proof;      /* malloc'd proof bytes (free with stwo_free_proof), NULL on error */
    uint64_t proof_len;
    double submit_ms, start_ms, done_ms; /* stwo_server_now_ms() clock */
    double device_done_ms; /* device time at which the job's last GPU operation ended, in ms
                              after the server's last stwo_server_mark_epoch(); -1 before any */
    stwo_prove_stats stats;
} stwo_server_result;

stwo_prover_server *stwo_server_create(uint32_t n_workers, uint64_t device_budget_bytes, uint32_t max_domain_log);
/* Queues a job (a0, a1 are host arrays, copied before the call returns). Fails when
 * the job is unsupported or can never fit the budget. */
int stwo_server_submit(stwo_prover_server *server, uint64_t job_id, const stwo_wide_fib_job *job, const uint32_t *a0,
                       const uint32_t *a1);
/* Queues a job whose inputs are already in device memory; the caller keeps a0_dev and
 * a1_dev valid until the job's result has been polled. */
int stwo_server_submit_device(stwo_prover_server *server, uint64_t job_id, const stwo_wide_fib_job *job,
                              const uint32_t *a0_dev, const uint32_t *a1_dev);
/* Moves up to max_results finished jobs into out and returns their number. Waits up to
 * timeout_ms for one (negative: until one finishes or nothing is queued or running). */
uint32_t stwo_server_poll(stwo_prover_server *server, stwo_server_result *out, uint32_t max_results,
                          int32_t timeout_ms);
void stwo_server_stats(stwo_prover_server *server, uint32_t *pending, uint32_t *running,
                       uint64_t *device_bytes_in_use);
/* Same-shape reuse so far: proofs that ran on a worker's retained slab (a queued job
 * with the shape of the worker's previous job takes its place at once), and of those
 * the proofs that replayed the captured launch sequence as one CUDA graph (all but
 * the first reuse of a slab). Off with STWO_SERVER_GRAPHS=0 at creation. */
void stwo_server_graph_stats(stwo_prover_server *server, uint64_t *slab_reuses, uint64_t *graph_replays);
/* Batches so far: launch sequences that proved several queued jobs of one shape at
 * once (stwo_wide_fib_prove_batch), and the jobs they proved. A worker that takes a
 * job of at most 2^16 trace rows also takes the queued jobs of its shape that
 * arrival-order admission would take next, up to 32 a batch (STWO_SERVER_BATCH: the
 * most, 1 for none; STWO_SERVER_BATCH_MAX_LOG: the largest log_n_rows, at creation). */
void stwo_server_batch_stats(stwo_prover_server *server, uint64_t *batches, uint64_t *batched_jobs);
double stwo_server_now_ms(void);
/* Records the server's device epoch now (on an idle stream of its own) and waits for
 * it: later results carry device_done_ms relative to it, so the device-side span of a
 * batch submitted after the mark is the largest device_done_ms of its results. */
int stwo_server_mark_epoch(stwo_prover_server *server);
/* Drops queued jobs, waits for running ones, frees everything (including unpolled proofs). */
void stwo_server_destroy(stwo_prover_server *server);
/* Removes a job that is still queued: its result (status STWO_ERR_CANCELLED) is
 * posted for stwo_server_poll. A job that is already running cannot be cancelled (its
 * kernels are in flight on its stream); it finishes normally. Returns
 * STWO_ERR_INVALID_ARGUMENT when no queued job has that id. */
int stwo_server_cancel(stwo_prover_server *server, uint64_t job_id);
/* paused != 0: workers start no queued job (running jobs finish; submissions are
 * still accepted and queue timeouts still apply); paused == 0: they resume, taking the
 * queue in arrival order. Holding the queue while a burst of jobs is submitted admits
 * the burst at once, so that jobs of one shape are proved in full batches. */
int stwo_server_pause(stwo_prover_server *server, int paused);
/* Jobs that wait in the queue longer than queue_timeout_ms (0: no limit, the default)
 * are not started: their result carries STWO_ERR_TIMEOUT. Checked whenever a worker
 * looks for work and while stwo_server_poll waits. */
int stwo_server_set_queue_timeout(stwo_prover_server *server, double queue_timeout_ms);
/* Test hook: the next n device allocations from the library's pool fail with
 * STWO_ERR_OUT_OF_MEMORY as if the device were full (the allocation call is not made),
 * so tests can check that a server job fails alone and the server carries on. */
void stwo_debug_fail_allocations(uint32_t n);

#ifdef __cplusplus
}
#endif
#endif /* STWO_B200_H */
