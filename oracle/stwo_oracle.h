/*
 * CPU oracle for the Stwo circle-STARK hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of what stwo's CpuBackend (stwo-prover git rev
 * ce5b975, the dependency named in stwo_gpu_backend/Cargo.toml:8, not vendored)
 * computes for each backend-trait method the GPU path implements. Its behaviour
 * is taken from the reference's CUDA kernels and the Rust tests that assert those
 * kernels equal CpuBackend (file:line cited per function in stwo_oracle.c).
 *
 * Only the test suite, the smoke check and the CPU-baseline leg of the benchmark
 * may load this library, and only as the checker. The product path never links it.
 *
 * All arithmetic is exact modulo p = 2^31 - 1 and every value is kept canonical
 * (in [0, p)).
 */
#ifndef STWO_ORACLE_H
#define STWO_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint32_t m31_t;
typedef struct { m31_t a, b; } cm31_t;           /* a + b*i,  i^2 = -1        */
typedef struct { cm31_t a, b; } qm31_t;          /* a + b*u,  u^2 = 2 + i     */
typedef struct { m31_t x, y; } cpoint_t;         /* point on x^2 + y^2 = 1    */
typedef struct { qm31_t x, y; } spoint_t;        /* point over QM31           */
typedef struct { uint32_t initial_index, step_size, log_size; } coset_t;

/* ---- field ---- */
m31_t  or_m31_mul(m31_t a, m31_t b);
m31_t  or_m31_inv(m31_t a);
qm31_t or_qm31_mul(qm31_t a, qm31_t b);
qm31_t or_qm31_inv(qm31_t a);
qm31_t or_qm31_pow(qm31_t a, uint64_t e);

/* ---- circle ---- */
cpoint_t or_index_to_point(uint32_t index);
cpoint_t or_coset_at(coset_t c, uint64_t i);
cpoint_t or_circle_domain_at(coset_t half_coset, uint64_t i);
uint32_t or_bit_reverse_index(uint32_t i, uint32_t log_size);
coset_t  or_canonic_half_coset(uint32_t domain_log_size);
coset_t  or_canonic_coset(uint32_t log_size);

/* ---- ColumnOps / FieldOps ---- */
void or_bit_reverse_u32(uint32_t *v, size_t n);
void or_bit_reverse_qm31(qm31_t *v, size_t n);
void or_batch_inverse_m31(const m31_t *src, m31_t *dst, size_t n);
void or_batch_inverse_qm31(const qm31_t *src, qm31_t *dst, size_t n);

/* ---- PolyOps ---- */
void or_precompute_twiddles(coset_t root, m31_t *twiddles, m31_t *itwiddles);
void or_new_canonical_ordered(uint32_t log_size, const m31_t *src, m31_t *dst);
int  or_interpolate(coset_t half_coset, m31_t *values, const m31_t *itwiddles, size_t tree_size);
int  or_evaluate(coset_t half_coset, m31_t *values, const m31_t *twiddles, size_t tree_size);
void or_evaluate_direct(coset_t half_coset, const m31_t *coeffs, uint32_t coeffs_log, m31_t *out);
qm31_t or_eval_at_point(const m31_t *coeffs, uint32_t log_size, spoint_t p);
qm31_t or_line_eval_at_point(const qm31_t *coeffs, uint32_t log_size, qm31_t x);
void or_interpolate_many(coset_t half_coset, m31_t *const *cols, size_t n_cols, const m31_t *itwiddles,
                         size_t tree_size);
void or_evaluate_many(coset_t half_coset, const m31_t *const *coeffs, size_t coeff_len, m31_t *const *out,
                      size_t n_cols, const m31_t *twiddles, size_t tree_size);
void or_eval_at_point_many(const m31_t *const *coeffs, const uint32_t *log_sizes, size_t n, spoint_t p,
                           qm31_t *out);

/* ---- FriOps ---- */
void or_fold_line(const m31_t *const src[4], size_t n, coset_t line_domain, qm31_t alpha,
                  m31_t *const dst[4]);
void or_fold_circle_into_line(const m31_t *const src[4], size_t n, coset_t circle_half_coset,
                              qm31_t alpha, m31_t *const dst[4]);

/* ---- MerkleOps<Blake2sMerkleHasher> ---- */
void or_blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t0, uint32_t t1,
                         uint32_t f0, uint32_t f1);
void or_blake2s_std(const uint8_t *msg, size_t len, uint8_t out[32]);
void or_merkle_commit_on_layer(uint32_t log_size, const uint32_t *prev_layer,
                               const uint32_t *const *columns, size_t n_columns,
                               uint32_t *out);

/* ---- QuotientOps ---- */
void or_accumulate_quotients(coset_t half_coset, const m31_t *const *columns, size_t n_columns,
                             qm31_t random_coeff, size_t n_batches, const spoint_t *points,
                             const uint32_t *batch_sizes, const uint32_t *col_indices,
                             const qm31_t *values, m31_t *const out[4]);

/* ---- AccumulationOps ---- */
void or_accumulate(m31_t *const left[4], const m31_t *const right[4], size_t n);

/* ---- wide-Fibonacci AIR ---- */
m31_t or_coset_vanishing_m31(coset_t coset, cpoint_t p);
void or_wide_fib_trace_row(m31_t a, m31_t b, size_t n_columns, m31_t *row);
void or_wide_fib_trace(const m31_t *a0, const m31_t *a1, size_t n_rows, size_t n_columns, m31_t *const *cols);
void or_vanishing_inverses(uint32_t log_n_rows, m31_t *den_inv);
void or_wide_fib_composition(const m31_t *const *trace_evals, size_t n_columns, size_t ext_size,
                             const qm31_t *coeff_powers, const m31_t *den_inv,
                             m31_t *const out[4]);

/* ---- wide-Fibonacci prover (stwo_oracle_prover.c) ---- */
typedef struct { uint32_t log_n_rows, n_columns, log_blowup, n_queries, pow_bits; } or_wide_fib_job;
/* Proof bytes in *proof (free with or_free). Returns 0, or -1 for unsupported
 * parameters, -2 / -3 when the OODS check / the last-layer degree check fails (the
 * bytes are still produced). */
int or_wide_fib_prove(const or_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1, uint8_t **proof,
                      size_t *proof_len);
void or_free(void *p);

/* ---- threading for the timed CPU baseline ---- */
void or_set_threads(int n);
int  or_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
