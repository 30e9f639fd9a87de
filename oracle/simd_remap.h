/* Builds the oracle prover (stwo_oracle_prover.c) on the SIMD functions of
 * stwo_simd.cc: force-included when compiling the prover into libstwo_simd_*.so, it
 * renames the prover's calls of the heavy oracle functions, and the prover itself,
 * so that library exports simd_wide_fib_prove beside the scalar oracle. Baseline
 * only; the oracle library is built without it. */
#ifndef STWO_SIMD_REMAP_H
#define STWO_SIMD_REMAP_H
#define or_precompute_twiddles simd_precompute_twiddles
#define or_interpolate_many simd_interpolate_many
#define or_evaluate_many simd_evaluate_many
#define or_eval_at_point_many simd_eval_at_point_many
#define or_merkle_commit_on_layer simd_merkle_commit_on_layer
#define or_accumulate_quotients simd_accumulate_quotients
#define or_wide_fib_composition simd_wide_fib_composition
#define or_wide_fib_trace simd_wide_fib_trace
#define or_vanishing_inverses simd_vanishing_inverses
#define or_fold_line simd_fold_line
#define or_fold_circle_into_line simd_fold_circle_into_line
#define or_batch_inverse_m31 simd_batch_inverse_m31
#define or_wide_fib_prove simd_wide_fib_prove
#define or_free simd_free
#endif
