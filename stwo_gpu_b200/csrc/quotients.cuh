// DEEP-quotient parameters shared by the quotient kernel (quotients.cu), its host
// entry points and the prover's device channel, which fills the sample-dependent
// fields on the device.
#pragma once
#include <cstdint>

#include "field.cuh"

namespace stwo {

constexpr int QUOT_MAX_COLS = 512;
constexpr int QUOT_MAX_SAMPLES = 512;
constexpr int QUOT_MAX_BATCHES = 16;

// Circle-group point tables (quotients.cu): G^i for i < 2^11, G^(2^11 i) for i < 2^11
// and G^(2^22 i) for i < 2^9, consecutive.
constexpr uint32_t CIRCLE_TAB_LO = 2048;
constexpr uint32_t CIRCLE_TAB_SIZE = 2 * CIRCLE_TAB_LO + 512;
// Device address of the tables on the current device (filled on first use).
int circle_point_table(const cpoint **out);

template <int MAXC, int MAXS>
struct QuotParamsT {
    const uint32_t *cols[MAXC];
    qm31 c2[MAXS];                        // c_j (canonical)
    uint16_t col_idx[MAXS];
    qm31 a_sum[QUOT_MAX_BATCHES], b_sum[QUOT_MAX_BATCHES], batch_coeff[QUOT_MAX_BATCHES];
    cm31 prx[QUOT_MAX_BATCHES], pry[QUOT_MAX_BATCHES], pix[QUOT_MAX_BATCHES], piy[QUOT_MAX_BATCHES];
    cm31 den_k[QUOT_MAX_BATCHES];          // Pr.x Pi.y - Pr.y Pi.x: den_b(p) = K_b - p.x Pi.y + p.y Pi.x
    uint32_t batch_end[QUOT_MAX_BATCHES];  // cumulative sample counts
    uint32_t n_batches;
    uint32_t half_init, half_step;        // half coset indices
    uint32_t log_size;                    // domain log size
    uint32_t *out[4];
    const cpoint *tab;                    // circle_point_table() of the launching device
};

// The prover's device-resident parameters: up to 1024 columns and samples.
using QuotParamsDev = QuotParamsT<1024, 1024>;

// Sample-dependent fields of batch b (samples off .. off+count-1 at point (px, py)):
// the batch coefficient rc^count and, per sample j with alpha = rc^(j+1),
// (a, b, c) = alpha * (conj(v) - v, v*c0 - a*py, c0), c0 = conj(py) - py
// (complex_conjugate_line_coeffs); a and b summed per batch, c stored per sample.
// With several batches, quot_scale_batches then folds the accumulation's Horner
// coefficients into these fields.
template <class QP>
__host__ __device__ inline void quot_fill_point(QP &p, uint32_t b, qm31 px, qm31 py) {
    p.prx[b] = px.a;
    p.pix[b] = px.b;
    p.pry[b] = py.a;
    p.piy[b] = py.b;
    p.den_k[b] = cm31_sub(cm31_mul(px.a, py.b), cm31_mul(py.a, px.b));
}

template <class QP>
__host__ __device__ inline void quot_fill_batch(QP &p, uint32_t b, qm31 rc, qm31 px, qm31 py, const qm31 *vals,
                                                uint32_t count, uint32_t off) {
    quot_fill_point(p, b, px, py);
    p.batch_coeff[b] = qm31_pow(rc, count);
    const qm31 c0 = qm31_sub(qm31_conj(py), py);
    qm31 alpha = qm31_one(), as = qm31_zero(), bs = qm31_zero();
    for (uint32_t j = 0; j < count; j++) {
        alpha = qm31_mul(alpha, rc);
        const qm31 v = vals[j];
        qm31 a = qm31_sub(qm31_conj(v), v);
        qm31 bb = qm31_sub(qm31_mul(v, c0), qm31_mul(a, py));
        a = qm31_mul(alpha, a);
        bb = qm31_mul(alpha, bb);
        const qm31 c = qm31_mul(alpha, c0);
        as = qm31_add(as, a);
        bs = qm31_add(bs, bb);
        p.c2[off + j] = c;
    }
    p.a_sum[b] = as;
    p.b_sum[b] = bs;
}

// The accumulation over batches, acc = acc * rc^|b| + num_b / den_b in batch order
// (quotients.cu:111-178), equals sum_b C_b num_b / den_b with C_b the product of the
// later batches' coefficients rc^|b'|. num_b is linear in the batch's a, b and c
// fields, so multiplying those by C_b (here, once per call) leaves the kernel a plain
// sum over batches. The last batch has C = 1; with one batch nothing changes.
template <class QP>
__host__ __device__ inline void quot_scale_batches(QP &p, uint32_t n_batches) {
    qm31 cb = qm31_one();
    for (int b = (int)n_batches - 1; b >= 0; b--) {
        if (b + 1 < (int)n_batches) {
            cb = qm31_mul(cb, p.batch_coeff[b + 1]);
            const uint32_t j0 = b == 0 ? 0u : p.batch_end[b - 1];
            for (uint32_t j = j0; j < p.batch_end[b]; j++) p.c2[j] = qm31_mul(p.c2[j], cb);
            p.a_sum[b] = qm31_mul(p.a_sum[b], cb);
            p.b_sum[b] = qm31_mul(p.b_sum[b], cb);
        }
    }
}

// Sum of one QM31 per thread over a CTA of blockDim.x <= 1024 threads; every thread
// gets the sum. sh: 32 QM31 of shared memory.
__device__ inline qm31 block_sum_qm31(qm31 v, qm31 *sh) {
    for (int m = 16; m >= 1; m >>= 1) {
        v.a.a = m31_add(v.a.a, __shfl_xor_sync(0xffffffffu, v.a.a, m));
        v.a.b = m31_add(v.a.b, __shfl_xor_sync(0xffffffffu, v.a.b, m));
        v.b.a = m31_add(v.b.a, __shfl_xor_sync(0xffffffffu, v.b.a, m));
        v.b.b = m31_add(v.b.b, __shfl_xor_sync(0xffffffffu, v.b.b, m));
    }
    __syncthreads();  // sh may hold a previous call's values
    if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    qm31 s = qm31_zero();
    for (uint32_t w = 0; w < (blockDim.x + 31) / 32; w++) s = qm31_add(s, sh[w]);
    return s;
}

// quot_fill_batch by a whole CTA: thread t takes samples t, t + T, ... with
// alpha = rc^(j+1), and the a / b sums are reduced across the CTA. For the prover's
// single-batch groups (no quot_scale_batches step is needed with one batch).
template <class QP>
__device__ inline void quot_fill_batch_block(QP &p, uint32_t b, qm31 rc, qm31 px, qm31 py, const qm31 *vals,
                                             uint32_t count, uint32_t off, qm31 *sh) {
    const uint32_t T = blockDim.x;
    const qm31 c0 = qm31_sub(qm31_conj(py), py);
    const qm31 step = qm31_pow(rc, T);
    qm31 alpha = qm31_pow(rc, threadIdx.x + 1), as = qm31_zero(), bs = qm31_zero();
    for (uint32_t j = threadIdx.x; j < count; j += T) {
        const qm31 v = vals[j];
        qm31 a = qm31_sub(qm31_conj(v), v);
        qm31 bb = qm31_sub(qm31_mul(v, c0), qm31_mul(a, py));
        a = qm31_mul(alpha, a);
        bb = qm31_mul(alpha, bb);
        const qm31 c = qm31_mul(alpha, c0);
        as = qm31_add(as, a);
        bs = qm31_add(bs, bb);
        p.c2[off + j] = c;
        alpha = qm31_mul(alpha, step);
    }
    as = block_sum_qm31(as, sh);
    bs = block_sum_qm31(bs, sh);
    if (threadIdx.x == 0) {
        quot_fill_point(p, b, px, py);
        p.batch_coeff[b] = qm31_pow(rc, count);
        p.a_sum[b] = as;
        p.b_sum[b] = bs;
    }
}

// The column-independent fields: domain, outputs, point tables.
template <class QP>
inline void quot_init_static(QP &p, uint32_t half_init, uint32_t half_step, uint32_t log_size, uint32_t *const *out4,
                             const cpoint *tab) {
    p.tab = tab;
    p.half_init = half_init;
    p.half_step = half_step;
    p.log_size = log_size;
    for (int c = 0; c < 4; c++) p.out[c] = out4[c];
}

// Launches the quotient kernel on parameters resident in device memory (n_samples:
// the total sample count, batch_end of the last batch); jobs parameter blocks of one
// shape at once, block k at p_dev moved by k * js bytes.
int quotients_dev_async(const QuotParamsDev *p_dev, uint32_t log_size, uint32_t n_samples, uint32_t jobs, size_t js,
                        cudaStream_t st);

}  // namespace stwo
