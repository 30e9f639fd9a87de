// QuotientOps::accumulate_quotients (DEEP quotients).
//
// Semantics (cuda/src/quotients.cu:49-178, stwo_gpu_backend/src/quotient.rs:17-115):
// for row r with domain point p = domain.at(bitrev(r)):
//   acc = sum over batches b, in order: acc * rc^|b| + den_b(p)^-1 * num_b(p),
//   num_b(p) = sum_j c_j col_j[r] - (a_j p.y + b_j),
//   (a_j, b_j, c_j) = rc^(j+1) * (conj(v)-v, v*c - a*P.y, conj(P.y)-P.y) of sample j,
//   den_b(p) = (Pr.x - p.x) Pi.y - (Pr.y - p.y) Pi.x in CM31 (P = Pr + u Pi).
// Line coefficients use each batch's own cumulative offset (the CpuBackend
// semantics; the reference kernel mis-indexes batches of different sizes).
//
// Design: the per-batch sums of a_j and b_j and the doubled c_j are computed once
// on the host and passed by value. A thread handles rows 2k and 2k+1, whose
// domain points are P and conj(P), so one point evaluation (a product of table
// powers of the circle generator) serves two rows. All 2 x n_batches CM31
// denominators of the thread are inverted with one field inversion (Montgomery's
// trick). The column terms accumulate unreduced 33-bit partial products in 64-bit
// registers and reduce once per batch.
#include <atomic>
#include <type_traits>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "quotients.cuh"

namespace stwo {
namespace {

using QuotParams = QuotParamsT<QUOT_MAX_COLS, QUOT_MAX_SAMPLES>;
#ifndef QUOT_PREFETCH_N
#define QUOT_PREFETCH_N 8
#endif
constexpr int QUOT_PREFETCH = QUOT_PREFETCH_N;  // column loads per group (two groups in flight)
static_assert(QUOT_PREFETCH % 4 == 0, "the fold cadence needs groups of a multiple of 4 columns");

// The kernel reads its parameters through get(): by value from the parameter block,
// or from a device-resident block (the prover's, filled by the device channel).
struct QuotByValue {
    QuotParams p;
    __device__ const QuotParams &get() const { return p; }
};
struct QuotByRef {
    const QuotParamsDev *p;
    __device__ const QuotParamsDev &get() const { return *p; }
};

// G^idx for a 31-bit circle-group index: the product of three table entries,
// G^(idx mod 2^11), G^(2^11 * (idx >> 11 mod 2^11)) and G^(2^22 * (idx >> 22)).
__device__ __forceinline__ cpoint point_from_tables(const cpoint *__restrict__ tab, uint32_t idx) {
    const uint2 *t = reinterpret_cast<const uint2 *>(tab);
    const uint2 a = __ldg(t + (idx & 2047u));
    const uint2 b = __ldg(t + CIRCLE_TAB_LO + ((idx >> 11) & 2047u));
    const uint2 c = __ldg(t + 2 * CIRCLE_TAB_LO + (idx >> 22));
    return point_mul(point_mul({a.x, a.y}, {b.x, b.y}), {c.x, c.y});
}

// Unreduced product: value congruent to a*b, in [0, 2p].
__device__ __forceinline__ uint32_t reduce64(uint64_t x) {
    // x < 2^62: fold twice
    uint64_t s = (x & P) + (x >> 31);
    s = (s & P) + (s >> 31);
    return reduce_once((uint32_t)s);
}

// den_b(p) of batch b at a domain point with x coordinate px and y coordinate py.
template <class QP>
__device__ __forceinline__ cm31 quot_den(const QP &p, uint32_t b, uint32_t px, uint32_t py) {
    const cm31 t1 = {m31_sub(p.prx[b].a, px), p.prx[b].b};
    const cm31 t2 = {m31_sub(p.pry[b].a, py), p.pry[b].b};
    return cm31_sub(cm31_mul(t1, p.piy[b]), cm31_mul(t2, p.pix[b]));
}

// STAGE: the CTA first copies every sample's column pointer and doubled coefficient
// into shared memory (n_stage samples), so the column loop reads them there instead
// of chasing col_idx -> cols through global memory (device-resident parameters).
// NB > 0: exactly NB sample batches, known at compile time, so the per-row
// denominators stay in registers (the prover's two quotient groups have one batch
// each: every column sampled at the OODS point); NB == 0: any count up to
// QUOT_MAX_BATCHES.
template <bool COLS_ON_DEVICE, bool STAGE, int NB, class PR>
__global__ void __launch_bounds__(256) quotients_kernel(const __grid_constant__ PR pr,
                                                        const uint32_t *const *__restrict__ dev_cols,
                                                        uint32_t n_stage, uint32_t two) {
    const auto &p = pr.get();
    extern __shared__ uint4 q_smem[];
    qm31 *s_c2 = reinterpret_cast<qm31 *>(q_smem);
    const uint32_t **s_cols = reinterpret_cast<const uint32_t **>(s_c2 + (STAGE ? n_stage : 0));
    if (STAGE) {
        for (uint32_t j = threadIdx.x; j < n_stage; j += blockDim.x) {
            s_c2[j] = p.c2[j];
            s_cols[j] = COLS_ON_DEVICE ? dev_cols[p.col_idx[j]] : p.cols[p.col_idx[j]];
        }
        __syncthreads();
    }
    constexpr int MAXB = NB > 0 ? NB : QUOT_MAX_BATCHES;
    const uint64_t n_pairs = 1ull << (p.log_size - 1);
    const uint32_t n_batches = NB > 0 ? (uint32_t)NB : p.n_batches;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n_pairs;
         k += (uint64_t)gridDim.x * blockDim.x) {
        // Rows 2k and 2k+1 are the domain point and its conjugate.
        const uint32_t hidx = bit_reverse_bits((uint32_t)k, p.log_size - 1);
        const cpoint pt = point_from_tables(p.tab, (p.half_init + p.half_step * hidx) & 0x7fffffffu);
        const uint32_t ys[2] = {pt.y, m31_neg(pt.y)};
        // The first column group's loads go out before the denominators' inversion, a
        // chain of dependent products, so that their latency overlaps it.
        uint2 va[QUOT_PREFETCH], vb[QUOT_PREFETCH];
        {
            const uint32_t j1 = p.batch_end[0];
#pragma unroll
            for (int u = 0; u < QUOT_PREFETCH; u++)
                if ((uint32_t)u < j1) {
                    const uint32_t *col = STAGE ? s_cols[u]
                                                : (COLS_ON_DEVICE ? dev_cols[p.col_idx[u]] : p.cols[p.col_idx[u]]);
                    va[u] = __ldg(reinterpret_cast<const uint2 *>(col) + k);
                }
        }
        // Denominator inverses of both rows, all batches: one inversion (Montgomery's trick).
        cm31 den[2][MAXB];
        {
            cm31 prefix = {1, 0};
            cm31 pre[2][MAXB];
#pragma unroll
            for (int b = 0; b < MAXB; b++) {
                if (NB == 0 && b >= (int)n_batches) break;
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    den[s][b] = quot_den(p, b, pt.x, ys[s]);
                    prefix = cm31_mul(prefix, den[s][b]);
                    pre[s][b] = prefix;
                }
            }
            cm31 inv = cm31_inv(prefix);
#pragma unroll
            for (int b = MAXB - 1; b >= 0; b--) {
                if (NB == 0 && b >= (int)n_batches) continue;
#pragma unroll
                for (int s = 1; s >= 0; s--) {
                    const cm31 prev = (s == 1) ? pre[0][b] : (b > 0 ? pre[1][b - 1] : cm31{1, 0});
                    const cm31 d = den[s][b];
                    den[s][b] = cm31_mul(inv, prev);  // inverse of d
                    inv = cm31_mul(inv, d);
                }
            }
        }
        qm31 acc[2] = {qm31_zero(), qm31_zero()};
        uint32_t j0 = 0;
#pragma unroll
        for (int b = 0; b < MAXB; b++) {
            if (NB == 0 && b >= (int)n_batches) break;
            uint64_t s0[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
            const uint32_t j1 = p.batch_end[b];
            // Column loads in groups of QUOT_PREFETCH, double-buffered: the next group's
            // loads are in flight while this group is accumulated.
            auto load_group = [&](uint32_t jb, uint2 (&v)[QUOT_PREFETCH]) {
#pragma unroll
                for (int u = 0; u < QUOT_PREFETCH; u++) {
                    const uint32_t j = jb + u;
                    if (j < j1) {
                        const uint32_t *col = STAGE ? s_cols[j]
                                                    : (COLS_ON_DEVICE ? dev_cols[p.col_idx[j]] : p.cols[p.col_idx[j]]);
                        v[u] = __ldg(reinterpret_cast<const uint2 *>(col) + k);
                    }
                }
            };
            // 64-bit multiply-accumulates of canonical values (products below 2^62),
            // folded (fold64_fma) after every fourth column: a folded sum plus four
            // products stays below 2^64. The group size is a multiple of 4.
            auto consume = [&](uint32_t jb, const uint2 (&v)[QUOT_PREFETCH]) {
#pragma unroll
                for (int u = 0; u < QUOT_PREFETCH; u++) {
                    if (jb + u >= j1) break;
                    const qm31 c = STAGE ? s_c2[jb + u] : p.c2[jb + u];
                    s0[0][0] = mac64(s0[0][0], v[u].x, c.a.a); s0[0][1] = mac64(s0[0][1], v[u].x, c.a.b);
                    s0[0][2] = mac64(s0[0][2], v[u].x, c.b.a); s0[0][3] = mac64(s0[0][3], v[u].x, c.b.b);
                    s0[1][0] = mac64(s0[1][0], v[u].y, c.a.a); s0[1][1] = mac64(s0[1][1], v[u].y, c.a.b);
                    s0[1][2] = mac64(s0[1][2], v[u].y, c.b.a); s0[1][3] = mac64(s0[1][3], v[u].y, c.b.b);
                    if (u % 4 == 3)
                        for (int s = 0; s < 2; s++)
                            for (int t = 0; t < 4; t++) s0[s][t] = fold64_fma(s0[s][t], two);
                }
            };
            if (b > 0 && j0 < j1) load_group(j0, va);  // batch 0's first group is in flight
            for (uint32_t jb = j0; jb < j1; jb += 2 * QUOT_PREFETCH) {
                if (jb + QUOT_PREFETCH < j1) load_group(jb + QUOT_PREFETCH, vb);
                consume(jb, va);
                if (jb + 2 * QUOT_PREFETCH < j1) load_group(jb + 2 * QUOT_PREFETCH, va);
                if (jb + QUOT_PREFETCH < j1) consume(jb + QUOT_PREFETCH, vb);
            }
            j0 = j1;
            for (int s = 0; s < 2; s++) {
                qm31 num = {{reduce64(s0[s][0]), reduce64(s0[s][1])}, {reduce64(s0[s][2]), reduce64(s0[s][3])}};
                qm31 lin = qm31_add(qm31_scale(p.a_sum[b], ys[s]), p.b_sum[b]);
                num = qm31_sub(num, lin);
                acc[s] = b == 0 ? qm31_mul_cm31(num, den[s][b])
                                : qm31_add(qm31_mul(acc[s], p.batch_coeff[b]), qm31_mul_cm31(num, den[s][b]));
            }
        }
        reinterpret_cast<uint2 *>(p.out[0])[k] = make_uint2(acc[0].a.a, acc[1].a.a);
        reinterpret_cast<uint2 *>(p.out[1])[k] = make_uint2(acc[0].a.b, acc[1].a.b);
        reinterpret_cast<uint2 *>(p.out[2])[k] = make_uint2(acc[0].b.a, acc[1].b.a);
        reinterpret_cast<uint2 *>(p.out[3])[k] = make_uint2(acc[0].b.b, acc[1].b.b);
    }
}

// The circle-group tables of point_from_tables on the current device: G^i for
// i < 2^11, G^(2^11 i) for i < 2^11, G^(2^22 i) for i < 2^9 (36 KiB), computed on the
// host and copied once per device.
__device__ cpoint g_circle_tab[CIRCLE_TAB_SIZE];

}  // namespace

int circle_point_table(const cpoint **out) {
    static std::atomic<uint64_t> done{0};
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    int rc = once_per_device(done, [] {
        std::vector<cpoint> t(CIRCLE_TAB_SIZE);
        cpoint step[3] = {index_to_point(1), index_to_point(1u << 11), index_to_point(1u << 22)};
        const uint32_t len[3] = {CIRCLE_TAB_LO, CIRCLE_TAB_LO, CIRCLE_TAB_SIZE - 2 * CIRCLE_TAB_LO};
        uint32_t off = 0;
        for (int s = 0; s < 3; s++) {
            cpoint r = {1, 0};
            for (uint32_t i = 0; i < len[s]; i++) {
                t[off + i] = r;
                r = point_mul(r, step[s]);
            }
            off += len[s];
        }
        STWO_CUDA_TRY(cudaMemcpyToSymbol(g_circle_tab, t.data(), sizeof(cpoint) * CIRCLE_TAB_SIZE));
        return (int)STWO_OK;
    });
    if (rc) return rc;
    void *addr = nullptr;
    STWO_CUDA_TRY(cudaGetSymbolAddress(&addr, g_circle_tab));
    *out = static_cast<const cpoint *>(addr);
    return STWO_OK;
}

namespace {

inline qm31 to_q(stwo_qm31 v) { return {{v.a, v.b}, {v.c, v.d}}; }


}  // namespace

int quotients_async(uint32_t half_init, uint32_t half_step, uint32_t log_size, const uint32_t *const *cols,
                    uint32_t n_cols, bool cols_on_device, stwo_qm31 rc_c, const stwo_spoint *pts,
                    const uint32_t *bsz, const uint32_t *cidx, const stwo_qm31 *vals, uint32_t n_batches,
                    uint32_t *const *out4, cudaStream_t st) {
    STWO_REQUIRE(log_size >= 1 && log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "domain log size %u", log_size);
    STWO_REQUIRE(n_batches <= (uint32_t)QUOT_MAX_BATCHES, STWO_ERR_UNSUPPORTED_SIZE, "at most %d sample batches",
                 QUOT_MAX_BATCHES);
    STWO_REQUIRE(cols_on_device || n_cols <= (uint32_t)QUOT_MAX_COLS, STWO_ERR_UNSUPPORTED_SIZE,
                 "at most %d columns", QUOT_MAX_COLS);
    auto holder = std::make_unique<QuotByValue>();
    QuotParams *p = &holder->p;
    const cpoint *tab = nullptr;
    int trc = circle_point_table(&tab);
    if (trc) return trc;
    quot_init_static(*p, half_init, half_step, log_size, out4, tab);
    p->n_batches = n_batches;
    if (!cols_on_device)
        for (uint32_t i = 0; i < n_cols; i++) p->cols[i] = cols[i];
    qm31 rcq = to_q(rc_c);
    uint32_t off = 0;
    std::vector<qm31> v;
    for (uint32_t b = 0; b < n_batches; b++) {
        STWO_REQUIRE(off + bsz[b] <= (uint32_t)QUOT_MAX_SAMPLES, STWO_ERR_UNSUPPORTED_SIZE, "at most %d samples",
                     QUOT_MAX_SAMPLES);
        v.resize(bsz[b]);
        for (uint32_t j = 0; j < bsz[b]; j++) {
            v[j] = to_q(vals[off + j]);
            STWO_REQUIRE(cidx[off + j] < n_cols, STWO_ERR_INVALID_ARGUMENT, "sample column index %u out of range",
                         cidx[off + j]);
            p->col_idx[off + j] = (uint16_t)cidx[off + j];
        }
        quot_fill_batch(*p, b, rcq, to_q(pts[b].x), to_q(pts[b].y), v.data(), bsz[b], off);
        off += bsz[b];
        p->batch_end[b] = off;
    }
    uint64_t pairs = 1ull << (log_size - 1);
    uint64_t blocks = (pairs + 255) / 256;
    uint64_t cap = (uint64_t)device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    // Every sample's coefficient and column pointer staged in shared memory (at most
    // QUOT_MAX_SAMPLES x 24 bytes = 12 KiB): the column loop then reads them there
    // instead of indexing the parameter block at run time.
    const uint32_t n_samples = off;
    const size_t smem = (size_t)n_samples * (sizeof(qm31) + sizeof(void *));
    auto launch = [&](auto nb) {
        constexpr int NBV = decltype(nb)::value;
        if (cols_on_device)
            quotients_kernel<true, true, NBV><<<(unsigned)blocks, 256, smem, st>>>(*holder, cols, n_samples, 2u);
        else
            quotients_kernel<false, true, NBV><<<(unsigned)blocks, 256, smem, st>>>(*holder, nullptr, n_samples, 2u);
    };
    switch (n_batches) {
    case 1: launch(std::integral_constant<int, 1>{}); break;
    case 2: launch(std::integral_constant<int, 2>{}); break;
    case 3: launch(std::integral_constant<int, 3>{}); break;
    case 4: launch(std::integral_constant<int, 4>{}); break;
    default: launch(std::integral_constant<int, 0>{}); break;
    }
    STWO_LAUNCH_CHECK("quotients_kernel");
    return STWO_OK;
}

int quotients_dev_async(const QuotParamsDev *p_dev, uint32_t log_size, uint32_t n_samples, cudaStream_t st) {
    STWO_REQUIRE(log_size >= 1 && log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "domain log size %u", log_size);
    STWO_REQUIRE(n_samples >= 1 && n_samples <= 1024, STWO_ERR_UNSUPPORTED_SIZE, "%u samples", n_samples);
    const size_t smem = (size_t)n_samples * (sizeof(qm31) + sizeof(void *));
    uint64_t pairs = 1ull << (log_size - 1);
    uint64_t blocks = (pairs + 255) / 256;
    uint64_t cap = (uint64_t)device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    quotients_kernel<false, true, 1><<<(unsigned)blocks, 256, smem, st>>>(QuotByRef{p_dev}, nullptr, n_samples, 2u);
    STWO_LAUNCH_CHECK("quotients_kernel");
    return STWO_OK;
}

}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_accumulate_quotients(uint32_t half_coset_initial_index, uint32_t half_coset_step_size,
                              uint32_t domain_log_size, const uint32_t *const *columns, uint32_t n_columns,
                              stwo_qm31 random_coeff, const stwo_spoint *sample_points, const uint32_t *batch_sizes,
                              const uint32_t *column_indices, const stwo_qm31 *sampled_values, uint32_t n_batches,
                              uint32_t *const *out4, void *stream) {
    return quotients_async(half_coset_initial_index, half_coset_step_size, domain_log_size, columns, n_columns, false,
                           random_coeff, sample_points, batch_sizes, column_indices, sampled_values, n_batches, out4,
                           as_stream(stream));
}

void accumulate_quotients(uint32_t half_coset_initial_index, uint32_t half_coset_step_size, uint32_t domain_size,
                          uint32_t *const *columns, size_t number_of_columns, stwo_qm31 random_coeff,
                          const uint32_t *sample_points, const uint32_t *sample_columns_indexes,
                          uint32_t sample_columns_indexes_size, const stwo_qm31 *sample_column_values,
                          const uint32_t *sample_column_and_values_sizes, uint32_t sample_size,
                          uint32_t *result_column_0, uint32_t *result_column_1, uint32_t *result_column_2,
                          uint32_t *result_column_3, uint32_t flattened_line_coeffs_size) {
    (void)sample_columns_indexes_size;
    (void)flattened_line_coeffs_size;
    if (!is_pow2(domain_size) || domain_size < 2) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "domain size %u is not a power of two >= 2", domain_size);
        return;
    }
    uint32_t *out[4] = {result_column_0, result_column_1, result_column_2, result_column_3};
    sync_default_stream(quotients_async(half_coset_initial_index, half_coset_step_size, log2_u64(domain_size),
                                        const_cast<const uint32_t *const *>(columns), (uint32_t)number_of_columns,
                                        true, random_coeff, reinterpret_cast<const stwo_spoint *>(sample_points),
                                        sample_column_and_values_sizes, sample_columns_indexes, sample_column_values,
                                        sample_size, out, 0));
}

}  // extern "C"
