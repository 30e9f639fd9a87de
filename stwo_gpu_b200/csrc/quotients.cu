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
#define QUOT_PREFETCH_N 4
#endif
constexpr int QUOT_PREFETCH = QUOT_PREFETCH_N;  // column loads per group (two groups in flight)
static_assert(QUOT_PREFETCH % 4 == 0, "the fold cadence needs groups of a multiple of 4 columns");
#ifndef QUOT_MIN_BLOCKS_N
#define QUOT_MIN_BLOCKS_N 3
#endif
constexpr int QUOT_MIN_BLOCKS = QUOT_MIN_BLOCKS_N;  // CTAs of 256 threads resident per SM (register cap)

// The kernel reads its parameters through get(): by value from the parameter block,
// or from a device-resident block (the prover's, filled by the device channel).
struct QuotByValue {
    QuotParams p;
    __device__ const QuotParams &get() const { return p; }
};
struct QuotByRef {
    const QuotParamsDev *p;
    size_t js;  // jobs' memory stride: blockIdx.y's block is job 0's moved by blockIdx.y * js
    __device__ const QuotParamsDev &get() const { return *job_ptr(p, js, blockIdx.y); }
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

// 64-bit multiply-accumulate acc += a * b (one wide multiply-add on the FMA pipe).
// (Written as plain C++: the same wide multiply-add as inline PTX measured 13% slower
// over the whole kernel on B200, the compiler scheduling around the asm blocks.)
__device__ __forceinline__ void mac_wide(uint64_t &acc, uint32_t a, uint32_t b) { acc = mac64(acc, a, b); }

// Samples staged per batch: the batch's count rounded up to whole column groups.
__host__ __device__ __forceinline__ uint32_t quot_padded(uint32_t count) {
    return (count + QUOT_PREFETCH - 1) / QUOT_PREFETCH * QUOT_PREFETCH;
}

// The CTA first copies every sample's column pointer and coefficient into shared
// memory, each batch padded to whole groups of QUOT_PREFETCH samples with zero
// coefficients (and the batch's first column, so the padding loads stay in bounds):
// the column loop then runs whole groups with no per-sample bound checks.
// NB > 0: exactly NB sample batches, known at compile time, so the per-row
// denominators stay in registers (the prover's two quotient groups have one batch
// each: every column sampled at the OODS point); NB == 0: any count up to
// QUOT_MAX_BATCHES. n_stage: the padded sample total.
//
// Per row pair (rows 2k and 2k + 1, at the domain point p and its conjugate):
//  * den_b = K_b - p.x Pi.y +- p.y Pi.x: the two rows share both products;
//  * the 2 NB denominators are inverted through their M31 norms
//    (1 / (a + b i) = (a - b i) / (a^2 + b^2)) with one field inversion;
//  * the batches' Horner coefficients are folded into their fields
//    (quot_scale_batches), so each batch adds num_b / den_b to the sum.
template <bool COLS_ON_DEVICE, int NB, class PR>
__global__ void __launch_bounds__(256, QUOT_MIN_BLOCKS) quotients_kernel(const __grid_constant__ PR pr,
                                                                         const uint32_t *const *__restrict__ dev_cols,
                                                                         uint32_t n_stage, uint32_t two) {
    const auto &p = pr.get();
    extern __shared__ uint4 q_smem[];
    qm31 *s_c2 = reinterpret_cast<qm31 *>(q_smem);
    const uint32_t **s_cols = reinterpret_cast<const uint32_t **>(s_c2 + n_stage);
    constexpr int MAXB = NB > 0 ? NB : QUOT_MAX_BATCHES;
    const uint32_t n_batches = NB > 0 ? (uint32_t)NB : p.n_batches;
    uint32_t ps[MAXB + 1];  // padded staged start of each batch
    ps[0] = 0;
#pragma unroll
    for (int b = 0; b < MAXB; b++) {
        if (NB == 0 && b >= (int)n_batches) break;
        ps[b + 1] = ps[b] + quot_padded(p.batch_end[b] - (b > 0 ? p.batch_end[b - 1] : 0u));
    }
    for (uint32_t js = threadIdx.x; js < n_stage; js += blockDim.x) {
        uint32_t b = 0, start = 0;  // the batch of staged index js and its padded start
        for (;;) {
            const uint32_t next = start + quot_padded(p.batch_end[b] - (b > 0 ? p.batch_end[b - 1] : 0u));
            if (b + 1 >= n_batches || js < next) break;
            start = next;
            b++;
        }
        const uint32_t e0 = b > 0 ? p.batch_end[b - 1] : 0u, u = js - start;
        const uint32_t j = e0 + u < p.batch_end[b] ? e0 + u : e0;
        s_c2[js] = e0 + u < p.batch_end[b] ? p.c2[j] : qm31_zero();
        s_cols[js] = COLS_ON_DEVICE ? dev_cols[p.col_idx[j]] : p.cols[p.col_idx[j]];
    }
    __syncthreads();
    const uint64_t n_pairs = 1ull << (p.log_size - 1);
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n_pairs;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t hidx = bit_reverse_bits((uint32_t)k, p.log_size - 1);
        const cpoint pt = point_from_tables(p.tab, (p.half_init + p.half_step * hidx) & 0x7fffffffu);
        // Column loads in groups of QUOT_PREFETCH, double-buffered: the next group's
        // loads are in flight while this group is accumulated.
        uint2 va[QUOT_PREFETCH], vb[QUOT_PREFETCH];
        auto load_group = [&](uint32_t jb, uint2 (&v)[QUOT_PREFETCH]) {
#pragma unroll
            for (int u = 0; u < QUOT_PREFETCH; u++)
                v[u] = __ldg(reinterpret_cast<const uint2 *>(s_cols[jb + u]) + k);
        };
        // The first column group's loads go out before the denominators' inversion, a
        // chain of dependent products, so that their latency overlaps it.
        if (ps[1] > 0) load_group(0, va);
        // Inverse denominators of both rows, every batch.
        cm31 dinv[2][MAXB];
        {
            uint32_t nrm[2][MAXB], pre[2][MAXB];
            uint32_t prefix = 1;
#pragma unroll
            for (int b = 0; b < MAXB; b++) {
                if (NB == 0 && b >= (int)n_batches) break;
                const cm31 u = cm31_sub(p.den_k[b], cm31_scale(p.piy[b], pt.x));
                const cm31 v = cm31_scale(p.pix[b], pt.y);
                dinv[0][b] = cm31_add(u, v);
                dinv[1][b] = cm31_sub(u, v);
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    uint64_t n = (uint64_t)dinv[s][b].a * dinv[s][b].a;
                    mac_wide(n, dinv[s][b].b, dinv[s][b].b);
                    nrm[s][b] = reduce64_p(n);
                    prefix = m31_mul(prefix, nrm[s][b]);
                    pre[s][b] = prefix;
                }
            }
            uint32_t inv = m31_inv(prefix);
#pragma unroll
            for (int b = MAXB - 1; b >= 0; b--) {
                if (NB == 0 && b >= (int)n_batches) continue;
#pragma unroll
                for (int s = 1; s >= 0; s--) {
                    const uint32_t prev = (s == 1) ? pre[0][b] : (b > 0 ? pre[1][b - 1] : 1u);
                    const uint32_t ni = m31_mul(inv, prev);  // 1 / norm
                    inv = m31_mul(inv, nrm[s][b]);
                    dinv[s][b] = {m31_mul(dinv[s][b].a, ni), m31_mul(m31_neg(dinv[s][b].b), ni)};
                }
            }
        }
        qm31 acc[2] = {qm31_zero(), qm31_zero()};
#pragma unroll
        for (int b = 0; b < MAXB; b++) {
            if (NB == 0 && b >= (int)n_batches) break;
            uint64_t s0[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
            const uint32_t j0 = ps[b], j1 = ps[b + 1];
            // 64-bit multiply-accumulates of canonical values (products below 2^62),
            // folded (fold64_fma) after every fourth column: a folded sum plus four
            // products stays below 2^64. The group size is a multiple of 4.
            auto consume = [&](uint32_t jb, const uint2 (&v)[QUOT_PREFETCH]) {
#pragma unroll
                for (int u = 0; u < QUOT_PREFETCH; u++) {
                    const qm31 c = s_c2[jb + u];
                    mac_wide(s0[0][0], v[u].x, c.a.a); mac_wide(s0[0][1], v[u].x, c.a.b);
                    mac_wide(s0[0][2], v[u].x, c.b.a); mac_wide(s0[0][3], v[u].x, c.b.b);
                    mac_wide(s0[1][0], v[u].y, c.a.a); mac_wide(s0[1][1], v[u].y, c.a.b);
                    mac_wide(s0[1][2], v[u].y, c.b.a); mac_wide(s0[1][3], v[u].y, c.b.b);
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
            // num_s = sum_j c_j col_j - (a y_s + b) with y_1 = -y_0: the rows share a y_0.
            const qm31 ay = qm31_scale(p.a_sum[b], pt.y);
            const qm31 lin[2] = {qm31_add(p.b_sum[b], ay), qm31_sub(p.b_sum[b], ay)};
#pragma unroll
            for (int s = 0; s < 2; s++) {
                qm31 num = {{reduce64_p(s0[s][0]), reduce64_p(s0[s][1])}, {reduce64_p(s0[s][2]), reduce64_p(s0[s][3])}};
                num = qm31_sub(num, lin[s]);
                acc[s] = qm31_add(acc[s], qm31_mul_cm31(num, dinv[s][b]));
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
    quot_scale_batches(*p, n_batches);
    uint64_t pairs = 1ull << (log_size - 1);
    uint64_t blocks = (pairs + 255) / 256;
    uint64_t cap = (uint64_t)device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    // Every sample's coefficient and column pointer staged in shared memory, each batch
    // padded to whole column groups (at most (QUOT_MAX_SAMPLES + QUOT_MAX_BATCHES *
    // QUOT_PREFETCH) x 24 bytes, 15 KiB): the column loop then reads them there
    // instead of indexing the parameter block at run time.
    uint32_t n_stage = 0;
    for (uint32_t b = 0; b < n_batches; b++) n_stage += quot_padded(bsz[b]);
    const size_t smem = (size_t)n_stage * (sizeof(qm31) + sizeof(void *));
    auto launch = [&](auto nb) {
        constexpr int NBV = decltype(nb)::value;
        if (cols_on_device)
            quotients_kernel<true, NBV><<<(unsigned)blocks, 256, smem, st>>>(*holder, cols, n_stage, 2u);
        else
            quotients_kernel<false, NBV><<<(unsigned)blocks, 256, smem, st>>>(*holder, nullptr, n_stage, 2u);
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

int quotients_dev_async(const QuotParamsDev *p_dev, uint32_t log_size, uint32_t n_samples, uint32_t jobs, size_t js,
                        cudaStream_t st) {
    STWO_REQUIRE(log_size >= 1 && log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "domain log size %u", log_size);
    STWO_REQUIRE(jobs >= 1 && jobs <= 65535, STWO_ERR_INVALID_ARGUMENT, "quotient groups per launch: %u", jobs);
    STWO_REQUIRE(n_samples >= 1 && n_samples <= 1024, STWO_ERR_UNSUPPORTED_SIZE, "%u samples", n_samples);
    const uint32_t n_stage = quot_padded(n_samples);  // one batch
    const size_t smem = (size_t)n_stage * (sizeof(qm31) + sizeof(void *));
    uint64_t pairs = 1ull << (log_size - 1);
    uint64_t blocks = (pairs + 255) / 256;
    uint64_t cap = (uint64_t)device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    quotients_kernel<false, 1><<<dim3((unsigned)blocks, jobs), 256, smem, st>>>(QuotByRef{p_dev, js}, nullptr, n_stage,
                                                                               2u);
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
