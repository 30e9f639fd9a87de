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
#include "tc.cuh"

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

// ---------------------------------------------------------------------------------
// Tensor-core form (tcgen05, 8-bit integer MMA). The column sums of every batch,
// S_b,q(r) = sum_c W[c][b].q * col_c[r] with W[c][b] the sum of the batch's
// coefficients on column c, are a product of the 2^n x C matrix of column values and
// the C x 4 NB matrix W. Over bytes: with v = sum_i v_i 2^(8i) (column value) and
// D_i = W.q * 2^(8i) mod p = sum_j d_ij 2^(8j),
//   S_b,q(r) = sum_j 2^(8j) T_j(r) (mod p),  T_j(r) = sum_(c, i) v_i(r) d_ij,
// a u8 x u8 product with K = 4 C (column c, byte i) and N = 16 NB (batch, component,
// byte j), accumulated exactly in 32 bits (K * 255^2 < 2^31 for C < 8256). A tile is
// 128 row pairs (rows 2k and 2k + 1, at conjugate domain points), one per TMEM lane;
// the even and the odd rows are two MMAs into adjacent halves of the accumulator, so
// one thread finishes both rows of its pair as quotients_kernel does (one point, shared
// denominator products, one inversion for the 2 NB denominators). A CTA of 13 warps
// streams tiles:
//  * warps 8-11 copy 16 columns of the tile per stage into one of QTC_STAGES K-major
//    stages in shared memory (4-byte asynchronous copies, up to QTC_STAGES stages in
//    flight, each completing its stage's "full" barrier); a stage holds slab 2 g + s
//    (columns 4g .. 4g + 3 of the rows of parity s) at (2 g + s) * 2048 bytes;
//  * one thread of warp 12 issues the stage's MMAs (128 x N x 32, one per 8 columns
//    and parity) into one of two TMEM accumulators and commits them to the stage's
//    "empty" barrier;
//  * warps 0-3 and 4-7 take the tiles in turn: each reads its tile's accumulator
//    (a row pair a thread), frees it, and finishes the pair.
// B (the byte matrix of W) is built by each CTA in shared memory from the samples.
// Every barrier wait gives up after QTC_WAIT_NS or once another role has given up;
// a CTA that gave up counts itself in g_quot_tc_faults (stwo_quotients_tc_faults).
constexpr int QTC_STAGES = 4;
constexpr uint32_t QTC_STAGE_BYTES = 128 * 2 * 16 * 4;  // 128 row pairs x 16 columns x 4 bytes
constexpr int QTC_THREADS = 13 * 32;
constexpr uint64_t QTC_WAIT_NS = 1000000000ull;
constexpr uint32_t QTC_MAX_B_BYTES = 64 * 1024;
constexpr size_t QTC_SMEM_FLOOR = 80 * 1024;  // more than a third of an SM's 228 KiB

__device__ uint32_t g_quot_tc_faults;

__host__ __device__ constexpr size_t qtc_b_bytes(uint32_t c8, int nb) { return (size_t)c8 * 16 * nb * 4; }
__host__ __device__ constexpr size_t qtc_smem_bytes(uint32_t c8, int nb) {
    return (size_t)QTC_STAGES * QTC_STAGE_BYTES + qtc_b_bytes(c8, nb) + (size_t)c8 * 8 + (2 * QTC_STAGES + 5) * 8 + 8;
}

template <int NB, bool COLS_ON_DEVICE, class PR>
__global__ void __launch_bounds__(QTC_THREADS, 2)
    quotients_tc_kernel(const __grid_constant__ PR pr, const uint32_t *const *__restrict__ dev_cols, uint32_t n_cols) {
    constexpr int N = 16 * NB;
    // two accumulators, each an even-row half and an odd-row half of N columns, every
    // half at a multiple of 32 columns
    constexpr uint32_t PAR = N <= 32 ? 32u : 64u, SLOT = 2 * PAR, TM_COLS = 2 * SLOT;
    constexpr uint32_t IDESC = tc::idesc_u8<128, N>();
    const auto &p = pr.get();
    extern __shared__ __align__(1024) uint8_t qsm[];
    const uint32_t C8 = (n_cols + 7) & ~7u;
    uint8_t *As = qsm;
    uint8_t *Bs = qsm + QTC_STAGES * QTC_STAGE_BYTES;
    const uint32_t **s_cols = reinterpret_cast<const uint32_t **>(Bs + qtc_b_bytes(C8, NB));
    uint64_t *bars = reinterpret_cast<uint64_t *>(s_cols + C8);
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bars + 2 * QTC_STAGES + 5);
    volatile uint32_t *s_abort = s_tmem + 1;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // ---- B = the bytes of W, from the samples
    for (uint32_t c = tid; c < C8; c += blockDim.x)
        s_cols[c] = c < n_cols ? (COLS_ON_DEVICE ? dev_cols[c] : p.cols[c]) : nullptr;
    unsigned long long *W = reinterpret_cast<unsigned long long *>(As);  // [C8][NB][4], in the stages
    for (uint32_t i = tid; i < C8 * NB * 4; i += blockDim.x) W[i] = 0;
    if (tid == 0) *s_abort = 0;
    __syncthreads();
    const uint32_t n_samples = p.batch_end[NB - 1];
    for (uint32_t j = tid; j < n_samples; j += blockDim.x) {
        uint32_t b = 0;
#pragma unroll
        for (int bb = 0; bb + 1 < NB; bb++) b += j >= p.batch_end[bb] ? 1u : 0u;
        const uint32_t c = p.col_idx[j];
        if (c >= C8) continue;
        const qm31 v = p.c2[j];
        unsigned long long *w = W + ((size_t)c * NB + b) * 4;
        atomicAdd(w + 0, (unsigned long long)v.a.a);
        atomicAdd(w + 1, (unsigned long long)v.a.b);
        atomicAdd(w + 2, (unsigned long long)v.b.a);
        atomicAdd(w + 3, (unsigned long long)v.b.b);
    }
    __syncthreads();
    for (uint32_t it = tid; it < C8 * NB * 4; it += blockDim.x) {
        const uint32_t c = it / (NB * 4), bq = it % (NB * 4);  // it = (c * NB + b) * 4 + q, bq = 4 b + q
        uint8_t *dst = Bs + ((size_t)(c >> 2) * N + bq * 4) * 16 + (c & 3) * 4;
        uint32_t d = reduce64_p(W[it]);
#pragma unroll
        for (int i = 0; i < 4; i++) {
#pragma unroll
            for (int jb = 0; jb < 4; jb++) dst[jb * 16 + i] = (uint8_t)(d >> (8 * jb));
            const uint64_t s = (uint64_t)d << 8;  // d * 2^8 mod p
            d = reduce_once((uint32_t)((s & P) + (s >> 31)));
        }
    }
    tc::fence_async_smem();
    const uint32_t bar0 = tc::smem_addr(bars);
    if (tid == 0) {
        for (int s = 0; s < QTC_STAGES; s++) {
            tc::mbar_init(bar0 + 8 * s, 128);                 // full: the loader threads
            tc::mbar_init(bar0 + 8 * (QTC_STAGES + s), 1);    // empty: one MMA commit
        }
        for (int e = 0; e < 2; e++) {
            tc::mbar_init(bar0 + 8 * (2 * QTC_STAGES + e), 1);       // accumulator full: one commit
            tc::mbar_init(bar0 + 8 * (2 * QTC_STAGES + 2 + e), 128); // accumulator empty: 4 warps
        }
        tc::mbar_init(bar0 + 8 * (2 * QTC_STAGES + 4), 1);  // all MMAs done
        tc::mbar_init_fence();
    }
    if (warp == 12) tc::tmem_alloc(s_tmem, TM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;
    const uint32_t n_tiles = 1u << (p.log_size - 8);
    const uint32_t n_chunks = (C8 + 15) / 16;
    auto FULL = [&](uint32_t s) { return bar0 + 8 * s; };
    auto EMPTY = [&](uint32_t s) { return bar0 + 8 * (QTC_STAGES + s); };
    auto TFULL = [&](uint32_t e) { return bar0 + 8 * (2 * QTC_STAGES + e); };
    auto TEMPTY = [&](uint32_t e) { return bar0 + 8 * (2 * QTC_STAGES + 2 + e); };
    const uint32_t DONE = bar0 + 8 * (2 * QTC_STAGES + 4);
    auto give_up = [&]() {
        if (!*s_abort) {
            *s_abort = 1;
            atomicAdd(&g_quot_tc_faults, 1u);
        }
    };

    if (warp >= 8 && warp < 12) {
        // ---- loaders: warp wl copies row pairs 32 wl .. 32 wl + 31 of the tile, 16
        // columns a stage, with 4-byte asynchronous copies (a warp's copy covers 8 pairs x
        // 4 columns of one parity: 128 contiguous bytes of the stage); the stage's "full"
        // barrier completes when all 128 loader threads' copies have landed.
        const uint32_t wl = warp - 8, ro = lane >> 2, co = lane & 3;
        const uint32_t st0 = tc::smem_addr(As) + (32 * wl + ro) * 16 + co * 4;
        uint32_t g = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x) {
            const size_t row0 = (size_t)tile * 256 + 2 * (32 * wl + ro);
            for (uint32_t kc = 0; kc < n_chunks; kc++, g++) {
                const uint32_t s = g % QTC_STAGES;
                if (!tc::mbar_wait(EMPTY(s), ((g / QTC_STAGES) & 1) ^ 1, s_abort, QTC_WAIT_NS)) {
                    give_up();
                    ok = false;
                    break;
                }
                const uint32_t dst = st0 + s * QTC_STAGE_BYTES;
#pragma unroll
                for (int cg = 0; cg < 4; cg++) {
                    const uint32_t c = kc * 16 + 4 * cg + co;
                    if (c < n_cols) {
                        const uint32_t *src = s_cols[c] + row0;
#pragma unroll
                        for (int pg = 0; pg < 4; pg++)
#pragma unroll
                            for (int par = 0; par < 2; par++)
                                tc::cp_async4(dst + (2 * cg + par) * 2048 + pg * 128, src + 16 * pg + par);
                    }
                }
                tc::cp_async_arrive(FULL(s));
            }
        }
    } else if (warp == 12) {
        // ---- the MMA thread
        if (lane == 0) {
            const uint32_t a0 = tc::smem_addr(As), b0 = tc::smem_addr(Bs);
            uint32_t g = 0;
            bool ok = true;
            for (uint32_t tl = 0, tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x, tl++) {
                const uint32_t e = tl & 1;
                if (!tc::mbar_wait(TEMPTY(e), ((tl >> 1) & 1) ^ 1, s_abort, QTC_WAIT_NS)) {
                    give_up();
                    break;
                }
                tc::fence_after_sync();
                for (uint32_t kc = 0; kc < n_chunks; kc++, g++) {
                    const uint32_t s = g % QTC_STAGES;
                    if (!tc::mbar_wait(FULL(s), (g / QTC_STAGES) & 1, s_abort, QTC_WAIT_NS)) {
                        give_up();
                        ok = false;
                        break;
                    }
                    tc::fence_async_smem();
                    tc::fence_after_sync();
                    const uint32_t left = (C8 - kc * 16) / 8, nm = left < 2 ? left : 2u;
                    for (uint32_t m = 0; m < nm; m++) {
                        const uint64_t bd = tc::smem_desc(b0 + (kc * 4 + 2 * m) * N * 16, N * 16, 128);
                        for (uint32_t par = 0; par < 2; par++) {
                            // slabs 4m + par and 4m + par + 2: columns 8m .. 8m + 7, parity par
                            const uint64_t ad =
                                tc::smem_desc(a0 + s * QTC_STAGE_BYTES + (4 * m + par) * 2048, 4096, 128);
                            tc::mma_u8(tmem + e * SLOT + par * PAR, ad, bd, IDESC, (kc | m) != 0);
                        }
                    }
                    tc::commit(EMPTY(s));
                }
                if (ok) tc::commit(TFULL(e));
            }
            // every MMA issued here completes before the accumulators are freed
            tc::commit(DONE);
            if (!tc::mbar_wait(DONE, 0, nullptr, QTC_WAIT_NS)) give_up();
        }
        __syncwarp();
    } else {
        // ---- epilogue group e: the tiles tl = e, e + 2, ... of this CTA, a row pair a thread
        const uint32_t e = warp >> 2, kp = 32 * (warp & 3) + lane;
        const uint32_t lane_base = tmem + ((32 * (warp & 3)) << 16) + e * SLOT;
        for (uint32_t tl = e, tile = blockIdx.x + e * gridDim.x; tile < n_tiles; tl += 2, tile += 2 * gridDim.x) {
            if (!tc::mbar_wait(TFULL(e), (tl >> 1) & 1, s_abort, QTC_WAIT_NS)) {
                give_up();
                break;
            }
            tc::fence_after_sync();
            uint32_t num[2][NB][4];
#pragma unroll
            for (int par = 0; par < 2; par++)
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    uint32_t r[16];
                    tc::tmem_ld16(lane_base + par * PAR + 16 * b, r);
                    tc::tmem_wait_ld();
                    // sum_j 2^(8j) T_j < 2^56: one fold leaves it below 2^31 + 2^25
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const uint64_t t = (uint64_t)r[4 * q] + ((uint64_t)r[4 * q + 1] << 8) +
                                           ((uint64_t)r[4 * q + 2] << 16) + ((uint64_t)r[4 * q + 3] << 24);
                        num[par][b][q] = reduce_once((uint32_t)(t & P) + (uint32_t)(t >> 31));
                    }
                }
            tc::fence_before_sync();
            tc::mbar_arrive(TEMPTY(e));
            const uint32_t k = tile * 128 + kp;  // rows 2k, 2k + 1
            const uint32_t hidx = bit_reverse_bits(k, p.log_size - 1);
            const cpoint pt = point_from_tables(p.tab, (p.half_init + p.half_step * hidx) & 0x7fffffffu);
            cm31 dinv[2][NB];
            uint32_t nrm[2][NB], pre[2][NB], prefix = 1;
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const cm31 u = cm31_sub(p.den_k[b], cm31_scale(p.piy[b], pt.x));
                const cm31 v = cm31_scale(p.pix[b], pt.y);
                dinv[0][b] = cm31_add(u, v);
                dinv[1][b] = cm31_sub(u, v);
#pragma unroll
                for (int sg = 0; sg < 2; sg++) {
                    uint64_t n2 = (uint64_t)dinv[sg][b].a * dinv[sg][b].a;
                    mac_wide(n2, dinv[sg][b].b, dinv[sg][b].b);
                    nrm[sg][b] = reduce64_p(n2);
                    prefix = m31_mul(prefix, nrm[sg][b]);
                    pre[sg][b] = prefix;
                }
            }
            uint32_t inv = m31_inv(prefix);
#pragma unroll
            for (int b = NB - 1; b >= 0; b--) {
#pragma unroll
                for (int sg = 1; sg >= 0; sg--) {
                    const uint32_t prev = sg == 1 ? pre[0][b] : (b > 0 ? pre[1][b - 1] : 1u);
                    const uint32_t ni = m31_mul(inv, prev);  // 1 / norm
                    inv = m31_mul(inv, nrm[sg][b]);
                    dinv[sg][b] = {m31_mul(dinv[sg][b].a, ni), m31_mul(m31_neg(dinv[sg][b].b), ni)};
                }
            }
            // sum_b (num_b - lin_b) * dinv_b, the QM31 x CM31 products accumulated unreduced
            // in 64 bits: (x + y i)(c + d i) = (x c + y (p - d)) + (x d + y c) i; two
            // products a batch and coordinate, folded after every second batch (a folded
            // sum plus four products of canonical values stays below 2^64).
            uint64_t ac[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const qm31 ay = qm31_scale(p.a_sum[b], pt.y);
                const qm31 lin[2] = {qm31_add(p.b_sum[b], ay), qm31_sub(p.b_sum[b], ay)};
#pragma unroll
                for (int sg = 0; sg < 2; sg++) {
                    const qm31 nb =
                        qm31_sub({{num[sg][b][0], num[sg][b][1]}, {num[sg][b][2], num[sg][b][3]}}, lin[sg]);
                    const uint32_t c = dinv[sg][b].a, d = dinv[sg][b].b, nd = P - d;
                    ac[sg][0] = mac64(mac64(ac[sg][0], nb.a.a, c), nb.a.b, nd);
                    ac[sg][1] = mac64(mac64(ac[sg][1], nb.a.a, d), nb.a.b, c);
                    ac[sg][2] = mac64(mac64(ac[sg][2], nb.b.a, c), nb.b.b, nd);
                    ac[sg][3] = mac64(mac64(ac[sg][3], nb.b.a, d), nb.b.b, c);
                    if (b & 1)
#pragma unroll
                        for (int q = 0; q < 4; q++) ac[sg][q] = fold64_fma(ac[sg][q], 2u);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                reinterpret_cast<uint2 *>(p.out[q])[k] = make_uint2(reduce64_p(ac[0][q]), reduce64_p(ac[1][q]));
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 12) tc::tmem_free(tmem, TM_COLS);
}

// Whether the tensor-core form takes a call: domains of at least 256 rows, 1..4
// batches, and the byte matrix of W within QTC_MAX_B_BYTES. With the
// quotients_tensor_cores tunable at 1 (the default) only calls of two or more batches
// over at least 2^16 rows, where it measured faster (32 columns x 4 points: 2^16 14.3
// vs 16.7 us, 2^19 34 vs 76 us, 2^22 0.19 vs 0.56 ms); one-batch calls (the prover's)
// gain 0-19% at 2^18 and above and lose below, and its CTAs (13 warps, 70-140 KiB of
// shared memory) crowd out concurrent jobs' kernels in the proof server, so they stay
// on the CUDA cores. At 2 every call it can take; at 0 none.
bool quot_tc_eligible(uint32_t log_size, uint32_t n_batches, uint32_t n_cols) {
    const uint32_t c8 = (n_cols + 7) & ~7u;
    const int mode = tunable(TUNE_QUOT_TENSOR);
    return mode != 0 && (mode == 2 || (n_batches >= 2 && log_size >= 16)) && log_size >= 8 && log_size <= 31 &&
           n_batches >= 1 && n_batches <= 4 && n_cols >= 1 && qtc_b_bytes(c8, (int)n_batches) <= QTC_MAX_B_BYTES;
}

template <int NB, bool COLS_ON_DEVICE, class PR>
int launch_quot_tc(const PR &pr, const uint32_t *const *dev_cols, uint32_t n_cols, uint32_t log_size, uint32_t jobs,
                   cudaStream_t st) {
    static std::atomic<uint64_t> attr_done{0};
    auto kern = quotients_tc_kernel<NB, COLS_ON_DEVICE, PR>;
    int rc = once_per_device(attr_done, [&] {
        STWO_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)qtc_smem_bytes(QTC_MAX_B_BYTES / (64 * NB), NB)));
        return (int)STWO_OK;
    });
    if (rc) return rc;
    const uint32_t c8 = (n_cols + 7) & ~7u;
    const uint64_t tiles = 1ull << (log_size - 8), cap = 2ull * device_sm_count();
    const unsigned gx = (unsigned)(tiles < cap ? tiles : cap);
    // With 3 or 4 batches a CTA holds 256 TMEM columns: at least QTC_SMEM_FLOOR bytes of
    // shared memory keep such CTAs to two an SM, so the SM's 512 columns always suffice.
    size_t smem = qtc_smem_bytes(c8, NB);
    if (NB >= 3 && smem < QTC_SMEM_FLOOR) smem = QTC_SMEM_FLOOR;
    kern<<<dim3(gx, jobs), QTC_THREADS, smem, st>>>(pr, dev_cols, n_cols);
    STWO_LAUNCH_CHECK("quotients_tc_kernel");
    return STWO_OK;
}

template <bool COLS_ON_DEVICE, class PR>
int launch_quot_tc_nb(uint32_t nb, const PR &pr, const uint32_t *const *dev_cols, uint32_t n_cols, uint32_t log_size,
                      uint32_t jobs, cudaStream_t st) {
    switch (nb) {
    case 1: return launch_quot_tc<1, COLS_ON_DEVICE>(pr, dev_cols, n_cols, log_size, jobs, st);
    case 2: return launch_quot_tc<2, COLS_ON_DEVICE>(pr, dev_cols, n_cols, log_size, jobs, st);
    case 3: return launch_quot_tc<3, COLS_ON_DEVICE>(pr, dev_cols, n_cols, log_size, jobs, st);
    default: return launch_quot_tc<4, COLS_ON_DEVICE>(pr, dev_cols, n_cols, log_size, jobs, st);
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
    if (quot_tc_eligible(log_size, n_batches, n_cols)) {
        if (cols_on_device) return launch_quot_tc_nb<true>(n_batches, *holder, cols, n_cols, log_size, 1, st);
        return launch_quot_tc_nb<false>(n_batches, *holder, nullptr, n_cols, log_size, 1, st);
    }
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
    // one batch; column j is sample j
    if (quot_tc_eligible(log_size, 1, n_samples))
        return launch_quot_tc<1, false>(QuotByRef{p_dev, js}, nullptr, n_samples, log_size, jobs, st);
    const uint32_t n_stage = quot_padded(n_samples);
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

int stwo_quotients_tc_faults(uint32_t *count, int reset) {
    STWO_REQUIRE(count, STWO_ERR_INVALID_ARGUMENT, "null count");
    STWO_CUDA_TRY(cudaMemcpyFromSymbol(count, g_quot_tc_faults, sizeof(uint32_t)));
    if (reset) {
        const uint32_t zero = 0;
        STWO_CUDA_TRY(cudaMemcpyToSymbol(g_quot_tc_faults, &zero, sizeof(uint32_t)));
    }
    return STWO_OK;
}

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
