// AccumulationOps::accumulate and the wide-Fibonacci composition kernel.
//
// accumulate (cuda/src/accumulate.cu:4-26): SoA QM31 left += right, 16-byte vectors.
//
// Wide-Fibonacci composition (cuda/src/examples/wide_fibonacci.cu:3-66,
// stwo_gpu_backend/src/examples/wide_fibonacci.rs:90-141): for every row of the
// extended domain
//   out = den_inv * sum_{i < N-2} (c_i^2 + c_{i+1}^2 - c_{i+2}) * powers[N-3-i].
// The reference launches it with grid and block swapped and clones the column
// pointer array with the wrong length (.cu:48,54); here the pointers travel in the
// parameter block or a device table, each thread does two consecutive rows (8-byte
// loads per column), and each QM31 coordinate of the sum accumulates unreduced
// partial products in 64 bits, reduced once per row.
#include <atomic>
#include <memory>

#include "common.cuh"
#include "tc.cuh"

namespace stwo {
namespace {

struct Acc4 { uint32_t *l[4]; const uint32_t *r[4]; };

__global__ void accumulate_kernel(const __grid_constant__ Acc4 p, uint64_t n4, uint64_t n) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n4; k += (uint64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (4 * k + 3 < n) {
                uint4 a = reinterpret_cast<const uint4 *>(p.l[c])[k];
                uint4 b = __ldg(reinterpret_cast<const uint4 *>(p.r[c]) + k);
                a.x = m31_add(a.x, b.x); a.y = m31_add(a.y, b.y); a.z = m31_add(a.z, b.z); a.w = m31_add(a.w, b.w);
                reinterpret_cast<uint4 *>(p.l[c])[k] = a;
            } else {
                for (uint64_t i = 4 * k; i < n; i++) p.l[c][i] = m31_add(p.l[c][i], p.r[c][i]);
            }
        }
    }
}

constexpr int WF_MAX_COLS = 2048;
static_assert(WF_MAX_COLS * (16 + 8) <= 48 * 1024, "staged powers and pointers fit the default shared memory");
constexpr int WF_GROUP = 4;  // columns a load group (the fold period: one fold after every group)

// Trace column pointers in the parameter block (CAP of them) or, for CAP == 1, in a
// device table.
template <int CAP>
struct WideFibParams {
    const uint32_t *trace[CAP];
    const uint32_t *const *trace_dev;
    uint32_t *out[4];
    const uint32_t *den_inv;  // per-row denominator inverses, or null:
    uint32_t den_half[2];     // the inverses on the first and second half of the (bit-reversed) rows
    const qm31 *powers_dev;   // device powers
    uint32_t n_cols;
    uint32_t log_size;
    uint32_t two;             // 2 (fold64_fma)
    size_t js;                // jobs' memory stride: blockIdx.y's job is job 0's moved by blockIdx.y * js
};

// Powers on the device (plain QM31). Two rows per thread (8-byte loads). The column
// loop runs over whole groups of WF_GROUP columns in two register buffers, the next
// group's loads issued before the current group is consumed (a warp keeps loads in
// flight while it computes), then over the remaining columns one at a time; the small
// per-thread state keeps four CTAs of 256 threads per SM. Each coordinate of the sum
// is a 64-bit multiply-accumulate of canonical values, folded (fold64_fma) after every
// group of four columns: a folded sum plus at most four products stays below 2^64.
template <int CAP>
__global__ void __launch_bounds__(256, 4) wide_fib_kernel(const __grid_constant__ WideFibParams<CAP> p) {
    const uint64_t n = 1ull << p.log_size;
    const uint64_t pairs = (n + 1) / 2;
    // The column pointers and each column's power, staged once per CTA: the column loop
    // then reads them from shared memory instead of chasing the device table (measured
    // 4-15% faster across 2^12..2^20-row proofs).
    extern __shared__ uint4 wf_smem[];
    qm31 *s_pow = reinterpret_cast<qm31 *>(wf_smem);
    const uint32_t **s_col = reinterpret_cast<const uint32_t **>(s_pow + p.n_cols);
    const uint32_t job = blockIdx.y;
    const uint32_t *const *trace_dev = job_ptr(p.trace_dev, p.js, job);
    const qm31 *powers_dev = job_ptr(p.powers_dev, p.js, job);
    const uint32_t *den_inv = job_ptr(p.den_inv, p.js, job);
    for (uint32_t c = threadIdx.x; c < p.n_cols; c += blockDim.x) {
        s_col[c] = CAP == 1 ? trace_dev[c] : p.trace[c];
        if (c >= 2) s_pow[c] = powers_dev[p.n_cols - 1 - c];
    }
    __syncthreads();
    auto colp = [&](uint32_t c) { return s_col[c]; };
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < pairs; k += (uint64_t)gridDim.x * blockDim.x) {
        const bool full = 2 * k + 1 < n;
        auto load = [&](uint32_t col) -> uint2 {
            const uint32_t *c = colp(col);
            if (full) return __ldg(reinterpret_cast<const uint2 *>(c) + k);
            return make_uint2(c[2 * k], 0u);
        };
        uint64_t acc[2][4] = {};
        uint32_t s0[2], s1[2];
        {
            const uint2 c0 = load(0), c1 = load(1);
            s0[0] = m31_sqr(c0.x); s0[1] = m31_sqr(c0.y);
            s1[0] = m31_sqr(c1.x); s1[1] = m31_sqr(c1.y);
        }
        // constraint col - 2 takes powers[N-3-(col-2)]
        auto consume_one = [&](uint32_t col, uint2 v) {
            const qm31 w = s_pow[col];
            const uint32_t vv[2] = {v.x, v.y};
#pragma unroll
            for (int r = 0; r < 2; r++) {
                const uint32_t cons = m31_sub(m31_add(s0[r], s1[r]), vv[r]);
                acc[r][0] = mac64(acc[r][0], cons, w.a.a);
                acc[r][1] = mac64(acc[r][1], cons, w.a.b);
                acc[r][2] = mac64(acc[r][2], cons, w.b.a);
                acc[r][3] = mac64(acc[r][3], cons, w.b.b);
                s0[r] = s1[r];
                s1[r] = m31_sqr(vv[r]);
            }
        };
        auto fold = [&] {
#pragma unroll
            for (int r = 0; r < 2; r++)
                for (int c = 0; c < 4; c++) acc[r][c] = fold64_fma(acc[r][c], p.two);
        };
        auto load_group = [&](uint32_t base, uint2 (&v)[WF_GROUP]) {
#pragma unroll
            for (int u = 0; u < WF_GROUP; u++) v[u] = load(base + u);
        };
        auto consume_group = [&](uint32_t base, const uint2 (&v)[WF_GROUP]) {
#pragma unroll
            for (int u = 0; u < WF_GROUP; u++) consume_one(base + u, v[u]);
            fold();
        };
        const uint32_t nc = p.n_cols;
        const uint32_t groups_end = nc < 2 ? nc : 2 + (nc - 2) / WF_GROUP * WF_GROUP;
        uint2 ga[WF_GROUP], gb[WF_GROUP];
        if (2 < groups_end) load_group(2, ga);
        for (uint32_t base = 2; base < groups_end; base += 2 * WF_GROUP) {
            if (base + WF_GROUP < groups_end) load_group(base + WF_GROUP, gb);
            consume_group(base, ga);
            if (base + WF_GROUP >= groups_end) break;
            if (base + 2 * WF_GROUP < groups_end) load_group(base + 2 * WF_GROUP, ga);
            consume_group(base + WF_GROUP, gb);
        }
        for (uint32_t col = groups_end; col < nc; col++) consume_one(col, load(col));  // at most three
        uint32_t o[4][2];
        for (int r = 0; r < 2; r++) {
            const uint64_t row = 2 * k + r;
            uint32_t d = row >= n ? 0u : den_inv ? __ldg(den_inv + row) : p.den_half[row >> (p.log_size - 1)];
            uint32_t d2 = d << 1;
            for (int c = 0; c < 4; c++) o[c][r] = m31_mul2(reduce64_p(acc[r][c]), d2);
        }
        for (int c = 0; c < 4; c++) {
            uint32_t *out = job_ptr(p.out[c], p.js, job);
            if (full) reinterpret_cast<uint2 *>(out)[k] = make_uint2(o[c][0], o[c][1]);
            else out[2 * k] = o[c][0];
        }
    }
}

// ---------------------------------------------------------------------------------
// Tensor-core form (tcgen05, 8-bit integer MMA). The sum over constraints
// sum_i P_i e_i (e_i = c_i^2 + c_(i+1)^2 - c_(i+2), P_i = powers[N-3-i]) is, over bytes
// (as in the tensor-core DEEP quotients), a u8 x u8 product with K = 4 bytes a
// constraint and N = 16 (QM31 coordinate, byte j of P_i.q * 2^(8b)), exact in 32 bits.
// A CTA of 13 warps streams tiles of 128 rows, 32 constraints a stage:
//  * warps 8-11 copy columns 32 kc .. 32 kc + 31 of the tile (4-byte asynchronous
//    copies, 8 rows x 4 columns a warp copy) into the stage's slabs (slab g: columns
//    4g .. 4g + 3, row r at r * 16 bytes), and columns 32 kc + 32, 32 kc + 33 into the
//    stage's look-ahead rows, and complete its "raw" barrier;
//  * warps 4-7 read their row's 34 values back and overwrite value i with e_i (value
//    i is no longer needed once e_i is known), then complete the stage's "full" barrier;
//  * one thread of warp 12 issues the stage's four MMAs (128 x 16 x 32) into one of two
//    TMEM accumulators;
//  * warps 0-3 read a tile's accumulator (a row a thread), release it, fold the four
//    coordinates mod p and multiply by the row's denominator inverse.
// Constraints past N-3 read stale values and have zero weights. Every barrier wait
// gives up after WTC_WAIT_NS or once another role gave up (counted in
// g_comp_tc_faults).
constexpr int WTC_STAGES = 3;
constexpr uint32_t WTC_STAGE_BYTES = 128 * 32 * 4;  // 128 rows x 32 values (then constraints)
constexpr uint32_t WTC_LA_BYTES = 2 * 128 * 4;      // the next two columns of the 128 rows
constexpr int WTC_THREADS = 13 * 32;
constexpr uint64_t WTC_WAIT_NS = 1000000000ull;
constexpr uint32_t WTC_MAX_COLS = 1024;

__device__ uint32_t g_comp_tc_faults;

__host__ __device__ constexpr uint32_t wtc_chunks(uint32_t nc) { return (nc - 2 + 31) / 32; }
__host__ __device__ constexpr size_t wtc_b_bytes(uint32_t nc) { return (size_t)wtc_chunks(nc) * 32 * 4 * 16; }
__host__ __device__ constexpr size_t wtc_smem_bytes(uint32_t nc) {
    return (size_t)WTC_STAGES * (WTC_STAGE_BYTES + WTC_LA_BYTES) + wtc_b_bytes(nc) + (size_t)nc * 8 +
           (3 * WTC_STAGES + 5) * 8 + 8;
}

__device__ __forceinline__ uint32_t qcoord(const qm31 &v, uint32_t q) {
    return q == 0 ? v.a.a : q == 1 ? v.a.b : q == 2 ? v.b.a : v.b.b;
}

template <int CAP>
__global__ void __launch_bounds__(WTC_THREADS, 3) wide_fib_tc_kernel(const __grid_constant__ WideFibParams<CAP> p) {
    constexpr int N = 16;
    constexpr uint32_t SLOT = 32, TM_COLS = 64;
    constexpr uint32_t IDESC = tc::idesc_u8<128, N>();
    extern __shared__ __align__(1024) uint8_t wsm[];
    const uint32_t nc = p.n_cols, n_chunks = wtc_chunks(nc);
    uint8_t *As = wsm;
    uint32_t *LA = reinterpret_cast<uint32_t *>(wsm + WTC_STAGES * WTC_STAGE_BYTES);
    uint8_t *Bs = wsm + WTC_STAGES * (WTC_STAGE_BYTES + WTC_LA_BYTES);
    const uint32_t **s_col = reinterpret_cast<const uint32_t **>(Bs + wtc_b_bytes(nc));
    uint64_t *bars = reinterpret_cast<uint64_t *>(s_col + nc);
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bars + 3 * WTC_STAGES + 5);
    volatile uint32_t *s_abort = s_tmem + 1;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, job = blockIdx.y;
    const uint32_t *const *trace_dev = job_ptr(p.trace_dev, p.js, job);
    const qm31 *powers = job_ptr(p.powers_dev, p.js, job);
    const uint32_t *den_inv = job_ptr(p.den_inv, p.js, job);

    for (uint32_t c = tid; c < nc; c += blockDim.x) s_col[c] = CAP == 1 ? trace_dev[c] : p.trace[c];
    if (tid == 0) *s_abort = 0;
    // B: slab g holds constraints 4g .. 4g + 3; row n = 4 q + byte of P_i.q * 2^(8b),
    // bytes b of constraint i at (i % 4) * 4 + b
    for (uint32_t it = tid; it < n_chunks * 32 * 4; it += blockDim.x) {
        const uint32_t i = it >> 2, q = it & 3;
        uint32_t w = i + 3 <= nc ? qcoord(powers[nc - 3 - i], q) : 0u;
        uint8_t *dst = Bs + ((size_t)(i >> 2) * N + q * 4) * 16 + (i & 3) * 4;
#pragma unroll
        for (int b = 0; b < 4; b++) {
#pragma unroll
            for (int jb = 0; jb < 4; jb++) dst[jb * 16 + b] = (uint8_t)(w >> (8 * jb));
            const uint64_t sh = (uint64_t)w << 8;  // w * 2^8 mod p
            w = reduce_once((uint32_t)((sh & P) + (sh >> 31)));
        }
    }
    tc::fence_async_smem();
    const uint32_t bar0 = tc::smem_addr(bars);
    auto RAW = [&](uint32_t s) { return bar0 + 8 * s; };
    auto FULL = [&](uint32_t s) { return bar0 + 8 * (WTC_STAGES + s); };
    auto EMPTY = [&](uint32_t s) { return bar0 + 8 * (2 * WTC_STAGES + s); };
    auto TFULL = [&](uint32_t e) { return bar0 + 8 * (3 * WTC_STAGES + e); };
    auto TEMPTY = [&](uint32_t e) { return bar0 + 8 * (3 * WTC_STAGES + 2 + e); };
    const uint32_t DONE = bar0 + 8 * (3 * WTC_STAGES + 4);
    if (tid == 0) {
        for (int s = 0; s < WTC_STAGES; s++) {
            tc::mbar_init(RAW(s), 128);   // the loader threads' copies
            tc::mbar_init(FULL(s), 128);  // the constraint threads
            tc::mbar_init(EMPTY(s), 1);   // one MMA commit
        }
        for (int e = 0; e < 2; e++) {
            tc::mbar_init(TFULL(e), 1);
            tc::mbar_init(TEMPTY(e), 128);
        }
        tc::mbar_init(DONE, 1);
        tc::mbar_init_fence();
    }
    if (warp == 12) tc::tmem_alloc(s_tmem, TM_COLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *s_tmem;
    const uint32_t n_tiles = 1u << (p.log_size - 7);
    auto give_up = [&]() {
        if (!*s_abort) {
            *s_abort = 1;
            atomicAdd(&g_comp_tc_faults, 1u);
        }
    };

    if (warp >= 8 && warp < 12) {
        // ---- loaders: rows 32 wl .. 32 wl + 31 of the tile
        const uint32_t wl = warp - 8, ro = lane >> 2, co = lane & 3;
        const uint32_t st0 = tc::smem_addr(As) + (32 * wl + ro) * 16 + co * 4;
        const uint32_t la0 = tc::smem_addr(LA) + (32 * wl + lane) * 4;
        uint32_t g = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x) {
            const size_t row0 = (size_t)tile * 128 + 32 * wl + ro;
            for (uint32_t kc = 0; kc < n_chunks; kc++, g++) {
                const uint32_t s = g % WTC_STAGES;
                if (!tc::mbar_wait(EMPTY(s), ((g / WTC_STAGES) & 1) ^ 1, s_abort, WTC_WAIT_NS)) {
                    give_up();
                    ok = false;
                    break;
                }
                const uint32_t dst = st0 + s * WTC_STAGE_BYTES;
#pragma unroll
                for (int cg = 0; cg < 8; cg++) {
                    const uint32_t c = kc * 32 + 4 * cg + co;
                    if (c < nc) {
                        const uint32_t *src = s_col[c] + row0;
#pragma unroll
                        for (int rg = 0; rg < 4; rg++) tc::cp_async4(dst + cg * 2048 + rg * 128, src + 8 * rg);
                    }
                }
#pragma unroll
                for (int t = 0; t < 2; t++) {
                    const uint32_t c = kc * 32 + 32 + t;
                    if (c < nc)
                        tc::cp_async4(la0 + s * WTC_LA_BYTES + t * 512, s_col[c] + (size_t)tile * 128 + 32 * wl + lane);
                }
                tc::cp_async_arrive(RAW(s));
            }
        }
    } else if (warp >= 4 && warp < 8) {
        // ---- constraints: row 32 (warp - 4) + lane of every stage, in place
        const uint32_t r = 32 * (warp - 4) + lane;
        uint32_t g = 0;
        bool ok = true;
        for (uint32_t tile = blockIdx.x; ok && tile < n_tiles; tile += gridDim.x) {
            for (uint32_t kc = 0; kc < n_chunks; kc++, g++) {
                const uint32_t s = g % WTC_STAGES;
                if (!tc::mbar_wait(RAW(s), (g / WTC_STAGES) & 1, s_abort, WTC_WAIT_NS)) {
                    give_up();
                    ok = false;
                    break;
                }
                uint8_t *stg = As + s * WTC_STAGE_BYTES + r * 16;
                uint32_t a[34];
#pragma unroll
                for (int cg = 0; cg < 8; cg++) {
                    const uint4 v = *reinterpret_cast<const uint4 *>(stg + cg * 2048);
                    a[4 * cg] = v.x;
                    a[4 * cg + 1] = v.y;
                    a[4 * cg + 2] = v.z;
                    a[4 * cg + 3] = v.w;
                }
                a[32] = LA[(s * WTC_LA_BYTES) / 4 + r];
                a[33] = LA[(s * WTC_LA_BYTES + 512) / 4 + r];
                uint32_t sp = m31_sqr(a[0]), sc = m31_sqr(a[1]);
#pragma unroll
                for (int cg = 0; cg < 8; cg++) {
                    uint32_t e4[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const uint32_t x = a[4 * cg + u + 2];
                        e4[u] = m31_sub(m31_add(sp, sc), x);
                        sp = sc;
                        sc = m31_sqr(x);
                    }
                    *reinterpret_cast<uint4 *>(stg + cg * 2048) = make_uint4(e4[0], e4[1], e4[2], e4[3]);
                }
                tc::fence_async_smem();
                tc::mbar_arrive(FULL(s));
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
                if (!tc::mbar_wait(TEMPTY(e), ((tl >> 1) & 1) ^ 1, s_abort, WTC_WAIT_NS)) {
                    give_up();
                    break;
                }
                tc::fence_after_sync();
                for (uint32_t kc = 0; kc < n_chunks; kc++, g++) {
                    const uint32_t s = g % WTC_STAGES;
                    if (!tc::mbar_wait(FULL(s), (g / WTC_STAGES) & 1, s_abort, WTC_WAIT_NS)) {
                        give_up();
                        ok = false;
                        break;
                    }
                    tc::fence_async_smem();
                    tc::fence_after_sync();
#pragma unroll
                    for (uint32_t m = 0; m < 4; m++) {
                        // slabs 2m, 2m + 1: constraints 8m .. 8m + 7 of the stage
                        const uint64_t ad = tc::smem_desc(a0 + s * WTC_STAGE_BYTES + (2 * m) * 2048, 2048, 128);
                        const uint64_t bd = tc::smem_desc(b0 + (kc * 8 + 2 * m) * N * 16, N * 16, 128);
                        tc::mma_u8(tmem + e * SLOT, ad, bd, IDESC, (kc | m) != 0);
                    }
                    tc::commit(EMPTY(s));
                }
                if (ok) tc::commit(TFULL(e));
            }
            // every MMA issued here completes before the accumulators are freed
            tc::commit(DONE);
            if (!tc::mbar_wait(DONE, 0, nullptr, WTC_WAIT_NS)) give_up();
        }
        __syncwarp();
    } else {
        // ---- epilogue: a row a thread, the tiles in turn through the two accumulators
        const uint32_t row = 32 * warp + lane;
        const uint32_t lane_base = tmem + ((32 * warp) << 16);
        uint32_t *out[4];
#pragma unroll
        for (int c = 0; c < 4; c++) out[c] = job_ptr(p.out[c], p.js, job);
        for (uint32_t tl = 0, tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, tl++) {
            const uint32_t e = tl & 1;
            if (!tc::mbar_wait(TFULL(e), (tl >> 1) & 1, s_abort, WTC_WAIT_NS)) {
                give_up();
                break;
            }
            tc::fence_after_sync();
            uint32_t r[16];
            tc::tmem_ld16(lane_base + e * SLOT, r);
            tc::tmem_wait_ld();
            tc::fence_before_sync();
            tc::mbar_arrive(TEMPTY(e));
            const uint32_t R = tile * 128 + row;
            const uint32_t d = den_inv ? __ldg(den_inv + R) : p.den_half[R >> (p.log_size - 1)];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                // sum_j 2^(8j) T_j < 2^56: one fold leaves it below 2^31 + 2^25
                const uint64_t t = (uint64_t)r[4 * q] + ((uint64_t)r[4 * q + 1] << 8) +
                                   ((uint64_t)r[4 * q + 2] << 16) + ((uint64_t)r[4 * q + 3] << 24);
                out[q][R] = m31_mul(reduce_once((uint32_t)(t & P) + (uint32_t)(t >> 31)), d);
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 12) tc::tmem_free(tmem, TM_COLS);
}

// The tensor-core form takes domains of at least 128 rows and 3..WTC_MAX_COLS columns
// when the composition_tensor_cores tunable is 1. It is off by default: against
// wide_fib_kernel it measured 2-4% faster at the prover's sizes (256 columns x 2^21:
// 0.578 vs 0.604 ms, 2^20: 0.307 vs 0.313 ms), 19% faster near 2^17, and slower with few
// columns (16 x 2^22: 0.140 vs 0.100 ms) or a 64 KiB weight matrix (1024 x 2^20: 1.31
// vs 1.21 ms), too little for its 13-warp CTAs in the proof server's concurrent mix. It
// needs its dynamic shared memory limit raised once per device.
template <int CAP>
bool launch_wf_tc(const WideFibParams<CAP> &p, uint32_t jobs, cudaStream_t st) {
    if (tunable(TUNE_COMP_TENSOR) != 1 || p.log_size < 7 || p.n_cols < 3 || p.n_cols > WTC_MAX_COLS) return false;
    static std::atomic<uint64_t> attr_done{0};
    if (once_per_device(attr_done, [] {
            STWO_CUDA_TRY(cudaFuncSetAttribute(wide_fib_tc_kernel<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)wtc_smem_bytes(WTC_MAX_COLS)));
            return (int)STWO_OK;
        }) != STWO_OK)
        return false;
    const uint64_t tiles = 1ull << (p.log_size - 7), cap = 2ull * device_sm_count();
    const unsigned gx = (unsigned)(tiles < cap ? tiles : cap);
    wide_fib_tc_kernel<CAP><<<dim3(gx, jobs), WTC_THREADS, wtc_smem_bytes(p.n_cols), st>>>(p);
    return true;
}

template <int CAP>
void launch_wf(const WideFibParams<CAP> &p, uint64_t pairs, uint32_t jobs, cudaStream_t st) {
    if (launch_wf_tc(p, jobs, st)) return;
    // Small domains: 64-thread CTAs so that more SMs share the rows.
    const uint32_t threads = pairs < (uint64_t)device_sm_count() * 256 ? 64 : 256;
    uint64_t blocks = (pairs + threads - 1) / threads, cap = (uint64_t)device_sm_count() * 32;
    if (blocks > cap) blocks = cap;
    // n_cols <= WF_MAX_COLS: at most 2048 x 24 bytes, the default dynamic limit.
    wide_fib_kernel<CAP>
        <<<dim3((unsigned)blocks, jobs), threads, (size_t)p.n_cols * (sizeof(qm31) + sizeof(void *)), st>>>(p);
}

template <int CAP>
int wide_fib_launch(const uint32_t *const *trace, const uint32_t *const *trace_dev, uint32_t n_cols, uint32_t log_size,
                    const stwo_qm31 *powers_host, const uint32_t *powers_dev, const uint32_t *den_inv,
                    const uint32_t *den_half, uint32_t *const *out4, uint32_t jobs, size_t js, cudaStream_t st) {
    auto p = std::make_unique<WideFibParams<CAP>>();
    if (CAP > 1)
        for (uint32_t i = 0; i < n_cols; i++) {
            p->trace[i] = trace[i];
            STWO_REQUIRE(((uintptr_t)trace[i] & 15) == 0, STWO_ERR_INVALID_ARGUMENT,
                         "trace columns must be 16-byte aligned");
        }
    p->trace_dev = trace_dev;
    for (int c = 0; c < 4; c++) p->out[c] = out4[c];
    p->den_inv = den_inv;
    if (den_half) {
        p->den_half[0] = den_half[0];
        p->den_half[1] = den_half[1];
    }
    p->n_cols = n_cols;
    p->log_size = log_size;
    p->two = 2;
    p->js = js;
    p->powers_dev = reinterpret_cast<const qm31 *>(powers_dev);
    const uint64_t n = 1ull << log_size, pairs = (n + 1) / 2;
    if (powers_dev) {
        launch_wf(*p, pairs, jobs, st);
        STWO_LAUNCH_CHECK("wide_fib_kernel");
        return STWO_OK;
    }
    // Host powers: staged into a stream-ordered buffer private to this call, so
    // concurrent calls on other streams never see each other's powers.
    std::unique_ptr<qm31[]> w2(new qm31[n_cols - 2]);
    for (uint32_t i = 0; i + 2 < n_cols; i++) {
        stwo_qm31 v = powers_host[i];
        w2[i] = {{v.a, v.b}, {v.c, v.d}};
    }
    void *buf = nullptr;
    {
        int arc = pool_alloc(&buf, sizeof(qm31) * (n_cols - 2), st);
        if (arc) return arc;
    }
    cudaError_t e = cudaMemcpyAsync(buf, w2.get(), sizeof(qm31) * (n_cols - 2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        p->powers_dev = static_cast<const qm31 *>(buf);
        launch_wf(*p, pairs, 1, st);
        count_launch();
        e = cudaGetLastError();
    }
    cudaFreeAsync(buf, st);
    if (e != cudaSuccess) return set_error(STWO_ERR_CUDA, "wide_fib_kernel: %s", cudaGetErrorString(e));
    return STWO_OK;
}

}  // namespace

int accumulate_async(uint32_t *const *left4, const uint32_t *const *right4, uint64_t n, cudaStream_t st) {
    Acc4 p;
    for (int c = 0; c < 4; c++) {
        p.l[c] = left4[c];
        p.r[c] = right4[c];
        STWO_REQUIRE(((uintptr_t)p.l[c] & 15) == 0 && ((uintptr_t)p.r[c] & 15) == 0, STWO_ERR_INVALID_ARGUMENT,
                     "accumulate columns must be 16-byte aligned");
    }
    if (n == 0) return STWO_OK;
    uint64_t n4 = (n + 3) / 4;
    uint64_t blocks = (n4 + 255) / 256, cap = (uint64_t)device_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    accumulate_kernel<<<(unsigned)blocks, 256, 0, st>>>(p, n4, n);
    STWO_LAUNCH_CHECK("accumulate_kernel");
    return STWO_OK;
}

int wide_fib_async(const uint32_t *const *trace, uint32_t n_cols, uint32_t log_size, const stwo_qm31 *powers_host,
                   const uint32_t *powers_dev, const uint32_t *den_inv, uint32_t *const *out4, cudaStream_t st) {
    STWO_REQUIRE(n_cols >= 2 && n_cols <= (uint32_t)WF_MAX_COLS, STWO_ERR_UNSUPPORTED_SIZE,
                 "wide-Fibonacci composition over %u columns", n_cols);
    STWO_REQUIRE(log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "domain log size %u", log_size);
    if (n_cols < 3) {
        // No constraints: the composition is zero.
        for (int c = 0; c < 4; c++) STWO_CUDA_TRY(cudaMemsetAsync(out4[c], 0, 4ull << log_size, st));
        return STWO_OK;
    }
    if (n_cols <= 64)
        return wide_fib_launch<64>(trace, nullptr, n_cols, log_size, powers_host, powers_dev, den_inv, nullptr, out4, 1,
                                   0, st);
    if (n_cols <= 256)
        return wide_fib_launch<256>(trace, nullptr, n_cols, log_size, powers_host, powers_dev, den_inv, nullptr, out4,
                                    1, 0, st);
    return wide_fib_launch<WF_MAX_COLS>(trace, nullptr, n_cols, log_size, powers_host, powers_dev, den_inv, nullptr,
                                        out4, 1, 0, st);
}

// Same, with the trace column pointers in a device table and the powers on the device;
// the denominator inverse of a row is den_half[0] on the first half of the rows and
// den_half[1] on the second (the vanishing polynomial of a canonic coset takes one
// value on each half of its blowup-2 domain in bit-reversed order).
// jobs compositions of one shape at once: job k's tables, powers and outputs are job
// 0's moved by k * js bytes.
int wide_fib_dev_async(const uint32_t *const *trace_dev, uint32_t n_cols, uint32_t log_size, const uint32_t *powers_dev,
                       const uint32_t den_half[2], uint32_t *const *out4, uint32_t jobs, size_t js, cudaStream_t st) {
    STWO_REQUIRE(n_cols >= 3 && log_size >= 1 && log_size <= 31 && powers_dev, STWO_ERR_UNSUPPORTED_SIZE,
                 "wide-Fibonacci composition over %u columns", n_cols);
    STWO_REQUIRE(jobs >= 1 && jobs <= 65535, STWO_ERR_INVALID_ARGUMENT, "compositions per launch: %u", jobs);
    return wide_fib_launch<1>(nullptr, trace_dev, n_cols, log_size, nullptr, powers_dev, nullptr, den_half, out4, jobs,
                              js, st);
}

}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_composition_tc_faults(uint32_t *count, int reset) {
    STWO_REQUIRE(count, STWO_ERR_INVALID_ARGUMENT, "null count");
    STWO_CUDA_TRY(cudaMemcpyFromSymbol(count, g_comp_tc_faults, sizeof(uint32_t)));
    if (reset) {
        const uint32_t zero = 0;
        STWO_CUDA_TRY(cudaMemcpyToSymbol(g_comp_tc_faults, &zero, sizeof(uint32_t)));
    }
    return STWO_OK;
}

int stwo_accumulate(uint32_t *const *left4, const uint32_t *const *right4, uint64_t n, void *stream) {
    return accumulate_async(left4, right4, n, as_stream(stream));
}

void accumulate(uint32_t size, uint32_t *const *left_columns, uint32_t *const *right_columns) {
    sync_default_stream(accumulate_async(left_columns, const_cast<const uint32_t *const *>(right_columns), size, 0));
}

int stwo_wide_fib_composition(const uint32_t *const *trace, uint32_t n_columns, uint32_t ext_log_size,
                              const stwo_qm31 *coeff_powers, const uint32_t *den_inv, uint32_t *const *out4,
                              void *stream) {
    return wide_fib_async(trace, n_columns, ext_log_size, coeff_powers, nullptr, den_inv, out4, as_stream(stream));
}

void evaluate_wide_fibonacci_constraint_quotients_on_domain(
    uint32_t *quotients_0, uint32_t *quotients_1, uint32_t *quotients_2, uint32_t *quotients_3,
    uint32_t *const *trace_evaluations, const uint32_t *random_coeff_powers, const uint32_t *denominator_inverses,
    uint32_t extended_domain_size, uint32_t number_of_columns) {
    if (!is_pow2(extended_domain_size)) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "domain size %u is not a power of two", extended_domain_size);
        return;
    }
    uint32_t *out[4] = {quotients_0, quotients_1, quotients_2, quotients_3};
    sync_default_stream(wide_fib_async(const_cast<const uint32_t *const *>(trace_evaluations), number_of_columns,
                                       log2_u64(extended_domain_size), nullptr, random_coeff_powers,
                                       denominator_inverses, out, 0));
}

}  // extern "C"
