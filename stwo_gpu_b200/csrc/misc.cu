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
#include <memory>

#include "common.cuh"

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

template <int CAP>
void launch_wf(const WideFibParams<CAP> &p, uint64_t pairs, uint32_t jobs, cudaStream_t st) {
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
