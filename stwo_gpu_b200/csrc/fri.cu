// FriOps::fold_line and FriOps::fold_circle_into_line on SoA QM31 columns.
//
// fold_line (cuda/src/fri/fold_line.cu:5-53, stwo_gpu_backend/src/fri.rs:16-43):
//   out[i] = (f[2i] + f[2i+1]) + alpha * (f[2i] - f[2i+1]) * itw[off + i]
// fold_circle_into_line (fold_circle_into_line.cu:7-69, fri.rs:45-66):
//   f' = same with the circle itwiddle of (itw + off) at i (pattern [y,-y,-x,x]),
//   dst[i] = dst[i] * alpha^2 + f'.
// Each thread folds two adjacent outputs, reading one 16-byte vector per input
// coordinate column and writing one 8-byte vector per output column.
#include "common.cuh"
#include "fri.cuh"

namespace stwo {

int small_circle_point(const uint32_t *suffix_end, uint64_t avail, uint32_t N, bool inv, uint32_t *tx, uint32_t *ty,
                       cudaStream_t st);

namespace {

struct Cols4 { const uint32_t *c[4]; };
struct MutCols4 { uint32_t *c[4]; };

// alpha_dev: when set, alpha is read from device memory (a challenge the device
// channel drew) instead of the by-value argument. JOBS: blockIdx.y is the job, whose
// columns and alpha are job 0's moved by blockIdx.y * js bytes (the twiddles are
// shared); the single-job instance carries no offset arithmetic.
template <bool CIRCLE, bool JOBS>
__global__ void fold_kernel(const __grid_constant__ Cols4 src_p, const __grid_constant__ MutCols4 dst_p, uint64_t n_out,
                            const uint32_t *__restrict__ tw, qm31 alpha, qm31 alpha_sq, const qm31 *alpha_dev,
                            size_t js) {
    // the column pointers stay in the parameter block; a job's offset is added at each
    // use (a multiply-add) rather than holding eight moved pointers in registers
    const size_t jo = JOBS ? (size_t)blockIdx.y * js : 0;
    struct {
        const Cols4 &p;
        size_t jo;
        __device__ const uint32_t *operator[](int c) const {
            return JOBS ? reinterpret_cast<const uint32_t *>(reinterpret_cast<uintptr_t>(p.c[c]) + jo) : p.c[c];
        }
    } src{src_p, jo};
    struct {
        const MutCols4 &p;
        size_t jo;
        __device__ uint32_t *operator[](int c) const {
            return JOBS ? reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(p.c[c]) + jo) : p.c[c];
        }
    } dst{dst_p, jo};
    if (JOBS) alpha_dev = job_ptr(alpha_dev, js, blockIdx.y);
    if (alpha_dev) {
        alpha = *alpha_dev;
        alpha_sq = qm31_mul(alpha, alpha);
    }
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; 2 * k < n_out;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = 2 * k;  // outputs i, i+1 <- inputs 2i .. 2i+3
        uint32_t in[4][4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            uint4 v = __ldg(reinterpret_cast<const uint4 *>(src[c]) + k);
            in[c][0] = v.x; in[c][1] = v.y; in[c][2] = v.z; in[c][3] = v.w;
        }
        qm31 f0 = {{in[0][0], in[1][0]}, {in[2][0], in[3][0]}};
        qm31 f1 = {{in[0][1], in[1][1]}, {in[2][1], in[3][1]}};
        qm31 f2 = {{in[0][2], in[1][2]}, {in[2][2], in[3][2]}};
        qm31 f3 = {{in[0][3], in[1][3]}, {in[2][3], in[3][3]}};
        uint32_t t0, t1;
        if (CIRCLE) {
            t0 = circle_itw(tw, i);
            t1 = circle_itw(tw, i + 1);
        } else {
            uint2 tt = __ldg(reinterpret_cast<const uint2 *>(tw + i));
            t0 = tt.x;
            t1 = tt.y;
        }
        qm31 r0 = fold_pair(f0, f1, t0, alpha);
        qm31 r1 = fold_pair(f2, f3, t1, alpha);
        if (CIRCLE) {
            uint2 d[4];
#pragma unroll
            for (int c = 0; c < 4; c++) d[c] = *(reinterpret_cast<const uint2 *>(dst[c]) + k);
            qm31 p0 = {{d[0].x, d[1].x}, {d[2].x, d[3].x}};
            qm31 p1 = {{d[0].y, d[1].y}, {d[2].y, d[3].y}};
            r0 = qm31_add(qm31_mul(p0, alpha_sq), r0);
            r1 = qm31_add(qm31_mul(p1, alpha_sq), r1);
        }
        *(reinterpret_cast<uint2 *>(dst[0]) + k) = make_uint2(r0.a.a, r1.a.a);
        *(reinterpret_cast<uint2 *>(dst[1]) + k) = make_uint2(r0.a.b, r1.a.b);
        *(reinterpret_cast<uint2 *>(dst[2]) + k) = make_uint2(r0.b.a, r1.b.a);
        *(reinterpret_cast<uint2 *>(dst[3]) + k) = make_uint2(r0.b.b, r1.b.b);
    }
}

// Folds with one or two outputs take their (inverse) twiddles by value: for the
// circle fold of a 2- or 4-point domain they are +-1/y of the half coset's first
// point, which the tree does not hold at those sizes (see small_circle_point).
template <bool CIRCLE>
__global__ void fold_small_kernel(const __grid_constant__ Cols4 src_p, const __grid_constant__ MutCols4 dst_p,
                                  uint32_t n_out, uint32_t t0, uint32_t t1, const uint32_t *tw, qm31 alpha,
                                  qm31 alpha_sq, const qm31 *alpha_dev, size_t js) {
    Cols4 src;
    MutCols4 dst;
    for (int c = 0; c < 4; c++) {
        src.c[c] = job_ptr(src_p.c[c], js, blockIdx.x);  // one thread a job
        dst.c[c] = job_ptr(dst_p.c[c], js, blockIdx.x);
    }
    alpha_dev = job_ptr(alpha_dev, js, blockIdx.x);
    if (alpha_dev) {
        alpha = *alpha_dev;
        alpha_sq = qm31_mul(alpha, alpha);
    }
    if (tw) {  // line fold: the inverse x twiddles are read from the tree
        t0 = tw[0];
        t1 = n_out > 1 ? tw[1] : 0u;
    }
    for (uint32_t i = 0; i < n_out; i++) {
        qm31 a = {{src.c[0][2 * i], src.c[1][2 * i]}, {src.c[2][2 * i], src.c[3][2 * i]}};
        qm31 b = {{src.c[0][2 * i + 1], src.c[1][2 * i + 1]}, {src.c[2][2 * i + 1], src.c[3][2 * i + 1]}};
        qm31 r = fold_pair(a, b, i == 0 ? t0 : t1, alpha);
        if (CIRCLE) {
            qm31 p = {{dst.c[0][i], dst.c[1][i]}, {dst.c[2][i], dst.c[3][i]}};
            r = qm31_add(qm31_mul(p, alpha_sq), r);
        }
        dst.c[0][i] = r.a.a; dst.c[1][i] = r.a.b; dst.c[2][i] = r.b.a; dst.c[3][i] = r.b.b;
    }
}

}  // namespace

// jobs folds of one shape at once: fold k's columns and alpha are fold 0's moved by
// k * js bytes; the twiddles are shared.
int fold_async(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha_c, const uint32_t *itw, uint64_t off,
               uint32_t *const *dst4, bool circle, cudaStream_t st, const void *alpha_dev, uint32_t jobs, size_t js) {
    const qm31 *ad = static_cast<const qm31 *>(alpha_dev);
    STWO_REQUIRE(jobs >= 1 && jobs <= 65535, STWO_ERR_INVALID_ARGUMENT, "folds per launch: %u", jobs);
    STWO_REQUIRE(n >= 2 && is_pow2(n), STWO_ERR_INVALID_ARGUMENT, "fold of %llu values", (unsigned long long)n);
    Cols4 s;
    MutCols4 d;
    for (int c = 0; c < 4; c++) {
        s.c[c] = src4[c];
        d.c[c] = dst4[c];
        STWO_REQUIRE(((uintptr_t)s.c[c] & 15) == 0 && ((uintptr_t)d.c[c] & 7) == 0, STWO_ERR_INVALID_ARGUMENT,
                     "fold columns must be 16-byte aligned");
    }
    qm31 alpha = {{alpha_c.a, alpha_c.b}, {alpha_c.c, alpha_c.d}};
    qm31 a2 = qm31_mul(alpha, alpha);
    const uint32_t *tw = itw + off;
    uint64_t n_out = n / 2;
    if (n_out <= 2) {
        uint32_t t[2] = {0, 0};
        if (circle) {
            uint32_t ix, iy;
            int rc = small_circle_point(tw + n / 2, off + n / 2, log2_u64(n), true, &ix, &iy, st);
            if (rc) return rc;
            t[0] = iy;
            t[1] = m31_neg(iy);
        }
        if (circle)
            fold_small_kernel<true><<<jobs, 1, 0, st>>>(s, d, (uint32_t)n_out, t[0], t[1], nullptr, alpha, a2, ad, js);
        else fold_small_kernel<false><<<jobs, 1, 0, st>>>(s, d, (uint32_t)n_out, 0u, 0u, tw, alpha, a2, ad, js);
        STWO_LAUNCH_CHECK("fold_small_kernel");
        return STWO_OK;
    }
    STWO_REQUIRE(circle || ((uintptr_t)tw & 7) == 0, STWO_ERR_INVALID_ARGUMENT,
                 "fold_line twiddle offset must be even");
    uint64_t threads = n_out / 2;
    uint32_t blocks = (uint32_t)((threads + 255) / 256);
    uint32_t cap = (uint32_t)device_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    const dim3 grid(blocks, jobs);
    if (jobs > 1) {
        if (circle) fold_kernel<true, true><<<grid, 256, 0, st>>>(s, d, n_out, tw, alpha, a2, ad, js);
        else fold_kernel<false, true><<<grid, 256, 0, st>>>(s, d, n_out, tw, alpha, a2, ad, js);
    } else {
        if (circle) fold_kernel<true, false><<<grid, 256, 0, st>>>(s, d, n_out, tw, alpha, a2, ad, 0);
        else fold_kernel<false, false><<<grid, 256, 0, st>>>(s, d, n_out, tw, alpha, a2, ad, 0);
    }
    STWO_LAUNCH_CHECK("fold_kernel");
    return STWO_OK;
}

}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_fold_line(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha, const uint32_t *itwiddles,
                   uint64_t twiddle_offset, uint32_t *const *dst4, void *stream) {
    return fold_async(src4, n, alpha, itwiddles, twiddle_offset, dst4, false, as_stream(stream), nullptr, 1, 0);
}

int stwo_fold_circle_into_line(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha, const uint32_t *itwiddles,
                               uint64_t twiddle_offset, uint32_t *const *dst4, void *stream) {
    return fold_async(src4, n, alpha, itwiddles, twiddle_offset, dst4, true, as_stream(stream), nullptr, 1, 0);
}

void fold_line(const uint32_t *gpu_domain, size_t twiddle_offset, size_t n, uint32_t *const *eval_values,
               stwo_qm31 alpha, uint32_t *const *folded_values) {
    sync_default_stream(
        fold_async(eval_values, n, alpha, gpu_domain, twiddle_offset, folded_values, false, 0, nullptr, 1, 0));
}

void fold_circle_into_line(const uint32_t *gpu_domain, size_t twiddle_offset, size_t n, uint32_t *const *eval_values,
                           stwo_qm31 alpha, uint32_t *const *folded_values) {
    sync_default_stream(
        fold_async(eval_values, n, alpha, gpu_domain, twiddle_offset, folded_values, true, 0, nullptr, 1, 0));
}

}  // extern "C"
