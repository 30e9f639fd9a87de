// ColumnOps::bit_reverse_column and FieldOps::batch_inverse.
//
// Bit reversal (reference: one thread per swap with uncoalesced 4/16-byte
// accesses, cuda/src/bit_reverse.cu:6-33). Here, for n = 2^L with L >= 10, the index
// splits as (a | b | c) with a and c of 5 bits: bitrev(a|b|c) = (rev c | rev b | rev a).
// A CTA takes the 32x32 block of (a, c) for middle b and the block for rev(b),
// loads both with 128-byte row reads, and writes each transposed-and-reversed into
// the other, so every HBM access is a full line and in-place is safe.
//
// Batch inverse (reference: per-block product tree in shared memory,
// cuda/src/batch_inverse.cu:25-155). Here each warp owns 256 elements with
// coalesced accesses (lane l takes elements l, l+32, ...): prefix products in
// registers, a multiplicative scan of the lane products in both directions with
// shuffles, one field inversion of the warp product (computed by every lane, so no
// barrier is needed) and back-substitution: 3 multiplications per element and one
// inversion per 256 elements. QM31 elements are inverted through their M31 norms, so
// the scan and its products stay in M31.
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace stwo {
namespace {

template <int WORDS>
struct Elem { uint32_t w[WORDS]; };

template <int WORDS>
__global__ void bitrev_simple_kernel(Elem<WORDS> *a, uint32_t L) {
    const uint64_t n = 1ull << L;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t j = bit_reverse_bits((uint32_t)i, L);
        if (j > i) {
            Elem<WORDS> t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
}

// One CTA per (b, rev b) pair with b <= rev b; 256 threads; WORDS words per element.
template <int WORDS>
__global__ void __launch_bounds__(256) bitrev_tiled_kernel(uint32_t *a, uint32_t L, const uint32_t *pairs) {
    __shared__ uint32_t t0[32][32 * WORDS + 1];
    __shared__ uint32_t t1[32][32 * WORDS + 1];
    const uint32_t mb = L - 10;  // middle bits
    const uint32_t b0 = pairs[blockIdx.x];
    const uint32_t b1 = bit_reverse_bits(b0, mb);
    const uint32_t tid = threadIdx.x;
    // Element (a, b, c) lives at index (a << (L-5)) | (b << 5) | c.
    for (uint32_t e = tid; e < 32 * 32 * WORDS; e += 256) {
        uint32_t row = e / (32 * WORDS), col = e % (32 * WORDS);
        uint64_t base0 = (((uint64_t)row << (L - 5)) | ((uint64_t)b0 << 5)) * WORDS;
        uint64_t base1 = (((uint64_t)row << (L - 5)) | ((uint64_t)b1 << 5)) * WORDS;
        t0[row][col] = a[base0 + col];
        t1[row][col] = a[base1 + col];
    }
    __syncthreads();
    // Destination of (a, b0, c) is (rev c, rev b0 = b1, rev a): row rev c of block b1, column rev a.
    for (uint32_t e = tid; e < 32 * 32 * WORDS; e += 256) {
        uint32_t row = e / (32 * WORDS), col = e % (32 * WORDS);
        uint32_t ci = col / WORDS, w = col % WORDS;  // ci = element column within the row
        uint32_t src_row = bit_reverse_bits(ci, 5), src_c = bit_reverse_bits(row, 5);
        uint64_t base1 = (((uint64_t)row << (L - 5)) | ((uint64_t)b1 << 5)) * WORDS;
        uint64_t base0 = (((uint64_t)row << (L - 5)) | ((uint64_t)b0 << 5)) * WORDS;
        a[base1 + col] = t0[src_row][src_c * WORDS + w];
        a[base0 + col] = t1[src_row][src_c * WORDS + w];
    }
}

// ---------------------------------------------------------------- batch inverse
constexpr int BI_THREADS = 256;
constexpr int BI_PER_THREAD = 8;

template <typename F>
struct FieldT;
template <>
struct FieldT<uint32_t> {
    __device__ static uint32_t one() { return 1u; }
    __device__ static uint32_t mul(uint32_t a, uint32_t b) { return m31_mul(a, b); }
    __device__ static uint32_t inv(uint32_t a) { return m31_inv(a); }
    __device__ static uint32_t shfl_up(uint32_t v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
    __device__ static uint32_t shfl_down(uint32_t v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
};

// Warp-level Montgomery batch inverse: each warp owns 32 x BI_PER_THREAD elements,
// lane l holding elements base + i*32 + l (coalesced loads and stores). Prefix
// products in registers, inclusive scans of the lane products in both directions
// with shuffles, and one field inversion of the warp product per warp (computed
// redundantly by every lane, so there is no barrier and no shared memory).
template <typename F>
__global__ void __launch_bounds__(BI_THREADS) batch_inverse_kernel(const F *__restrict__ src, F *__restrict__ dst,
                                                                    uint64_t n) {
    using T = FieldT<F>;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp_global = ((uint64_t)blockIdx.x * BI_THREADS + threadIdx.x) >> 5;
    const uint64_t base = warp_global * (32 * BI_PER_THREAD) + lane;
    F v[BI_PER_THREAD], pre[BI_PER_THREAD];
    F run = T::one();
#pragma unroll
    for (int i = 0; i < BI_PER_THREAD; i++) {
        const uint64_t idx = base + (uint64_t)i * 32;
        v[i] = (idx < n) ? src[idx] : T::one();
        run = T::mul(run, v[i]);
        pre[i] = run;
    }
    // Inclusive scans of lane products, forward (prefix) and backward (suffix).
    F inc = run, suf = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        F u = T::shfl_up(inc, d);
        F w = T::shfl_down(suf, d);
        if (lane >= (uint32_t)d) inc = T::mul(inc, u);
        if (lane + d < 32u) suf = T::mul(suf, w);
    }
    const F total = T::shfl_down(inc, 31 - lane);  // lane 31's inclusive prefix, broadcast via shuffles
    F ex_pre = T::shfl_up(inc, 1), ex_suf = T::shfl_down(suf, 1);
    if (lane == 0) ex_pre = T::one();
    if (lane == 31) ex_suf = T::one();
    // inverse of this lane's product = inv(total) * (product before) * (product after)
    F r = T::mul(T::inv(total), T::mul(ex_pre, ex_suf));
#pragma unroll
    for (int i = BI_PER_THREAD - 1; i >= 0; i--) {
        F inv_i = i > 0 ? T::mul(r, pre[i - 1]) : r;
        const uint64_t idx = base + (uint64_t)i * 32;
        if (idx < n) dst[idx] = inv_i;
        r = T::mul(r, v[i]);
    }
}

// QM31 batch inverse through norms. For z = a + b u (a, b in CM31, u^2 = R = 2 + i):
// z (a - b u) = a^2 - R b^2 = N in CM31, and N conj(N) = |N|^2 in M31, so
// z^-1 = (a - b u) conj(N) / |N|^2. The warp's Montgomery inverse then runs on the
// M31 norms (three M31 products an element, one-word shuffles, one M31 inversion a
// warp) instead of on QM31 values (three QM31 products an element); the inverse is
// unique, so the values are the same.
__global__ void __launch_bounds__(BI_THREADS) batch_inverse_qm31_norm_kernel(const qm31 *__restrict__ src,
                                                                             qm31 *__restrict__ dst, uint64_t n) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp_global = ((uint64_t)blockIdx.x * BI_THREADS + threadIdx.x) >> 5;
    const uint64_t base = warp_global * (32 * BI_PER_THREAD) + lane;
    qm31 v[BI_PER_THREAD];
    cm31 nrm[BI_PER_THREAD];
    uint32_t pre[BI_PER_THREAD], mag[BI_PER_THREAD];
    uint32_t run = 1;
#pragma unroll
    for (int i = 0; i < BI_PER_THREAD; i++) {
        const uint64_t idx = base + (uint64_t)i * 32;
        v[i] = (idx < n) ? src[idx] : qm31_one();
        const cm31 a2 = cm31_sqr(v[i].a), b2 = cm31_sqr(v[i].b);
        const cm31 rb2 = {m31_sub(m31_add(b2.a, b2.a), b2.b), m31_add(m31_add(b2.b, b2.b), b2.a)};  // R b^2
        nrm[i] = cm31_sub(a2, rb2);
        mag[i] = reduce64_p((uint64_t)nrm[i].a * nrm[i].a + (uint64_t)nrm[i].b * nrm[i].b);
        run = m31_mul(run, mag[i]);
        pre[i] = run;
    }
    // Inclusive scans of the lanes' norm products, forward (prefix) and backward (suffix).
    uint32_t inc = run, suf = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, inc, d);
        const uint32_t w = __shfl_down_sync(0xffffffffu, suf, d);
        if (lane >= (uint32_t)d) inc = m31_mul(inc, u);
        if (lane + d < 32u) suf = m31_mul(suf, w);
    }
    const uint32_t total = __shfl_down_sync(0xffffffffu, inc, 31 - lane);
    uint32_t ex_pre = __shfl_up_sync(0xffffffffu, inc, 1), ex_suf = __shfl_down_sync(0xffffffffu, suf, 1);
    if (lane == 0) ex_pre = 1;
    if (lane == 31) ex_suf = 1;
    uint32_t r = m31_mul(m31_inv(total), m31_mul(ex_pre, ex_suf));
#pragma unroll
    for (int i = BI_PER_THREAD - 1; i >= 0; i--) {
        const uint32_t minv = i > 0 ? m31_mul(r, pre[i - 1]) : r;  // 1 / |N_i|^2
        const uint64_t idx = base + (uint64_t)i * 32;
        r = m31_mul(r, mag[i]);
        // 1 / N_i = c + d i with c = N.a / |N|^2, d = -N.b / |N|^2; the products
        // (x + y i)(c + d i) = (x c + y (p - d)) + (x d + y c) i reduced once each
        const uint32_t c = m31_mul(nrm[i].a, minv), nd = m31_mul(nrm[i].b, minv), d = m31_neg(nd);
        const qm31 z = v[i];
        const cm31 lo = {reduce64_p((uint64_t)z.a.a * c + (uint64_t)z.a.b * nd),
                         reduce64_p((uint64_t)z.a.a * d + (uint64_t)z.a.b * c)};
        const cm31 hi = {reduce64_p((uint64_t)z.b.a * c + (uint64_t)z.b.b * nd),
                         reduce64_p((uint64_t)z.b.a * d + (uint64_t)z.b.b * c)};
        if (idx < n) dst[idx] = {lo, cm31_neg(hi)};
    }
}

}  // namespace

int bit_reverse_async(uint32_t *col, uint64_t n, uint32_t words, cudaStream_t st) {
    STWO_REQUIRE(is_pow2(n) && n <= (1ull << 31), STWO_ERR_INVALID_ARGUMENT, "bit reverse of %llu elements",
                 (unsigned long long)n);
    STWO_REQUIRE(words == 1 || words == 4, STWO_ERR_INVALID_ARGUMENT, "element of %u words", words);
    uint32_t L = log2_u64(n);
    if (L < 10) {
        uint32_t blocks = (uint32_t)((n + 255) / 256);
        if (words == 1) bitrev_simple_kernel<1><<<blocks, 256, 0, st>>>(reinterpret_cast<Elem<1> *>(col), L);
        else bitrev_simple_kernel<4><<<blocks, 256, 0, st>>>(reinterpret_cast<Elem<4> *>(col), L);
        STWO_LAUNCH_CHECK("bitrev_simple_kernel");
        return STWO_OK;
    }
    // Middle indices b with b <= rev(b): built on the host once per device and size, and
    // cached (the cache is shared by all threads and streams, under a lock).
    static std::mutex mu;
    static std::map<std::pair<int, uint32_t>, std::pair<uint32_t *, uint32_t>> cache;
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    uint32_t *pairs = nullptr, cnt = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find({dev, L});
        if (it == cache.end()) {
            uint32_t mb = L - 10, m = 1u << mb;
            std::vector<uint32_t> h;
            h.reserve(m);
            for (uint32_t b = 0; b < m; b++)
                if (b <= bit_reverse_bits(b, mb)) h.push_back(b);
            uint32_t *d = nullptr;
            cudaError_t e = cudaMalloc(&d, sizeof(uint32_t) * h.size());
            if (e == cudaSuccess) e = cudaMemcpy(d, h.data(), sizeof(uint32_t) * h.size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return set_error(STWO_ERR_CUDA, "bit reverse table: %s", cudaGetErrorString(e));
            it = cache.emplace(std::make_pair(dev, L), std::make_pair(d, (uint32_t)h.size())).first;
        }
        pairs = it->second.first;
        cnt = it->second.second;
    }
    if (words == 1) bitrev_tiled_kernel<1><<<cnt, 256, 0, st>>>(col, L, pairs);
    else bitrev_tiled_kernel<4><<<cnt, 256, 0, st>>>(col, L, pairs);
    STWO_LAUNCH_CHECK("bitrev_tiled_kernel");
    return STWO_OK;
}

int batch_inverse_m31_async(const uint32_t *src, uint32_t *dst, uint64_t n, cudaStream_t st) {
    if (n == 0) return STWO_OK;
    uint64_t blocks = (n + BI_THREADS * BI_PER_THREAD - 1) / (BI_THREADS * BI_PER_THREAD);
    batch_inverse_kernel<uint32_t><<<(unsigned)blocks, BI_THREADS, 0, st>>>(src, dst, n);
    STWO_LAUNCH_CHECK("batch_inverse_kernel<m31>");
    return STWO_OK;
}

int batch_inverse_qm31_async(const uint32_t *src, uint32_t *dst, uint64_t n, cudaStream_t st) {
    if (n == 0) return STWO_OK;
    uint64_t blocks = (n + BI_THREADS * BI_PER_THREAD - 1) / (BI_THREADS * BI_PER_THREAD);
    batch_inverse_qm31_norm_kernel<<<(unsigned)blocks, BI_THREADS, 0, st>>>(reinterpret_cast<const qm31 *>(src),
                                                                            reinterpret_cast<qm31 *>(dst), n);
    STWO_LAUNCH_CHECK("batch_inverse_qm31_norm_kernel");
    return STWO_OK;
}

}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_bit_reverse_m31(uint32_t *column, uint64_t n, void *stream) {
    return bit_reverse_async(column, n, 1, as_stream(stream));
}
int stwo_bit_reverse_qm31(uint32_t *column, uint64_t n, void *stream) {
    return bit_reverse_async(column, n, 4, as_stream(stream));
}
int stwo_batch_inverse_m31(const uint32_t *src, uint32_t *dst, uint64_t n, void *stream) {
    return batch_inverse_m31_async(src, dst, n, as_stream(stream));
}
int stwo_batch_inverse_qm31(const uint32_t *src, uint32_t *dst, uint64_t n, void *stream) {
    return batch_inverse_qm31_async(src, dst, n, as_stream(stream));
}

void bit_reverse_base_field(uint32_t *array, size_t size) { sync_default_stream(bit_reverse_async(array, size, 1, 0)); }
void bit_reverse_secure_field(uint32_t *array, size_t size) { sync_default_stream(bit_reverse_async(array, size, 4, 0)); }
void batch_inverse_base_field(const uint32_t *from, uint32_t *dst, size_t size) {
    sync_default_stream(batch_inverse_m31_async(from, dst, size, 0));
}
void batch_inverse_secure_field(const uint32_t *from, uint32_t *dst, size_t size) {
    sync_default_stream(batch_inverse_qm31_async(from, dst, size, 0));
}

}  // extern "C"
