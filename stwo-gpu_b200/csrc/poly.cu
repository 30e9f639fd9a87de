// PolyOps entry points: twiddle trees, canonic -> bit-reversed reordering,
// interpolate / evaluate (reference-compatible and native), eval_at_point.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace stwo {

int fft_columns(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st);
int batch_inverse_m31_async(const uint32_t *src, uint32_t *dst, uint64_t n, cudaStream_t st);
int bit_reverse_async(uint32_t *col, uint64_t n, uint32_t words, cudaStream_t st);

namespace {

// ------------------------------------------------------------------ twiddles
// Tree layer j of root coset (I, S, m): entries h < 2^(m-j-1) at offset
// 2^m - 2^(m-j) hold x(I^(2^j) * S^(2^j * bitrev_{m-j-1}(h))) (twiddles.cu:29-73).
// Points are products of table entries: pows[b] = S^(2^b), inits[j] = I^(2^j).
struct TwiddleParams {
    cpoint pows[32];
    cpoint inits[32];
    uint32_t m;
};

__global__ void twiddle_tree_kernel(const __grid_constant__ TwiddleParams p, uint32_t *tw) {
    const uint64_t size = 1ull << p.m;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i + 1 < size;
         i += (uint64_t)gridDim.x * blockDim.x) {
        // layer j: offset 2^m - 2^(m-j) <= i < 2^m - 2^(m-j-1)
        uint32_t j = 0;
        while (i >= size - (size >> (j + 1))) j++;
        uint64_t off = size - (size >> j);
        uint32_t hl = p.m - j - 1;
        uint32_t e = bit_reverse_bits((uint32_t)(i - off), hl);
        cpoint r = p.inits[j];
        for (uint32_t b = 0; b < hl; b++)
            if ((e >> b) & 1u) r = point_mul(r, p.pows[b + j]);
        tw[i] = r.x;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) tw[size - 1] = 1u;
}

int precompute_tree(cpoint initial, cpoint step, uint32_t m, uint32_t *tw, uint32_t *itw, cudaStream_t st) {
    STWO_REQUIRE(m <= 30, STWO_ERR_UNSUPPORTED_SIZE, "root coset of log size %u unsupported", m);
    STWO_REQUIRE(tw || itw, STWO_ERR_INVALID_ARGUMENT, "no output buffer");
    TwiddleParams p{};
    p.m = m;
    cpoint s = step, ini = initial;
    for (uint32_t b = 0; b < 32; b++) {
        p.pows[b] = s;
        p.inits[b] = ini;
        s = point_mul(s, s);
        ini = point_mul(ini, ini);
    }
    uint64_t size = 1ull << m;
    uint32_t *dst = tw;
    uint32_t *tmp = nullptr;
    if (!dst) {
        int arc = pool_alloc((void **)&tmp, size * 4, st);
        if (arc) return arc;
        dst = tmp;
    }
    uint32_t blocks = (uint32_t)std::min<uint64_t>((size + 255) / 256, (uint64_t)device_sm_count() * 16);
    twiddle_tree_kernel<<<std::max(1u, blocks), 256, 0, st>>>(p, dst);
    STWO_LAUNCH_CHECK("twiddle_tree_kernel");
    int rc = STWO_OK;
    if (itw) rc = batch_inverse_m31_async(dst, itw, size, st);
    if (tmp) cudaFreeAsync(tmp, st);
    return rc;
}

// ------------------------------------------------------------------ canonic order
// new_canonical_ordered (twiddles.cu:4-27): position br(q) <- src[2q] for q < n/2,
// src[n - 1 - 2(q - n/2)] otherwise; written as a gather over output positions.
__global__ void canonic_to_bitrev_kernel(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, uint32_t L) {
    const uint64_t n = 1ull << L, half = n >> 1;
    for (uint64_t pos = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; pos < n; pos += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t q = bit_reverse_bits((uint32_t)pos, L);
        uint64_t s = q < half ? (q << 1) : (n - 1 - ((q - half) << 1));
        dst[pos] = __ldg(src + s);
    }
}

// ------------------------------------------------------------------ eval_at_point
// p(P) = sum_i c_i prod_{bit b of i} f_b with f_0 = y, f_1 = x, f_b = pi^(b-1)(x),
// pi(x) = 2x^2 - 1 (eval_at_point.cu:99-109). A CTA folds a chunk of 2^15
// coefficients as 4 groups of 8192: a thread takes 32 consecutive coefficients (bits
// 0..4) and forms sum_i c_i F_i against the CTA's table F_i = prod_{b in i} f_b, an
// M31-by-QM31 dot product of 64-bit multiply-accumulates; the lanes fold bits 5..9
// and the warps bits 10..12. Group partials are weighted by their group index's
// factors (bits 13..14) before the lane fold, which is linear, so one fold serves the
// whole chunk. The chunk partial takes the factors of its chunk index; the last CTA
// of each polynomial (atomic ticket) adds the partials.
constexpr int EAP_THREADS = 256;
constexpr int EAP_PER_THREAD_LOG = 5;                    // 32 coefficients per thread
constexpr int EAP_GROUP_LOG = EAP_PER_THREAD_LOG + 8;    // x 256 threads
constexpr int EAP_ITER_LOG = 2;                          // groups per CTA: 4
constexpr int EAP_CHUNK_LOG = EAP_GROUP_LOG + EAP_ITER_LOG;
constexpr int EAP_MAX_POLYS = 32;

struct EapParams {
    const uint32_t *coeffs[EAP_MAX_POLYS];
    qm31 factors[EAP_MAX_POLYS][32];
    uint32_t log_size[EAP_MAX_POLYS];
    uint32_t block_start[EAP_MAX_POLYS + 1];  // prefix sum of CTAs per polynomial
    uint32_t n_polys;
    qm31 *partials;                            // one per CTA
    uint32_t *tickets;                         // one per polynomial, zero on entry, reset on exit
    qm31 *results;
};

__device__ __forceinline__ qm31 shfl_xor_q(qm31 v, int m) {
    v.a.a = __shfl_xor_sync(0xffffffffu, v.a.a, m);
    v.a.b = __shfl_xor_sync(0xffffffffu, v.a.b, m);
    v.b.a = __shfl_xor_sync(0xffffffffu, v.b.a, m);
    v.b.b = __shfl_xor_sync(0xffffffffu, v.b.b, m);
    return v;
}

// One CTA's share of polynomial `poly`: chunk `chunk` of its 2^L coefficients c with
// factors f; its CTAs are blk_first .. blk_first + nblk - 1 (partials indexed by CTA).
__device__ __forceinline__ void eap_body(uint32_t poly, uint32_t chunk, uint32_t L, const qm31 *f, const uint32_t *c,
                                         uint32_t blk_first, uint32_t nblk, qm31 *partials, uint32_t *tickets,
                                         qm31 *results) {
    __shared__ qm31 warp_vals[EAP_THREADS / 32];
    __shared__ qm31 g[1 << EAP_ITER_LOG];
    __shared__ qm31 F2[1 << EAP_PER_THREAD_LOG];  // F_i
    __shared__ bool is_last;
    const uint32_t tid = threadIdx.x;
    const uint64_t n = 1ull << L;
    if (tid < (1u << EAP_PER_THREAD_LOG)) {
        qm31 w = qm31_one();
        for (int b = 0; b < EAP_PER_THREAD_LOG; b++)
            if ((tid >> b) & 1u) w = qm31_mul(w, f[b]);
        F2[tid] = w;
    } else if (tid < (1u << EAP_PER_THREAD_LOG) + (1u << EAP_ITER_LOG)) {
        // group weights: products of f_{13+b} over the set bits b of the group index
        const uint32_t it = tid - (1u << EAP_PER_THREAD_LOG);
        qm31 w = qm31_one();
        for (int b = 0; b < EAP_ITER_LOG; b++)
            if ((it >> b) & 1u) w = qm31_mul(w, f[EAP_GROUP_LOG + b]);
        g[it] = w;
    }
    __syncthreads();

    qm31 acc = qm31_zero();
    for (uint32_t it = 0; it < (1u << EAP_ITER_LOG); it++) {
        const uint64_t base = ((uint64_t)chunk << EAP_CHUNK_LOG) + ((uint64_t)it << EAP_GROUP_LOG) +
                              ((uint64_t)tid << EAP_PER_THREAD_LOG);
        if (base >= n) break;
        uint64_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        // 64-bit multiply-accumulates of canonical values, folded after every third term
        auto term = [&](uint32_t v, uint32_t i) {
            const qm31 w = F2[i];
            s0 = mac64(s0, v, w.a.a);
            s1 = mac64(s1, v, w.a.b);
            s2 = mac64(s2, v, w.b.a);
            s3 = mac64(s3, v, w.b.b);
            if (i % 3 == 2) {
                s0 = fold64(s0);
                s1 = fold64(s1);
                s2 = fold64(s2);
                s3 = fold64(s3);
            }
        };
        if (base + 32 <= n) {
            const uint4 *q = reinterpret_cast<const uint4 *>(c + base);
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const uint4 x = __ldg(q + u);
                term(x.x, 4 * u);
                term(x.y, 4 * u + 1);
                term(x.z, 4 * u + 2);
                term(x.w, 4 * u + 3);
            }
        } else {
            for (uint32_t i = 0; base + i < n && i < 32; i++) term(__ldg(c + base + i), i);
        }
        const qm31 part = {{reduce64_p(s0), reduce64_p(s1)}, {reduce64_p(s2), reduce64_p(s3)}};
        acc = qm31_add(acc, it == 0 ? part : qm31_mul(part, g[it]));
    }
    // Across lanes: bits 5..9 (lane bit j <-> factor 5 + j).
    const uint32_t lane = tid & 31u;
#pragma unroll
    for (int j = 0; j < 5; j++) {
        qm31 other = shfl_xor_q(acc, 1 << j);
        // lane with bit j clear keeps lo + hi * f; the other result is discarded.
        qm31 lo = (lane >> j) & 1u ? other : acc;
        qm31 hi = (lane >> j) & 1u ? acc : other;
        acc = qm31_add(lo, qm31_mul(hi, f[EAP_PER_THREAD_LOG + j]));
    }
    if (lane == 0) warp_vals[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        // Warps: bits 10..12.
        qm31 w[8];
        for (int i = 0; i < 8; i++) w[i] = warp_vals[i];
        for (int lvl = 0; lvl < 3; lvl++)
            for (int i = 0; i < (8 >> (lvl + 1)); i++)
                w[i] = qm31_add(w[2 * i], qm31_mul(w[2 * i + 1], f[EAP_PER_THREAD_LOG + 5 + lvl]));
        qm31 s = w[0];
        // Chunk index bits -> factors 15.. .
        for (uint32_t b = 0; EAP_CHUNK_LOG + b < L; b++)
            if ((chunk >> b) & 1u) s = qm31_mul(s, f[EAP_CHUNK_LOG + b]);
        partials[blockIdx.x] = s;
        __threadfence();
        uint32_t t = atomicAdd(&tickets[poly], 1u);
        is_last = (t == nblk - 1);
    }
    __syncthreads();
    if (is_last) {
        // The whole last CTA sums the partials: strided per thread, then across lanes
        // and warps (field addition, so the order does not change the sum).
        __threadfence();
        qm31 s = qm31_zero();
        for (uint32_t b = blk_first + tid; b < blk_first + nblk; b += EAP_THREADS) {
            qm31 v;
            const volatile uint32_t *pv = reinterpret_cast<const volatile uint32_t *>(&partials[b]);
            v.a.a = pv[0]; v.a.b = pv[1]; v.b.a = pv[2]; v.b.b = pv[3];
            s = qm31_add(s, v);
        }
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) s = qm31_add(s, shfl_xor_q(s, m));
        if (lane == 0) warp_vals[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) {
            qm31 t = qm31_zero();
            for (int i = 0; i < EAP_THREADS / 32; i++) t = qm31_add(t, warp_vals[i]);
            results[poly] = t;
            tickets[poly] = 0;  // ready for the next launch
        }
    }
}

__global__ void __launch_bounds__(EAP_THREADS) eval_at_point_kernel(const __grid_constant__ EapParams p) {
    uint32_t poly = 0;
    while (poly + 1 < p.n_polys && blockIdx.x >= p.block_start[poly + 1]) poly++;
    eap_body(poly, blockIdx.x - p.block_start[poly], p.log_size[poly], p.factors[poly], p.coeffs[poly],
             p.block_start[poly], p.block_start[poly + 1] - p.block_start[poly], p.partials, p.tickets, p.results);
}

// Polynomials described in device memory, all evaluated at one point also in device
// memory (x then y); each CTA derives its polynomial's factors itself.
struct EapDevPoly {
    const uint32_t *coeffs;
    uint32_t log_size;
    uint32_t block_start;  // first CTA of the polynomial
};

__global__ void __launch_bounds__(EAP_THREADS) eval_at_point_dev_kernel(const EapDevPoly *__restrict__ polys,
                                                                        uint32_t n_polys, const qm31 *point,
                                                                        qm31 *partials, uint32_t *tickets,
                                                                        qm31 *results) {
    __shared__ qm31 f[32];
    // the last polynomial whose first CTA is <= blockIdx.x
    uint32_t lo = 0, hi = n_polys - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) / 2;
        if (polys[mid].block_start <= blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const EapDevPoly d = polys[lo];
    const uint32_t next = lo + 1 < n_polys ? polys[lo + 1].block_start : gridDim.x;
    if (threadIdx.x == 0) {
        // f_0 = y, f_1 = x, f_b = pi^(b-1)(x)
        f[0] = point[1];
        qm31 x = point[0];
        for (uint32_t b = 1; b < 32; b++) {
            f[b] = x;
            qm31 sq = qm31_mul(x, x);
            x = qm31_sub(qm31_add(sq, sq), qm31_one());
        }
    }
    __syncthreads();
    eap_body(lo, blockIdx.x - d.block_start, d.log_size, f, d.coeffs, d.block_start, next - d.block_start, partials,
             tickets, results);
}


inline qm31 to_q(stwo_qm31 v) { return {{v.a, v.b}, {v.c, v.d}}; }
inline stwo_qm31 from_q(qm31 v) { return {v.a.a, v.a.b, v.b.a, v.b.b}; }

void eap_factors(qm31 *f, stwo_spoint pt, uint32_t L) {
    // f_0 = y, f_1 = x, f_b = pi^(b-1)(x)
    for (uint32_t b = 0; b < 32; b++) f[b] = qm31_zero();
    f[0] = to_q(pt.y);
    qm31 x = to_q(pt.x);
    for (uint32_t b = 1; b < std::max<uint32_t>(L, 2u) && b < 32; b++) {
        f[b] = x;
        qm31 sq = qm31_mul(x, x);
        x = qm31_sub(qm31_add(sq, sq), qm31_one());
    }
}

uint32_t eap_blocks(uint32_t L) { return L <= (uint32_t)EAP_CHUNK_LOG ? 1u : 1u << (L - EAP_CHUNK_LOG); }

}  // namespace

size_t eval_at_points_scratch_bytes(const uint32_t *log_sizes, uint32_t n_polys) {
    size_t blocks = 0;
    for (uint32_t i = 0; i < n_polys; i++) blocks += eap_blocks(log_sizes[i]);
    return blocks * sizeof(qm31) + ((size_t)n_polys * 4 + 15) / 16 * 16 + 256;
}

// scratch: partials followed by zeroed tickets (the kernel leaves them zero).
int eval_at_points_async(const uint32_t *const *coeffs, const uint32_t *log_sizes, uint32_t n_polys,
                         const stwo_spoint *points, stwo_qm31 *results, void *scratch, size_t scratch_bytes,
                         bool tickets_zeroed, cudaStream_t st) {
    STWO_REQUIRE(scratch_bytes >= eval_at_points_scratch_bytes(log_sizes, n_polys), STWO_ERR_INVALID_ARGUMENT,
                 "eval_at_point scratch too small");
    size_t blocks_total = 0;
    for (uint32_t i = 0; i < n_polys; i++) {
        STWO_REQUIRE(log_sizes[i] <= 30, STWO_ERR_UNSUPPORTED_SIZE, "polynomial of log size %u unsupported", log_sizes[i]);
        blocks_total += eap_blocks(log_sizes[i]);
    }
    uint32_t *tickets = reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) + blocks_total * sizeof(qm31));
    if (!tickets_zeroed) STWO_CUDA_TRY(cudaMemsetAsync(tickets, 0, (size_t)n_polys * 4, st));
    qm31 *partials = static_cast<qm31 *>(scratch);
    uint32_t done = 0;
    size_t part_off = 0;
    while (done < n_polys) {
        EapParams p{};
        uint32_t cnt = std::min<uint32_t>(EAP_MAX_POLYS, n_polys - done);
        uint32_t b = 0;
        for (uint32_t i = 0; i < cnt; i++) {
            uint32_t L = log_sizes[done + i];
            p.coeffs[i] = coeffs[done + i];
            p.log_size[i] = L;
            eap_factors(p.factors[i], points[done + i], L);
            p.block_start[i] = b;
            b += eap_blocks(L);
        }
        p.block_start[cnt] = b;
        p.n_polys = cnt;
        p.partials = partials + part_off;
        p.tickets = tickets + done;
        p.results = reinterpret_cast<qm31 *>(results) + done;
        eval_at_point_kernel<<<b, EAP_THREADS, 0, st>>>(p);
        STWO_LAUNCH_CHECK("eval_at_point_kernel");
        part_off += b;
        done += cnt;
    }
    return STWO_OK;
}

// eval_at_point for polynomials described in device memory (polys_dev: n_polys
// EapDevPoly), at the device point point_dev (QM31 x then y). partials: total_blocks
// QM31; tickets: n_polys zeroed words (left zeroed).
int eval_at_points_dev_async(const void *polys_dev, uint32_t n_polys, uint32_t total_blocks, const void *point_dev,
                             void *results, void *partials, uint32_t *tickets, cudaStream_t st) {
    STWO_REQUIRE(n_polys >= 1 && total_blocks >= n_polys, STWO_ERR_INVALID_ARGUMENT, "eval_at_point descriptors");
    eval_at_point_dev_kernel<<<total_blocks, EAP_THREADS, 0, st>>>(
        static_cast<const EapDevPoly *>(polys_dev), n_polys, static_cast<const qm31 *>(point_dev),
        static_cast<qm31 *>(partials), tickets, static_cast<qm31 *>(results));
    STWO_LAUNCH_CHECK("eval_at_point_dev_kernel");
    return STWO_OK;
}

uint32_t eval_at_point_blocks(uint32_t log_size) { return eap_blocks(log_size); }

int extend_evaluate_async(const uint32_t *const *coeffs, const uint32_t *coeff_logs, uint32_t *const *outs,
                          uint32_t log_blowup, uint32_t n, const uint32_t *tw, uint64_t tree_size, cudaStream_t st) {
    // Group columns by size so each size is one launch sequence.
    std::map<uint32_t, std::vector<uint32_t>> by_size;
    for (uint32_t i = 0; i < n; i++) by_size[coeff_logs[i]].push_back(i);
    for (auto &kv : by_size) {
        std::vector<const uint32_t *> s;
        std::vector<uint32_t *> d;
        for (uint32_t i : kv.second) {
            s.push_back(coeffs[i]);
            d.push_back(outs[i]);
        }
        uint32_t L = kv.first, N = L + log_blowup;
        int rc;
        if (L == N || N <= 2) {
            // No extension (or a tiny one): copy then transform in place.
            for (size_t i = 0; i < s.size(); i++) {
                if (s[i] != d[i]) STWO_CUDA_TRY(cudaMemcpyAsync(d[i], s[i], 4ull << L, cudaMemcpyDeviceToDevice, st));
                if (N > L) STWO_CUDA_TRY(cudaMemsetAsync(d[i] + (1ull << L), 0, (4ull << N) - (4ull << L), st));
            }
            rc = fft_columns(d.data(), d.data(), (uint32_t)d.size(), N, N, tw, tree_size, false, st);
        } else {
            rc = fft_columns(s.data(), d.data(), (uint32_t)d.size(), N, L, tw, tree_size, false, st);
        }
        if (rc) return rc;
    }
    return STWO_OK;
}

int columns_fft_async(uint32_t *const *cols, const uint32_t *logs, uint32_t n, const uint32_t *tree,
                      uint64_t tree_size, bool inv, cudaStream_t st) {
    std::map<uint32_t, std::vector<uint32_t *>> by_size;
    for (uint32_t i = 0; i < n; i++) by_size[logs[i]].push_back(cols[i]);
    for (auto &kv : by_size) {
        int rc = fft_columns(kv.second.data(), kv.second.data(), (uint32_t)kv.second.size(), kv.first, kv.first,
                             tree, tree_size, inv, st);
        if (rc) return rc;
    }
    return STWO_OK;
}

}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_precompute_twiddles(uint32_t root_initial_index, uint32_t root_step_size, uint32_t root_log_size,
                             uint32_t *twiddles, uint32_t *itwiddles, void *stream) {
    return precompute_tree(index_to_point(root_initial_index), index_to_point(root_step_size), root_log_size,
                           twiddles, itwiddles, as_stream(stream));
}

uint32_t *precompute_twiddles(stwo_point initial, stwo_point step, size_t total_size) {
    if (!is_pow2(total_size)) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "twiddle tree size %zu is not a power of two", total_size);
        return nullptr;
    }
    uint32_t *tw = cuda_malloc_uint32_t((uint32_t)total_size);
    if (!tw) return nullptr;
    int rc = precompute_tree({initial.x, initial.y}, {step.x, step.y}, log2_u64(total_size), tw, nullptr, 0);
    if (sync_default_stream(rc) != STWO_OK) {
        cudaFree(tw);
        return nullptr;
    }
    return tw;
}

int stwo_new_canonical_ordered(const uint32_t *src, uint32_t *dst, uint32_t log_size, void *stream) {
    STWO_REQUIRE(log_size >= 1 && log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "log size %u unsupported", log_size);
    STWO_REQUIRE(src != dst, STWO_ERR_INVALID_ARGUMENT, "new_canonical_ordered is out of place");
    uint64_t n = 1ull << log_size;
    uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)device_sm_count() * 32);
    canonic_to_bitrev_kernel<<<blocks, 256, 0, as_stream(stream)>>>(src, dst, log_size);
    STWO_LAUNCH_CHECK("canonic_to_bitrev_kernel");
    return STWO_OK;
}

uint32_t *sort_values_and_permute_with_bit_reverse_order(const uint32_t *from, size_t size) {
    if (!is_pow2(size) || size < 2) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "size %zu is not a power of two >= 2", size);
        return nullptr;
    }
    uint32_t *dst = cuda_malloc_uint32_t((uint32_t)size);
    if (!dst) return nullptr;
    if (sync_default_stream(stwo_new_canonical_ordered(from, dst, log2_u64(size), nullptr)) != STWO_OK) {
        cudaFree(dst);
        return nullptr;
    }
    return dst;
}

int stwo_interpolate_columns(uint32_t *const *columns, const uint32_t *log_sizes, uint32_t n_columns,
                             const uint32_t *itwiddles, uint64_t tree_size, void *stream) {
    return columns_fft_async(columns, log_sizes, n_columns, itwiddles, tree_size, true, as_stream(stream));
}

int stwo_evaluate_columns(uint32_t *const *columns, const uint32_t *log_sizes, uint32_t n_columns,
                          const uint32_t *twiddles, uint64_t tree_size, void *stream) {
    return columns_fft_async(columns, log_sizes, n_columns, twiddles, tree_size, false, as_stream(stream));
}

int stwo_extend_evaluate_columns(const uint32_t *const *coeffs, const uint32_t *coeff_log_sizes,
                                 uint32_t *const *outputs, uint32_t log_blowup, uint32_t n_columns,
                                 const uint32_t *twiddles, uint64_t tree_size, void *stream) {
    for (uint32_t i = 0; i < n_columns; i++)
        STWO_REQUIRE(log_blowup == 0 || coeffs[i] != outputs[i], STWO_ERR_INVALID_ARGUMENT,
                     "extend_evaluate needs distinct coefficient and output buffers");
    return extend_evaluate_async(coeffs, coeff_log_sizes, outputs, log_blowup, n_columns, twiddles, tree_size,
                                 as_stream(stream));
}

// Reference-compatible forms: eval_domain_size is the half-coset size, i.e. half
// of values_size; the column is transformed in place (ifft.cu:41-65, rfft.cu:45-64).
void interpolate(uint32_t eval_domain_size, uint32_t *values, const uint32_t *inverse_twiddles_tree,
                 uint32_t inverse_twiddle_tree_size, uint32_t values_size) {
    (void)eval_domain_size;
    if (!is_pow2(values_size) || values_size < 2) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "values_size %u is not a power of two >= 2", values_size);
        return;
    }
    uint32_t L = log2_u64(values_size);
    sync_default_stream(columns_fft_async(&values, &L, 1, inverse_twiddles_tree, inverse_twiddle_tree_size, true, 0));
}

void interpolate_columns(uint32_t eval_domain_size, uint32_t *const *values, const uint32_t *inverse_twiddles_tree,
                         uint32_t inverse_twiddle_tree_size, uint32_t values_size, uint32_t number_of_rows) {
    (void)eval_domain_size;
    if (!is_pow2(number_of_rows) || number_of_rows < 2) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "number_of_rows %u is not a power of two >= 2", number_of_rows);
        return;
    }
    std::vector<uint32_t> logs(values_size, log2_u64(number_of_rows));
    sync_default_stream(columns_fft_async(values, logs.data(), values_size, inverse_twiddles_tree,
                                          inverse_twiddle_tree_size, true, 0));
}

void evaluate(uint32_t eval_domain_size, uint32_t *values, const uint32_t *twiddles_tree, uint32_t twiddle_tree_size,
              uint32_t values_size) {
    (void)eval_domain_size;
    if (!is_pow2(values_size) || values_size < 2) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "values_size %u is not a power of two >= 2", values_size);
        return;
    }
    uint32_t L = log2_u64(values_size);
    sync_default_stream(columns_fft_async(&values, &L, 1, twiddles_tree, twiddle_tree_size, false, 0));
}

void evaluate_columns(const uint32_t *eval_domain_sizes, uint32_t *const *values, const uint32_t *twiddles_tree,
                      uint32_t twiddle_tree_size, uint32_t number_of_columns, const uint32_t *column_sizes) {
    (void)eval_domain_sizes;
    std::vector<uint32_t> logs(number_of_columns);
    for (uint32_t i = 0; i < number_of_columns; i++) {
        if (!is_pow2(column_sizes[i]) || column_sizes[i] < 2) {
            set_error(STWO_ERR_INVALID_ARGUMENT, "column size %u is not a power of two >= 2", column_sizes[i]);
            return;
        }
        logs[i] = log2_u64(column_sizes[i]);
    }
    sync_default_stream(columns_fft_async(values, logs.data(), number_of_columns, twiddles_tree, twiddle_tree_size,
                                          false, 0));
}

size_t stwo_eval_at_points_scratch_bytes(const uint32_t *log_sizes, uint32_t n_polys) {
    return eval_at_points_scratch_bytes(log_sizes, n_polys);
}

int stwo_eval_at_points(const uint32_t *const *coeffs, const uint32_t *log_sizes, uint32_t n_polys,
                        const stwo_spoint *points, stwo_qm31 *results, void *scratch, size_t scratch_bytes,
                        void *stream) {
    return eval_at_points_async(coeffs, log_sizes, n_polys, points, results, scratch, scratch_bytes, false,
                                as_stream(stream));
}

// Reference-compatible: allocates its scratch per call, as eval_at_point.cu:118 does.
stwo_qm31 eval_at_point(const uint32_t *coeffs, uint32_t coeffs_size, stwo_qm31 point_x, stwo_qm31 point_y) {
    stwo_qm31 out = {0, 0, 0, 0};
    if (!is_pow2(coeffs_size)) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "coeffs_size %u is not a power of two", coeffs_size);
        return out;
    }
    uint32_t L = log2_u64(coeffs_size);
    stwo_spoint pt = {point_x, point_y};
    const size_t need = eval_at_points_scratch_bytes(&L, 1);
    char *scratch = nullptr;
    if (cudaMalloc((void **)&scratch, need + 256) != cudaSuccess) {
        set_error(STWO_ERR_OUT_OF_MEMORY, "eval_at_point scratch allocation failed");
        return out;
    }
    stwo_qm31 *res = reinterpret_cast<stwo_qm31 *>(scratch);  // result slot, then the kernel scratch
    int rc = eval_at_points_async(&coeffs, &L, 1, &pt, res, scratch + 256, need, false, 0);
    if (rc == STWO_OK) {
        if (cudaMemcpy(&out, res, sizeof(out), cudaMemcpyDeviceToHost) != cudaSuccess)
            set_error(STWO_ERR_CUDA, "eval_at_point copy failed");
    }
    cudaFree(scratch);
    return out;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// eval_at_point without any allocation.
//
// Some callers cannot call cudaMalloc: a proof server that hands every byte of
// HBM to its own pool at start-up and admits jobs against that fixed budget, a
// host library embedded in a process whose allocator owns the device, or a
// latency-critical loop that must not pay the implicit device-wide
// synchronisation of cudaMalloc/cudaFree. For them this entry point evaluates a
// polynomial at a point with its per-block partial sums and completion tickets in
// a fixed device array of this library instead of freshly allocated memory.
//
// The array is a file-scope __device__ variable: every GPU that loads the library
// holds its 512.5 KiB until the process exits. Host code only knows a stand-in symbol
// for it, so its device address is looked up with cudaGetSymbolAddress once per
// device, on that device's first call (which therefore should come before any
// stream capture), and the address is what the kernel receives.
// All calls share the one array, so calls whose work overlaps on the GPU (two
// streams, or two host threads) race and must be serialised by the caller; the
// completion tickets are cleared at the start of every call, and the partial sums
// are fully rewritten before they are read.
// ---------------------------------------------------------------------------
constexpr uint32_t EAP_NOALLOC_MAX_LOG = 26;  // 2^26 coefficients, 2^15 partial sums
constexpr size_t EAP_NOALLOC_BYTES =
    (((size_t)1 << (EAP_NOALLOC_MAX_LOG - EAP_CHUNK_LOG)) * sizeof(qm31) + 16 + 256 + 255) / 256 * 256;

static __device__ __align__(256) unsigned char g_eap_noalloc_scratch[EAP_NOALLOC_BYTES];

namespace {

constexpr int EAP_NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_addr[EAP_NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device (looked up once).
int noalloc_scratch(void **out) {
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    STWO_REQUIRE(dev >= 0 && dev < EAP_NOALLOC_MAX_DEVICES, STWO_ERR_UNSUPPORTED_SIZE, "device ordinal %d", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_eap_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            return set_error(STWO_ERR_CUDA, "cudaGetSymbolAddress of the eval_at_point scratch failed: %s",
                             cudaGetErrorString(e));
        g_noalloc_addr[dev] = ptr;
    }
    *out = g_noalloc_addr[dev];
    return STWO_OK;
}

}  // namespace

extern "C" int stwo_eval_at_point_no_alloc(const uint32_t *coeffs, uint32_t log_size, stwo_qm31 point_x,
                                           stwo_qm31 point_y, stwo_qm31 *result, void *stream) {
    STWO_REQUIRE(log_size <= EAP_NOALLOC_MAX_LOG, STWO_ERR_UNSUPPORTED_SIZE,
                 "stwo_eval_at_point_no_alloc handles at most 2^%u coefficients (got 2^%u); use eval_at_point",
                 EAP_NOALLOC_MAX_LOG, log_size);
    STWO_REQUIRE(coeffs != nullptr && result != nullptr, STWO_ERR_INVALID_ARGUMENT, "null coefficient or result pointer");
    void *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    const stwo_spoint pt = {point_x, point_y};
    // tickets_zeroed = false: the ticket words are cleared with cudaMemsetAsync first.
    return eval_at_points_async(&coeffs, &log_size, 1, &pt, result, scratch, EAP_NOALLOC_BYTES, false,
                                as_stream(stream));
}
