// PolyOps entry points: twiddle trees, canonic -> bit-reversed reordering,
// interpolate / evaluate (reference-compatible and native), eval_at_point.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include <cuda.h>

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
// pi(x) = 2x^2 - 1 (eval_at_point.cu:99-109). A CTA folds a chunk of
// 2^(13 + iter_log) coefficients as groups of 8192: a warp reads 1024 consecutive
// coefficients with coalesced loads, a thread's 32 of them cover index bits 0, 1 and
// 7..9, and the thread forms sum_i c_i F_i against the CTA's table of the products of
// those bits' factors, an M31-by-QM31 dot product of 64-bit multiply-accumulates; the
// lanes fold bits 2..6 and the warps bits 10..12. Group partials are weighted by
// their group index's factors (bits 13..) before the lane fold, which is linear, so
// one fold serves the whole chunk. The chunk partial takes the factors of its chunk
// index; the last CTA of each polynomial (atomic ticket) adds the partials.
constexpr int EAP_THREADS = 256;
constexpr int EAP_PER_THREAD_LOG = 5;                    // 32 coefficients per thread
constexpr int EAP_GROUP_LOG = EAP_PER_THREAD_LOG + 8;    // x 256 threads
// Groups per CTA, 2^iter_log, chosen per launch (eap_iter_log): larger chunks spread
// each CTA's set-up over more coefficients; smaller ones keep small launches wide.
constexpr int EAP_ITER_LOG_MIN = 2;
constexpr int EAP_ITER_LOG_MAX = 4;
constexpr int EAP_CHUNK_LOG_MIN = EAP_GROUP_LOG + EAP_ITER_LOG_MIN;
constexpr int EAP_MAX_POLYS = 32;

struct EapParams {
    const uint32_t *coeffs[EAP_MAX_POLYS];
    qm31 factors[EAP_MAX_POLYS][32];
    uint32_t log_size[EAP_MAX_POLYS];
    uint32_t block_start[EAP_MAX_POLYS + 1];  // prefix sum of CTAs per polynomial
    uint32_t n_polys;
    uint32_t iter_log;                         // groups per CTA: 2^iter_log
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

// A warp reads 1024 consecutive coefficients of a group as 8 coalesced loads of 512
// bytes: load u gives lane l coefficients 128u + 4l + k, k = 0..3. So a thread's 32
// coefficients span index bits 0, 1 (k) and 7, 8, 9 (u), and the lanes bits 2..6.
// First coefficient of this warp's share of group `it` of chunk `chunk` (chunks of
// 2^chunk_log coefficients).
__device__ __forceinline__ uint64_t eap_base(uint32_t chunk, uint32_t chunk_log, uint32_t it) {
    return ((uint64_t)chunk << chunk_log) + ((uint64_t)it << EAP_GROUP_LOG) + ((uint64_t)(threadIdx.x >> 5) << 10);
}

// Factor index of bit b of a thread's term index 4u + k.
__device__ __forceinline__ constexpr int eap_term_bit(int b) { return b < 2 ? b : b + 5; }

// This thread's 32 coefficients of group `it` when the warp's 1024 all exist (a
// ragged group is read coefficient by coefficient instead).
__device__ __forceinline__ void eap_load(const uint32_t *c, uint64_t n, uint32_t chunk, uint32_t chunk_log, uint32_t it,
                                         uint4 (&v)[8]) {
    const uint64_t base = eap_base(chunk, chunk_log, it);
    if (base + 1024 <= n) {
        const uint4 *q = reinterpret_cast<const uint4 *>(c + base) + (threadIdx.x & 31u);
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = __ldg(q + 32 * u);
    }
}

// Folds values held by 2^LEVELS consecutive lanes, lane bit j <-> factor fj[j]: the
// lane with bit j clear forms lo + hi * fj[j], and its partner forms the same value.
template <int LEVELS>
__device__ __forceinline__ qm31 eap_lane_fold(qm31 acc, const qm31 *fj) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int j = 0; j < LEVELS; j++) {
        qm31 other = shfl_xor_q(acc, 1 << j);
        qm31 lo = (lane >> j) & 1u ? other : acc;
        qm31 hi = (lane >> j) & 1u ? acc : other;
        acc = qm31_add(lo, qm31_mul(hi, fj[j]));
    }
    return acc;
}

// One CTA's share of polynomial `poly`: chunk `chunk` (2^iter_log groups) of its 2^L
// coefficients c with factors f; its CTAs are blk_first .. blk_first + nblk - 1
// (partials indexed by CTA).
// cur holds this thread's first group, loaded by the caller before the factors were
// ready, so that those loads overlap the set-up of the tables.
// partials, tickets and results belong to job 0; this CTA's job is blockIdx.y, whose
// are moved by blockIdx.y * js bytes (applied where they are used, after the loop).
__device__ __forceinline__ void eap_body(uint32_t poly, uint32_t chunk, uint32_t L, const qm31 *f, const uint32_t *c,
                                         uint32_t iter_log, uint32_t blk_first, uint32_t nblk, qm31 *partials,
                                         uint32_t *tickets, qm31 *results, uint4 (&cur)[8], size_t js = 0) {
    __shared__ qm31 warp_vals[EAP_THREADS / 32];
    __shared__ qm31 g[1 << EAP_ITER_LOG_MAX];
    __shared__ qm31 F2[1 << EAP_PER_THREAD_LOG];  // F_i
    __shared__ qm31 chunk_w;
    __shared__ bool is_last;
    const uint32_t tid = threadIdx.x;
    const uint64_t n = 1ull << L;
    const uint32_t chunk_log = EAP_GROUP_LOG + iter_log;
    if (tid < (1u << EAP_PER_THREAD_LOG)) {
        qm31 w = qm31_one();
        for (int b = 0; b < EAP_PER_THREAD_LOG; b++)
            if ((tid >> b) & 1u) w = qm31_mul(w, f[eap_term_bit(b)]);
        F2[tid] = w;
    } else if (tid >= 32 && tid < 32 + (1u << iter_log)) {
        // group weights: products of f_{13+b} over the set bits b of the group index
        const uint32_t it = tid - 32;
        qm31 w = qm31_one();
        for (uint32_t b = 0; b < iter_log; b++)
            if ((it >> b) & 1u) w = qm31_mul(w, f[EAP_GROUP_LOG + b]);
        g[it] = w;
    }
    __syncthreads();
    if (tid == 64) {
        // The chunk weight (the factors of the chunk index's bits) is used only after
        // the last group; one thread forms it while its own loads are in flight.
        qm31 w = qm31_one();
        for (uint32_t b = 0; chunk_log + b < L; b++)
            if ((chunk >> b) & 1u) w = qm31_mul(w, f[chunk_log + b]);
        chunk_w = w;
    }

    qm31 acc = qm31_zero();
    for (uint32_t it = 0; it < (1u << iter_log); it++) {
        const uint64_t base = eap_base(chunk, chunk_log, it);
        if (base >= n) break;
        if (it > 0) eap_load(c, n, chunk, chunk_log, it, cur);
        uint64_t s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        // 64-bit multiply-accumulates of canonical values, folded after every fourth
        // term: a fold leaves less than 2^34, and four products of values below 2^31 - 1
        // add less than 2^64 - 2^34. (The folds stay on the ALU pipe here: as FMA-pipe
        // multiply-adds, fold64_fma, this loop measured 5% slower.)
        auto term = [&](uint32_t v, uint32_t i) {
            const qm31 w = F2[i];
            s0 = mac64(s0, v, w.a.a);
            s1 = mac64(s1, v, w.a.b);
            s2 = mac64(s2, v, w.b.a);
            s3 = mac64(s3, v, w.b.b);
            if (i % 4 == 3) {
                s0 = fold64(s0);
                s1 = fold64(s1);
                s2 = fold64(s2);
                s3 = fold64(s3);
            }
        };
        if (base + 1024 <= n) {
#pragma unroll
            for (int u = 0; u < 8; u++) {
                term(cur[u].x, 4 * u);
                term(cur[u].y, 4 * u + 1);
                term(cur[u].z, 4 * u + 2);
                term(cur[u].w, 4 * u + 3);
            }
        } else {
            for (uint32_t i = 0; i < 32; i++) {
                const uint64_t at = base + 128 * (i >> 2) + 4 * (tid & 31u) + (i & 3u);
                if (at >= n) break;  // positions grow with i
                term(__ldg(c + at), i);
            }
        }
        const qm31 part = {{reduce64_p(s0), reduce64_p(s1)}, {reduce64_p(s2), reduce64_p(s3)}};
        acc = qm31_add(acc, it == 0 ? part : qm31_mul(part, g[it]));
    }
    // Across lanes: bits 2..6; across the 8 warps (in warp 0): bits 10..12.
    acc = eap_lane_fold<5>(acc, f + 2);
    if ((tid & 31u) == 0) warp_vals[tid >> 5] = acc;
    __syncthreads();
    if (tid < 32) {
        qm31 w = tid < EAP_THREADS / 32 ? warp_vals[tid] : qm31_zero();
        w = eap_lane_fold<3>(w, f + 10);
        if (tid == 0) {
            job_ptr(partials, js, blockIdx.y)[blockIdx.x] = qm31_mul(w, chunk_w);
            __threadfence();
            uint32_t t = atomicAdd(&job_ptr(tickets, js, blockIdx.y)[poly], 1u);
            is_last = (t == nblk - 1);
        }
    }
    __syncthreads();
    if (is_last) {
        partials = job_ptr(partials, js, blockIdx.y);
        tickets = job_ptr(tickets, js, blockIdx.y);
        results = job_ptr(results, js, blockIdx.y);
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
        if ((tid & 31u) == 0) warp_vals[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) {
            qm31 t = qm31_zero();
            for (int i = 0; i < EAP_THREADS / 32; i++) t = qm31_add(t, warp_vals[i]);
            results[poly] = t;
            tickets[poly] = 0;  // ready for the next launch
        }
    }
}

// Three CTAs per SM: at four the per-polynomial factor tables read from the kernel
// parameters spill (measured 3% slower over 32 x 2^22 coefficients).
__global__ void __launch_bounds__(EAP_THREADS, 3) eval_at_point_kernel(const __grid_constant__ EapParams p) {
    uint32_t poly = 0;
    while (poly + 1 < p.n_polys && blockIdx.x >= p.block_start[poly + 1]) poly++;
    const uint32_t chunk = blockIdx.x - p.block_start[poly];
    uint4 cur[8];
    eap_load(p.coeffs[poly], 1ull << p.log_size[poly], chunk, EAP_GROUP_LOG + p.iter_log, 0, cur);
    eap_body(poly, chunk, p.log_size[poly], p.factors[poly], p.coeffs[poly], p.iter_log, p.block_start[poly],
             p.block_start[poly + 1] - p.block_start[poly], p.partials, p.tickets, p.results, cur);
}

// Polynomials described in device memory, all evaluated at one point also in device
// memory (x then y); each CTA derives its polynomial's factors itself.
struct EapDevPoly {
    const uint32_t *coeffs;
    uint32_t log_size;
    uint32_t block_start;  // first CTA of the polynomial
};

__global__ void __launch_bounds__(EAP_THREADS, 4) eval_at_point_dev_kernel(const EapDevPoly *__restrict__ polys,
                                                                           uint32_t n_polys, uint32_t iter_log,
                                                                           const qm31 *point, qm31 *partials,
                                                                           uint32_t *tickets, qm31 *results, size_t js) {
    // blockIdx.y: the job, whose descriptors, point, partials, tickets and results are
    // job 0's moved by blockIdx.y * js bytes
    polys = job_ptr(polys, js, blockIdx.y);
    __shared__ qm31 f[32];
    // The last polynomial whose first CTA is <= blockIdx.x, by a 32-way search: each
    // round lane k tests candidate lo + k * step, and polys[lo] always qualifies.
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lo = 0, count = n_polys;
    while (count > 1) {
        const uint32_t step = (count + 31) / 32;
        const bool ok = lane * step < count && polys[lo + lane * step].block_start <= blockIdx.x;
        const uint32_t t = 31 - __clz(__ballot_sync(0xffffffffu, ok));
        lo += t * step;
        count = min(step, count - t * step);
    }
    const EapDevPoly d = polys[lo];
    const uint32_t next = lo + 1 < n_polys ? polys[lo + 1].block_start : gridDim.x;
    const uint32_t chunk = blockIdx.x - d.block_start;
    uint4 cur[8];
    eap_load(d.coeffs, 1ull << d.log_size, chunk, EAP_GROUP_LOG + iter_log, 0, cur);
    if (threadIdx.x == 0) {
        // f_0 = y, f_1 = x, f_b = pi^(b-1)(x)
        point = job_ptr(point, js, blockIdx.y);
        f[0] = point[1];
        qm31 x = point[0];
        for (uint32_t b = 1; b < 32; b++) {
            f[b] = x;
            qm31 sq = qm31_mul(x, x);
            x = qm31_sub(qm31_add(sq, sq), qm31_one());
        }
    }
    __syncthreads();
    eap_body(lo, chunk, d.log_size, f, d.coeffs, iter_log, d.block_start, next - d.block_start, partials, tickets,
             results, cur, js);
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

uint32_t eap_blocks(uint32_t L, uint32_t iter_log) {
    const uint32_t chunk_log = EAP_GROUP_LOG + iter_log;
    return L <= chunk_log ? 1u : 1u << (L - chunk_log);
}

// Groups per CTA for a launch over these polynomials: the largest chunks that still
// give at least two CTAs per SM (unless the eval_at_point_groups_log tunable fixes it).
uint32_t eap_iter_log(const uint32_t *log_sizes, uint32_t n) {
    const int forced = tunable(TUNE_EAP_GROUPS_LOG);
    if (forced >= EAP_ITER_LOG_MIN && forced <= EAP_ITER_LOG_MAX) return (uint32_t)forced;
    const uint64_t want = 2ull * device_sm_count();
    for (uint32_t k = EAP_ITER_LOG_MAX; k > EAP_ITER_LOG_MIN; k--) {
        uint64_t blocks = 0;
        for (uint32_t i = 0; i < n; i++) blocks += eap_blocks(log_sizes[i], k);
        if (blocks >= want) return k;
    }
    return EAP_ITER_LOG_MIN;
}

}  // namespace

size_t eval_at_points_scratch_bytes(const uint32_t *log_sizes, uint32_t n_polys) {
    size_t blocks = 0;
    for (uint32_t i = 0; i < n_polys; i++) blocks += eap_blocks(log_sizes[i], EAP_ITER_LOG_MIN);
    return blocks * sizeof(qm31) + ((size_t)n_polys * 4 + 15) / 16 * 16 + 256;
}

// scratch: partials followed by zeroed tickets (the kernel leaves them zero); the
// tickets sit after room for the partials of the smallest chunks, whatever a launch
// chooses.
int eval_at_points_async(const uint32_t *const *coeffs, const uint32_t *log_sizes, uint32_t n_polys,
                         const stwo_spoint *points, stwo_qm31 *results, void *scratch, size_t scratch_bytes,
                         bool tickets_zeroed, cudaStream_t st) {
    STWO_REQUIRE(scratch_bytes >= eval_at_points_scratch_bytes(log_sizes, n_polys), STWO_ERR_INVALID_ARGUMENT,
                 "eval_at_point scratch too small");
    size_t blocks_total = 0;
    for (uint32_t i = 0; i < n_polys; i++) {
        STWO_REQUIRE(log_sizes[i] <= 30, STWO_ERR_UNSUPPORTED_SIZE, "polynomial of log size %u unsupported", log_sizes[i]);
        blocks_total += eap_blocks(log_sizes[i], EAP_ITER_LOG_MIN);
    }
    uint32_t *tickets = reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) + blocks_total * sizeof(qm31));
    if (!tickets_zeroed) STWO_CUDA_TRY(cudaMemsetAsync(tickets, 0, (size_t)n_polys * 4, st));
    qm31 *partials = static_cast<qm31 *>(scratch);
    uint32_t done = 0;
    size_t part_off = 0;
    while (done < n_polys) {
        EapParams p{};
        uint32_t cnt = std::min<uint32_t>(EAP_MAX_POLYS, n_polys - done);
        p.iter_log = eap_iter_log(log_sizes + done, cnt);
        uint32_t b = 0;
        for (uint32_t i = 0; i < cnt; i++) {
            uint32_t L = log_sizes[done + i];
            p.coeffs[i] = coeffs[done + i];
            p.log_size[i] = L;
            eap_factors(p.factors[i], points[done + i], L);
            p.block_start[i] = b;
            b += eap_blocks(L, p.iter_log);
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
// EapDevPoly, CTAs counted with eval_at_point_blocks(log size, iter_log)), at the
// device point point_dev (QM31 x then y). partials: total_blocks QM31; tickets:
// n_polys zeroed words (left zeroed). jobs sets of one shape at once: set k's
// descriptors, point, results, partials and tickets are set 0's moved by k * js bytes.
int eval_at_points_dev_async(const void *polys_dev, uint32_t n_polys, uint32_t iter_log, uint32_t total_blocks,
                             const void *point_dev, void *results, void *partials, uint32_t *tickets, uint32_t jobs,
                             size_t js, cudaStream_t st) {
    STWO_REQUIRE(n_polys >= 1 && total_blocks >= n_polys, STWO_ERR_INVALID_ARGUMENT, "eval_at_point descriptors");
    STWO_REQUIRE(jobs >= 1 && jobs <= 65535, STWO_ERR_INVALID_ARGUMENT, "eval_at_point sets per launch: %u", jobs);
    STWO_REQUIRE(iter_log >= (uint32_t)EAP_ITER_LOG_MIN && iter_log <= (uint32_t)EAP_ITER_LOG_MAX,
                 STWO_ERR_INVALID_ARGUMENT, "eval_at_point groups per CTA 2^%u", iter_log);
    eval_at_point_dev_kernel<<<dim3(total_blocks, jobs), EAP_THREADS, 0, st>>>(
        static_cast<const EapDevPoly *>(polys_dev), n_polys, iter_log, static_cast<const qm31 *>(point_dev),
        static_cast<qm31 *>(partials), tickets, static_cast<qm31 *>(results), js);
    STWO_LAUNCH_CHECK("eval_at_point_dev_kernel");
    return STWO_OK;
}

// CTAs of one polynomial of 2^log_size coefficients at 2^iter_log groups per CTA;
// iter_log 0 asks for the most CTAs any launch uses (an upper bound for sizing).
uint32_t eval_at_point_blocks(uint32_t log_size, uint32_t iter_log) {
    return eap_blocks(log_size, iter_log ? iter_log : (uint32_t)EAP_ITER_LOG_MIN);
}

uint32_t eval_at_point_iter_log(const uint32_t *log_sizes, uint32_t n) { return eap_iter_log(log_sizes, n); }

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
// holds its 32.5 KiB until the process exits. Host code only knows a stand-in symbol
// for it, so its device address is looked up with cudaGetSymbolAddress once per
// device, on that device's first call (which therefore should come before any
// stream capture), and the address is what the kernel receives. A device reset
// gives the device a new context in which the array has a new address; the next
// call sees the changed context and looks the address up again.
// All calls share the one array, so calls whose work overlaps on the GPU (two
// streams, or two host threads) race and must be serialised by the caller; the
// completion tickets are cleared at the start of every call, and the partial sums
// are fully rewritten before they are read.
// ---------------------------------------------------------------------------
constexpr uint32_t EAP_NOALLOC_MAX_LOG = 26;  // 2^26 coefficients, at most 2^11 partial sums
constexpr size_t EAP_NOALLOC_BYTES =
    (((size_t)1 << (EAP_NOALLOC_MAX_LOG - EAP_CHUNK_LOG_MIN)) * sizeof(qm31) + 16 + 256 + 255) / 256 * 256;
static_assert(EAP_NOALLOC_BYTES == 33280, "the documented size of the no-allocation scratch is 32.5 KiB");

static __device__ __align__(256) unsigned char g_eap_noalloc_scratch[EAP_NOALLOC_BYTES];

namespace {

constexpr int EAP_NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
struct NoallocSlot {
    void *addr;
    unsigned long long ctx_id;  // unique id of the context the address belongs to
};
NoallocSlot g_noalloc[EAP_NOALLOC_MAX_DEVICES] = {};

// Unique id of the calling thread's current context (0 when there is none). The
// address of a __device__ array belongs to one context: after cudaDeviceReset, or a
// released and re-created primary context, the array lives at a new address, and
// the id (never reused within a process) tells the two apart. The driver functions
// come through the runtime's entry-point query, so the library still links only
// against cudart.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
                       q == cudaDriverEntryPointSuccess
                   ? reinterpret_cast<CtxGetCurrentFn>(f)
                   : nullptr;
    }();
    static CtxGetIdFn get_id = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
                       q == cudaDriverEntryPointSuccess
                   ? reinterpret_cast<CtxGetIdFn>(f)
                   : nullptr;
    }();
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr ||
        get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array on the current device: looked up with the
// device current on its first call, and again whenever the device's context has
// changed since (a reset).
int noalloc_scratch(void **out) {
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    STWO_REQUIRE(dev >= 0 && dev < EAP_NOALLOC_MAX_DEVICES, STWO_ERR_UNSUPPORTED_SIZE, "device ordinal %d", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocSlot &slot = g_noalloc[dev];
    const unsigned long long id = current_context_id();
    if (!slot.addr || id == 0 || id != slot.ctx_id) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_eap_noalloc_scratch);  // makes the context current
        if (e != cudaSuccess || ptr == nullptr)
            return set_error(STWO_ERR_CUDA, "cudaGetSymbolAddress of the eval_at_point scratch failed: %s",
                             cudaGetErrorString(e));
        slot.addr = ptr;
        slot.ctx_id = current_context_id();
    }
    *out = slot.addr;
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
