// Wide-Fibonacci STARK prover: stwo's prove() for the wide-Fibonacci AIR, driven on
// the host in C++ over this library's kernels, with the Fiat-Shamir channel on the
// device.
//
// The protocol is stwo's (stwo-prover @ ce5b975, as the reference drives it in
// stwo_gpu_backend/src/examples/wide_fibonacci.rs:205-250 with PcsConfig::default()
// = {pow_bits 5, FriConfig{log_last_layer_degree_bound 0, log_blowup 1, n_queries 3}}):
//
//   1. trace: 2^L rows of N columns (a, b, a^2+b^2, ...), interpolated, evaluated on
//      CanonicCoset(L+B), committed in a Blake2s Merkle tree; root mixed into the
//      Blake2s channel.
//   2. composition: random coefficient r; the N-2 constraints combined with powers of r
//      and divided by the vanishing polynomial of CanonicCoset(L).coset on
//      CanonicCoset(L+1); interpolated; its 4 coordinate polynomials evaluated on
//      CanonicCoset(L+1+B) and committed.
//   3. out-of-domain sampling at a random circle point (get_random_point); sampled
//      values mixed; the composition value checked against the constraints there.
//   4. DEEP quotients per column size, FRI commitment (circle fold of the largest
//      quotient, line folds, smaller quotients folded in when sizes meet) down to a
//      constant last layer.
//   5. proof of work (least nonce with pow_bits trailing zeros), query positions,
//      Merkle and FRI decommitments, gathered from device memory in one launch.
//
// Steps 1-5 up to the query positions are one asynchronous sequence of launches on the
// job's stream: the channel (channel.cuh) runs in single-thread kernels between the
// data kernels and leaves every challenge in device memory, where the next kernel
// reads it. The host synchronises twice per proof: to read the channel's record (roots,
// sampled values, last layer, nonce, query words) and to read the decommitted words.
// All of a job's buffers, column-pointer tables and kernel parameters that depend on
// the channel live in one slab from the library's memory pool.
//
// The proof bytes are the CommitmentSchemeProof fields in declaration order, little
// endian, vectors prefixed with a u64 length, hashes as 32 raw bytes, field elements as
// u32 words (a bincode-style layout):
//   commitments, sampled_values, decommitments, queried_values, proof_of_work,
//   fri_proof{first_layer, inner_layers, last_layer_poly{coeffs, log_size}}.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <vector>

#include "blake2s.cuh"
#include "channel.cuh"
#include "common.cuh"
#include "fri.cuh"
#include "prover.cuh"
#include "quotients.cuh"

namespace stwo {

int fft_columns(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st);
int fft_columns_tab(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                    const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st, const void *dev_table);
int merkle_tree_dev_async(uint32_t max_log, const uint32_t *const *const *level_cols, const uint32_t *level_ncols,
                          uint32_t *const *layers, uint32_t *tickets, uint32_t n_tickets, uint32_t jobs, size_t js,
                          cudaStream_t st);
uint32_t merkle_tree_tickets(uint32_t max_log);
int fold_async(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha_c, const uint32_t *itw, uint64_t off,
               uint32_t *const *dst4, bool circle, cudaStream_t st, const void *alpha_dev, uint32_t jobs, size_t js);
int wide_fib_dev_async(const uint32_t *const *trace_dev, uint32_t n_cols, uint32_t log_size, const uint32_t *powers_dev,
                       const uint32_t den_half[2], uint32_t *const *out4, uint32_t jobs, size_t js, cudaStream_t st);
int eval_at_points_dev_async(const void *polys_dev, uint32_t n_polys, uint32_t iter_log, uint32_t total_blocks,
                             const void *point_dev, void *results, void *partials, uint32_t *tickets, uint32_t jobs,
                             size_t js, cudaStream_t st);
uint32_t eval_at_point_blocks(uint32_t log_size, uint32_t iter_log);
uint32_t eval_at_point_iter_log(const uint32_t *log_sizes, uint32_t n);

namespace {

constexpr uint32_t WF_MAX_TRACE_COLS = 1024;
constexpr uint32_t MAX_JOBS_PER_LAUNCH = 256;  // proofs of one shape in one launch sequence
constexpr uint32_t MAX_DOMAIN_LOG = 27;  // largest committed domain CanonicCoset(L+1+B)
constexpr uint32_t MAX_LAYERS = 32;      // FRI inner layers
constexpr uint32_t MAX_QUERIES = 1024;

// ------------------------------------------------------------------ device state

// What the device channel records for the host: the tree roots in commitment order
// (trace, composition, FRI first layer, FRI inner layers), the challenges, the last
// layer, the nonce and the raw query words. The sampled values follow it in memory.
struct ProofState {
    fs::DevChannel ch;
    uint32_t error;
    uint32_t pad;
    unsigned long long nonce;  // least valid proof-of-work nonce (all ones: none yet)
    qm31 rc, qrc, last_coeff;
    qm31 oods[2];  // x, y
    qm31 alphas[MAX_LAYERS + 1];
    uint32_t roots[MAX_LAYERS + 3][8];
    uint32_t query_words[MAX_QUERIES];
};

// The polynomial descriptors of the OODS evaluation (eval_at_points_dev_async).
struct EapDevPoly {
    const uint32_t *coeffs;
    uint32_t log_size;
    uint32_t block_start;
};

// ------------------------------------------------------------------ device kernels

// Trace rows (write_trace_row, wide_fibonacci.rs:196-203): a_0 = a0[r], a_1 = a1[r],
// a_{j+2} = a_j^2 + a_{j+1}^2. Row r is position r of every column, the bit-reversed
// storage order of the trace evaluations. Column pointers come from a device table.
// blockIdx.y: the job (js: the jobs' memory stride).
__global__ void __launch_bounds__(256) wide_fib_trace_kernel(const uint32_t *__restrict__ a0,
                                                             const uint32_t *__restrict__ a1,
                                                             uint32_t *const *__restrict__ cols, uint32_t n_cols,
                                                             uint64_t rows, size_t js) {
    a0 = job_ptr(a0, js, blockIdx.y);
    a1 = job_ptr(a1, js, blockIdx.y);
    cols = job_ptr(cols, js, blockIdx.y);
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t x = a0[r], y = a1[r];
        cols[0][r] = x;
        cols[1][r] = y;
        for (uint32_t j = 2; j < n_cols; j++) {
            uint32_t z = m31_add(m31_sqr(x), m31_sqr(y));
            cols[j][r] = z;
            x = y;
            y = z;
        }
    }
}

// Half coset {initial index, step index} of CanonicCoset(log).circle_domain():
// 2^(30-log) and 2^(32-log).
inline uint32_t half_coset_init(uint32_t log) { return 1u << (30 - log); }
inline uint32_t half_coset_step(uint32_t log) { return (uint32_t)((1ull << (32 - log)) & 0x7fffffffu); }

// -initial + step/2 of CanonicCoset(log).coset (initial index 2^(30-log), step 2^(31-log)).
__host__ __device__ inline cpoint vanishing_shift(uint32_t log) {
    cpoint init = index_to_point(1u << (30 - log));
    cpoint half_step = index_to_point(1u << (30 - log));
    return point_mul(point_conj(init), half_step);
}

// Vanishing polynomial of CanonicCoset(L).coset on the circle domain CanonicCoset(L + 1)
// in bit-reversed order (coset_vanishing as wide_fibonacci.rs:99-117 calls it: p ->
// p - initial + step/2, then the x coordinate doubled L - 1 times). After L - 1
// doublings the 2^(L+1) domain points land on two values, one for each half of the
// bit-reversed order, so the composition needs only their two inverses: the values
// at bit-reversed positions 0 and 2^L, i.e. the half-coset points of indices 0 and 1.
inline void vanishing_inverses(uint32_t L, uint32_t out[2]) {
    const uint32_t E = L + 1;
    const uint32_t idx[2] = {half_coset_init(E), half_coset_init(E) + half_coset_step(E)};
    const cpoint sh = vanishing_shift(L);
    for (int h = 0; h < 2; h++) {
        uint32_t x = point_mul(index_to_point(idx[h] & 0x7fffffffu), sh).x;
        for (uint32_t d = 0; d + 1 < L; d++) x = m31_sub(m31_add(m31_sqr(x), m31_sqr(x)), 1);
        out[h] = m31_inv(x);
    }
}

// Channel step after the trace tree: mix its root, draw the composition coefficient r,
// and write powers[k] = r^k (k < n_powers; lane l computes k = l, l + 32, ...).
__global__ void fs_trace_kernel(ProofState *s, const uint32_t *root, qm31 *powers, uint32_t n_powers, size_t js) {
    s = job_ptr(s, js, blockIdx.x);  // one CTA a job
    root = job_ptr(root, js, blockIdx.x);
    powers = job_ptr(powers, js, blockIdx.x);
    __shared__ qm31 rc;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 8; i++) s->roots[0][i] = root[i];
        fs::ch_mix_root(s->ch, root);
        rc = fs::ch_draw_felt(s->ch, s->error);
        s->rc = rc;
    }
    __syncthreads();
    const qm31 r = rc;
    qm31 p = qm31_pow(r, threadIdx.x);
    const qm31 step = qm31_pow(r, blockDim.x);
    for (uint32_t k = threadIdx.x; k < n_powers; k += blockDim.x) {
        powers[k] = p;
        p = qm31_mul(p, step);
    }
}

// Channel step after the composition tree: mix its root, draw t and take the OODS
// point (CirclePoint::get_random_point): x = (1 - t^2) / (1 + t^2), y = 2t / (1 + t^2).
__global__ void fs_comp_kernel(ProofState *s, const uint32_t *root, size_t js) {
    s = job_ptr(s, js, blockIdx.x);  // one thread a job
    root = job_ptr(root, js, blockIdx.x);
    for (int i = 0; i < 8; i++) s->roots[1][i] = root[i];
    fs::ch_mix_root(s->ch, root);
    const qm31 t = fs::ch_draw_felt(s->ch, s->error), t2 = qm31_mul(t, t);
    const qm31 inv = qm31_inv(qm31_add(t2, qm31_one()));
    s->oods[0] = qm31_mul(qm31_sub(qm31_one(), t2), inv);
    s->oods[1] = qm31_mul(qm31_add(t, t), inv);
}


// Channel step after the OODS evaluation, by one CTA: the constraint sum
// sum_i r^(N-3-i) (c_i^2 + c_{i+1}^2 - c_{i+2}) over the sampled trace values (powers
// from fs_trace_kernel), checked against the composition's sampled value times the
// vanishing polynomial at the OODS point; thread 0 mixes the sampled values (N trace
// values, then the composition's 4 coordinates) and draws the quotient coefficient;
// then the quotient kernels' sample-dependent parameters of both column groups.
// The sampled values are first staged in shared memory (up to OODS_STAGED of them), so
// that the serial hash reads each chunk without an L2 round trip; the constraint check
// runs on another warp while thread 0 hashes. vsh: vanishing_shift(L), from the host.
constexpr uint32_t OODS_STAGED = 1024;
__global__ void __launch_bounds__(256) fs_oods_kernel(ProofState *s, const qm31 *sampled, const qm31 *powers,
                                                      uint32_t N, uint32_t L, cpoint vsh, QuotParamsDev *q_comp,
                                                      QuotParamsDev *q_trace, size_t js) {
    s = job_ptr(s, js, blockIdx.x);  // one CTA a job
    sampled = job_ptr(sampled, js, blockIdx.x);
    powers = job_ptr(powers, js, blockIdx.x);
    q_comp = job_ptr(q_comp, js, blockIdx.x);
    q_trace = job_ptr(q_trace, js, blockIdx.x);
    __shared__ qm31 sh[32];
    __shared__ qm31 qrc_sh;
    __shared__ qm31 staged[OODS_STAGED];
    __shared__ uint32_t bad_sh;
    const uint32_t n_vals = N + 4;
    const bool stage = n_vals <= OODS_STAGED;
    if (stage)
        for (uint32_t i = threadIdx.x; i < n_vals; i += blockDim.x) staged[i] = sampled[i];
    __syncthreads();
    const qm31 *vals = stage ? staged : sampled;
    qm31 part = qm31_zero();
    for (uint32_t i = threadIdx.x; i + 2 < N; i += blockDim.x) {
        const qm31 cons = qm31_sub(qm31_add(qm31_mul(vals[i], vals[i]), qm31_mul(vals[i + 1], vals[i + 1])), vals[i + 2]);
        part = qm31_add(part, qm31_mul(cons, powers[N - 3 - i]));
    }
    const qm31 acc = block_sum_qm31(part, sh);
    const qm31 ox = s->oods[0], oy = s->oods[1];
    if (threadIdx.x == 0) {
        fs::ch_mix_felts(s->ch, vals, n_vals);
        const qm31 qrc = fs::ch_draw_felt(s->ch, s->error);
        s->qrc = qrc;
        qrc_sh = qrc;
    } else if (threadIdx.x == 32) {
        // composition value: from_partial_evals over the basis 1, i, u, iu
        const qm31 basis[4] = {{{1, 0}, {0, 0}}, {{0, 1}, {0, 0}}, {{0, 0}, {1, 0}}, {{0, 0}, {0, 1}}};
        qm31 comp = qm31_zero();
        for (int k = 0; k < 4; k++) comp = qm31_add(comp, qm31_mul(vals[N + k], basis[k]));
        // coset_vanishing(CanonicCoset(L).coset, oods)
        qm31 x = qm31_sub(qm31_scale(ox, vsh.x), qm31_scale(oy, vsh.y));
        for (uint32_t d = 0; d + 1 < L; d++) {
            qm31 q = qm31_mul(x, x);
            x = qm31_sub(qm31_add(q, q), qm31_one());
        }
        bad_sh = qm31_eq(qm31_mul(acc, qm31_inv(x)), comp) ? 0u : fs::ERR_CONSTRAINTS;
    }
    __syncthreads();
    if (threadIdx.x == 0) s->error |= bad_sh;
    const qm31 qrc = qrc_sh;
    quot_fill_batch_block(*q_comp, 0, qrc, ox, oy, vals + N, 4, 0, sh);
    quot_fill_batch_block(*q_trace, 0, qrc, ox, oy, vals, N, 0, sh);
}

// Channel step after an FRI tree: mix its root, draw the folding alpha.
__global__ void fs_layer_kernel(ProofState *s, const uint32_t *root, uint32_t root_slot, uint32_t alpha_slot,
                                size_t js) {
    s = job_ptr(s, js, blockIdx.x);  // one thread a job
    root = job_ptr(root, js, blockIdx.x);
    for (int i = 0; i < 8; i++) s->roots[root_slot][i] = root[i];
    fs::ch_mix_root(s->ch, root);
    s->alphas[alpha_slot] = fs::ch_draw_felt(s->ch, s->error);
}

// Last FRI layer: 2^log values (bit-reversed) over the line domain
// Coset(2^(29-log), 2^(31-log)) interpolated (LineEvaluation::interpolate); every
// coefficient but the constant must vanish (degree bound 1); the constant is mixed.

__device__ void fs_last(ProofState *s, const uint32_t *const c[4], uint32_t log) {
    const uint32_t n = 1u << log;  // log <= 4
    qm31 v[16];
    for (uint32_t i = 0; i < n; i++) v[bit_reverse_bits(i, log)] = {{c[0][i], c[1][i]}, {c[2][i], c[3][i]}};
    uint32_t di = 1u << (29 - log), ds = 1u << (31 - log);
    for (uint32_t size = n; size > 1; size >>= 1) {
        for (uint32_t c0 = 0; c0 < n; c0 += size)
            for (uint32_t i = 0; i < size / 2; i++) {
                const uint32_t xi = m31_inv(index_to_point((di + ds * i) & 0x7fffffffu).x);
                const qm31 a = v[c0 + i], b = v[c0 + i + size / 2];
                v[c0 + i] = qm31_add(a, b);
                v[c0 + i + size / 2] = qm31_scale(qm31_sub(a, b), xi);
            }
        di = (di * 2) & 0x7fffffffu;
        ds = (ds * 2) & 0x7fffffffu;
    }
    const uint32_t ninv = m31_inv(n);
    for (uint32_t i = 1; i < n; i++)  // any non-constant coefficient (storage order is irrelevant here)
        if (!qm31_eq(v[i], qm31_zero())) s->error |= fs::ERR_LAST_LAYER;
    const qm31 c0 = qm31_scale(v[0], ninv);
    s->last_coeff = c0;
    fs::ch_mix_felts(s->ch, &c0, 1);
}

// The FRI tail in one launch: one CTA of 1024 threads runs every inner layer of log
// size <= TAIL_MAX_LOG in order, then the last layer, exactly as the per-layer
// launches do:
//   [the trace quotient's circle fold into the layer, with the previous alpha]
//   -> the layer's Merkle tree over its 4 coordinate columns (leaves: one compression
//      of the 4 values; nodes: one compression of the two children), every level
//      written to its global buffer for the decommitment and kept in shared memory
//      for the next level
//   -> thread 0: mix the root, draw the layer's alpha
//   -> fold_line into the next layer.
// Values this kernel wrote are read back with plain (coherent) loads after a
// barrier; nothing is read through the non-coherent path except the trace quotient
// and the twiddles.
constexpr uint32_t TAIL_MAX_LOG = 10;
constexpr uint32_t TAIL_MAX = TAIL_MAX_LOG;  // inner layers of log size 2 .. TAIL_MAX_LOG
constexpr uint32_t TAIL_THREADS = 1024;
constexpr size_t TAIL_SMEM = (32ull << TAIL_MAX_LOG) + (32ull << (TAIL_MAX_LOG - 1));

struct TailParams {
    uint32_t li0, n_tail, lg0, last_log;
    uint32_t circle_t;                            // tail index of the layer the trace quotient folds into, or ~0
    const uint32_t *qt[4];                        // trace quotient (2 * 2^lg values at circle_t)
    const uint32_t *circle_tw;                    // inverse-twiddle suffix of that fold
    uint32_t *lay[TAIL_MAX + 1][4];               // tail layers, then the last layer
    uint4 *nodes[TAIL_MAX][TAIL_MAX_LOG + 1];     // tree layers of each tail layer
    const uint32_t *line_tw[TAIL_MAX];            // inverse-twiddle suffix of each layer's line fold
};

__global__ void __launch_bounds__(TAIL_THREADS) fri_tail_kernel(ProofState *s, const TailParams *__restrict__ tp,
                                                                 uint32_t one, size_t js) {
    s = job_ptr(s, js, blockIdx.x);  // one CTA a job; the job's parameters hold its own pointers
    tp = job_ptr(tp, js, blockIdx.x);
    extern __shared__ uint4 t_buf[];
    // the two node buffers, by computed address (an indexed pointer array would live
    // in local memory)
    auto buf = [&](uint32_t which) { return t_buf + (which ? (2u << TAIL_MAX_LOG) : 0u); };
    __shared__ qm31 alpha_sh;
    const uint32_t tid = threadIdx.x;
    for (uint32_t t = 0; t < tp->n_tail; t++) {
        const uint32_t li = tp->li0 + t, lg = tp->lg0 - t, n = 1u << lg;
        uint32_t *const *cur = tp->lay[t];
        if (t == tp->circle_t) {
            const qm31 a = s->alphas[li], a2 = qm31_mul(a, a);
            for (uint32_t i = tid; i < n; i += TAIL_THREADS) {
                const qm31 f0 = {{__ldg(tp->qt[0] + 2 * i), __ldg(tp->qt[1] + 2 * i)},
                                 {__ldg(tp->qt[2] + 2 * i), __ldg(tp->qt[3] + 2 * i)}};
                const qm31 f1 = {{__ldg(tp->qt[0] + 2 * i + 1), __ldg(tp->qt[1] + 2 * i + 1)},
                                 {__ldg(tp->qt[2] + 2 * i + 1), __ldg(tp->qt[3] + 2 * i + 1)}};
                const qm31 f = fold_pair(f0, f1, circle_itw(tp->circle_tw, i), a);
                const qm31 p = {{cur[0][i], cur[1][i]}, {cur[2][i], cur[3][i]}};
                const qm31 r = qm31_add(qm31_mul(p, a2), f);
                cur[0][i] = r.a.a;
                cur[1][i] = r.a.b;
                cur[2][i] = r.b.a;
                cur[3][i] = r.b.b;
            }
            __syncthreads();
        }
        // Leaves: one compression of the layer's 4 values.
        for (uint32_t i = tid; i < n; i += TAIL_THREADS) {
            uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t m[16] = {cur[0][i], cur[1][i], cur[2][i], cur[3][i], 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            blake::compress(h, m, one);
            const uint4 lo = make_uint4(h[0], h[1], h[2], h[3]), hi = make_uint4(h[4], h[5], h[6], h[7]);
            tp->nodes[t][lg][2 * i] = lo;
            tp->nodes[t][lg][2 * i + 1] = hi;
            buf(0)[2 * i] = lo;
            buf(0)[2 * i + 1] = hi;
        }
        __syncthreads();
        // Nodes, level by level: children from one shared buffer, parents into the other.
        // Levels of at most 32 nodes are left to the first warp, which synchronises
        // with itself only.
        auto node = [&](uint32_t l, uint32_t k, uint32_t src) {
            uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t m[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint4 v = buf(src)[4 * k + q];
                m[4 * q] = v.x; m[4 * q + 1] = v.y; m[4 * q + 2] = v.z; m[4 * q + 3] = v.w;
            }
            blake::compress(h, m, one);
            const uint4 lo = make_uint4(h[0], h[1], h[2], h[3]), hi = make_uint4(h[4], h[5], h[6], h[7]);
            tp->nodes[t][l][2 * k] = lo;
            tp->nodes[t][l][2 * k + 1] = hi;
            buf(src ^ 1)[2 * k] = lo;
            buf(src ^ 1)[2 * k + 1] = hi;
        };
        uint32_t src = 0;
        int l = (int)lg - 1;
        for (; l >= 0 && (1u << l) > 32u; l--) {
            for (uint32_t k = tid; k < (1u << l); k += TAIL_THREADS) node((uint32_t)l, k, src);
            src ^= 1;
            __syncthreads();
        }
        if (tid < 32) {  // src is only read by thread 0 below
            for (; l >= 0; l--) {
                if (tid < (1u << l)) node((uint32_t)l, tid, src);
                src ^= 1;
                __syncwarp();
            }
        }
        if (tid == 0) {
            const uint4 lo = buf(src)[0], hi = buf(src)[1];
            const uint32_t root[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
            for (int i = 0; i < 8; i++) s->roots[3 + li][i] = root[i];
            fs::ch_mix_root(s->ch, root);
            const qm31 a = fs::ch_draw_felt(s->ch, s->error);
            s->alphas[li + 1] = a;
            alpha_sh = a;
        }
        __syncthreads();
        // fold_line into the next layer.
        const qm31 alpha = alpha_sh;
        uint32_t *const *nxt = tp->lay[t + 1];
        for (uint32_t i = tid; i < n / 2; i += TAIL_THREADS) {
            const qm31 f0 = {{cur[0][2 * i], cur[1][2 * i]}, {cur[2][2 * i], cur[3][2 * i]}};
            const qm31 f1 = {{cur[0][2 * i + 1], cur[1][2 * i + 1]}, {cur[2][2 * i + 1], cur[3][2 * i + 1]}};
            const qm31 r = fold_pair(f0, f1, __ldg(tp->line_tw[t] + i), alpha);
            nxt[0][i] = r.a.a;
            nxt[1][i] = r.a.b;
            nxt[2][i] = r.b.a;
            nxt[3][i] = r.b.b;
        }
        __syncthreads();
    }
    if (tid == 0) fs_last(s, tp->lay[tp->n_tail], tp->last_log);
}

int launch_fri_tail(ProofState *s, const TailParams *tp, uint32_t jobs, size_t js, cudaStream_t st) {
    static std::atomic<uint64_t> attr_set{0};
    int rc = once_per_device(attr_set, [] {
        STWO_CUDA_TRY(cudaFuncSetAttribute(fri_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TAIL_SMEM));
        return (int)STWO_OK;
    });
    if (rc) return rc;
    fri_tail_kernel<<<jobs, TAIL_THREADS, TAIL_SMEM, st>>>(s, tp, 1u, js);
    STWO_LAUNCH_CHECK("fri_tail_kernel");
    return STWO_OK;
}

// Proof-of-work search (GrindOps::grind): nonce k is valid when the digest mixed with k
// (one compression of the digest with message [lo(k), hi(k), 0...]) has at least
// pow_bits trailing zero bits as a little-endian u128. Thread t tries t, t + G, t + 2G ...
// (G = grid size) and stops once its next nonce is not below the least valid nonce
// found so far, so the result is the least valid nonce below max_k * G.
__device__ __forceinline__ uint32_t ctz128(const uint32_t w[4]) {
    if (w[0]) return __ffs(w[0]) - 1;
    if (w[1]) return 32 + __ffs(w[1]) - 1;
    if (w[2]) return 64 + __ffs(w[2]) - 1;
    if (w[3]) return 96 + __ffs(w[3]) - 1;
    return 128;
}

__global__ void __launch_bounds__(256) grind_kernel(ProofState *s, uint32_t pow_bits, uint64_t max_k, size_t js) {
    s = job_ptr(s, js, blockIdx.y);
    const uint32_t one = 1;
    uint32_t d[8];
#pragma unroll
    for (int i = 0; i < 8; i++) d[i] = s->ch.digest[i];
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    volatile unsigned long long *best = &s->nonce;
    for (uint64_t k = 0; k < max_k; k++) {
        const uint64_t nonce = t + k * stride;
        if (nonce >= *best) return;
        uint32_t h[8], m[16] = {0};
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = d[i];
        m[0] = (uint32_t)nonce;
        m[1] = (uint32_t)(nonce >> 32);
        blake::compress(h, m, one);
        if (ctz128(h) >= pow_bits) {
            atomicMin(&s->nonce, (unsigned long long)nonce);
            return;
        }
    }
}

// After the search: mix the nonce and draw the raw query words (Queries::generate takes
// each u32 masked to the largest domain's log size).
__global__ void fs_finish_kernel(ProofState *s, uint32_t n_queries, size_t js) {
    s = job_ptr(s, js, blockIdx.x);  // one thread a job
    if (s->nonce == ~0ull) {
        s->error |= fs::ERR_GRIND;
        return;
    }
    fs::ch_mix_nonce(s->ch, s->nonce);
    for (uint32_t q = 0; q < n_queries; q += 8) {
        uint32_t w[8];
        fs::ch_draw_words(s->ch, w);
        for (uint32_t i = 0; i < 8 && q + i < n_queries; i++) s->query_words[q + i] = w[i];
    }
}

// Reads of single words from device buffers (decommitment values and witnesses).
struct GatherReq {
    const uint32_t *ptr;
    uint64_t idx;
};

__global__ void gather_kernel(const GatherReq *__restrict__ req, uint32_t n, uint32_t *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = req[i].ptr[req[i].idx];
}

// ------------------------------------------------------------------ host plumbing

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Stream-ordered device memory of one job: one slab from the library pool, sized by
// the job's bound and carved with a bump pointer (256-byte aligned), so a proof costs
// one pool allocation and one free; anything past the slab gets its own allocation.
// All of it is released, stream-ordered, when the job ends.
struct Arena {
    cudaStream_t st;
    uint8_t *slab = nullptr;
    uint64_t cap = 0, used = 0;
    std::vector<void *> extra;
    uint64_t bytes = 0;
    bool retain = false;  // the slab belongs to a ProveCache: not freed here
    explicit Arena(cudaStream_t s) : st(s) {}
    ~Arena() {
        if (slab && !retain) cudaFreeAsync(slab, st);
        for (void *p : extra) cudaFreeAsync(p, st);
    }
    void adopt(uint8_t *s, uint64_t c) {
        slab = s;
        cap = c;
        retain = true;
    }
    int reserve(uint64_t b) {
        void *p = nullptr;
        int rc = pool_alloc(&p, b, st);
        if (rc) return rc;
        slab = static_cast<uint8_t *>(p);
        cap = b;
        return STWO_OK;
    }
    template <typename T = uint32_t>
    T *alloc(size_t count) {
        size_t b = std::max<size_t>(count * sizeof(T), 16);
        b = (b + 255) & ~size_t(255);
        bytes += b;
        if (slab && used + b <= cap) {
            void *p = slab + used;
            used += b;
            return static_cast<T *>(p);
        }
        void *p = nullptr;
        if (pool_alloc(&p, b, st) != STWO_OK) return nullptr;
        extra.push_back(p);
        return static_cast<T *>(p);
    }
};

#define PV_ALLOC(var, T, count)  \
    T *var = ar.alloc<T>(count);  \
    if (!var) return STWO_ERR_OUT_OF_MEMORY  // pool_alloc recorded the message

#define PV_TRY(expr)              \
    do {                          \
        int _rc = (expr);         \
        if (_rc) return _rc;      \
    } while (0)

// Host image of device data uploaded in one copy: blobs appended at 256-byte aligned
// offsets of a device region whose address is known once the image is complete.
struct Upload {
    std::vector<uint8_t> host;
    size_t add(const void *p, size_t n) {
        size_t off = (host.size() + 255) & ~size_t(255);
        host.resize(off + n);
        if (p) memcpy(host.data() + off, p, n);
        else memset(host.data() + off, 0, n);
        return off;
    }
    template <class T>
    T *at(size_t off) {
        return reinterpret_cast<T *>(host.data() + off);
    }
};

// A Merkle tree whose columns are given per layer: the host keeps the layer buffers,
// the columns (for decommitment) and the device tables the tree kernel reads.
struct MerkleTree {
    std::vector<uint32_t *> layers;  // layers[l]: 2^l nodes of 8 words
    std::vector<std::pair<uint32_t, const uint32_t *>> cols;  // (log size, column), decreasing size, stable
    std::vector<const uint32_t *const *> level_tables;        // device column table per layer
    std::vector<uint32_t> level_n;
    std::vector<std::pair<size_t, uint32_t>> table_offsets;   // (image offset, layer) of each table
    size_t ticket_offset = 0;                                 // image offset of the tree kernel's tickets
    uint32_t *tickets = nullptr;
    uint32_t n_tickets = 0;
    uint32_t max_log = 0;
};

int plan_tree(MerkleTree &t, std::vector<std::pair<uint32_t, const uint32_t *>> cols, Arena &ar, Upload &up) {
    std::stable_sort(cols.begin(), cols.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    t.cols = cols;
    t.max_log = cols[0].first;
    t.layers.assign(t.max_log + 1, nullptr);
    t.level_tables.assign(t.max_log + 1, nullptr);
    t.level_n.assign(t.max_log + 1, 0);
    for (int l = (int)t.max_log; l >= 0; l--) {
        PV_ALLOC(layer, uint32_t, (size_t)8 << l);
        t.layers[l] = layer;
        std::vector<const uint32_t *> lc;
        for (auto &c : cols)
            if (c.first == (uint32_t)l) lc.push_back(c.second);
        if (!lc.empty()) {
            t.table_offsets.push_back({up.add(lc.data(), lc.size() * sizeof(void *)), (uint32_t)l});
            t.level_n[l] = (uint32_t)lc.size();
        }
    }
    // zeroed in the image; the kernel leaves them zeroed
    t.n_tickets = merkle_tree_tickets(t.max_log);
    t.ticket_offset = up.add(nullptr, 4 * std::max<size_t>(t.n_tickets, 1));
    return STWO_OK;
}

// Word reads from device memory, planned on the host and executed in one launch.
struct Gatherer {
    std::vector<GatherReq> reqs;
    std::vector<uint32_t> vals;
    size_t add(const uint32_t *p, uint64_t idx) {
        reqs.push_back({p, idx});
        return reqs.size() - 1;
    }
    int run(Arena &ar, cudaStream_t st) {
        vals.assign(reqs.size(), 0);
        if (reqs.empty()) return STWO_OK;
        PV_ALLOC(dreq, GatherReq, reqs.size());
        PV_ALLOC(dout, uint32_t, reqs.size());
        const size_t req_bytes = reqs.size() * sizeof(GatherReq);
        void *stage = nullptr;
        PV_TRY(host_stage(req_bytes + reqs.size() * 4, &stage));
        memcpy(stage, reqs.data(), req_bytes);
        uint32_t *out_stage = reinterpret_cast<uint32_t *>(static_cast<uint8_t *>(stage) + req_bytes);
        STWO_CUDA_TRY(cudaMemcpyAsync(dreq, stage, req_bytes, cudaMemcpyHostToDevice, st));
        gather_kernel<<<(unsigned)((reqs.size() + 255) / 256), 256, 0, st>>>(dreq, (uint32_t)reqs.size(), dout);
        STWO_LAUNCH_CHECK("gather_kernel");
        STWO_CUDA_TRY(cudaMemcpyAsync(out_stage, dout, reqs.size() * 4, cudaMemcpyDeviceToHost, st));
        PV_TRY(wait_stream(st));
        memcpy(vals.data(), out_stage, reqs.size() * 4);
        return STWO_OK;
    }
};

// MerkleProver::decommit, planned: layer by layer from the leaves, the nodes to open
// are the parents of the layer below's opened nodes and the layer's queried positions.
// A child that is not itself opened goes to the hash witness; the column values of an
// opened node are queried values when the node is a queried position, else column
// witness.
struct TreeDecommit {
    std::vector<size_t> hash_words;            // 8 gather indices per witness hash
    std::vector<size_t> column_witness;        // gather indices
    std::vector<std::vector<size_t>> queried;  // per column (tree order), gather indices
};

TreeDecommit plan_decommit(const MerkleTree &t, const std::map<uint32_t, std::vector<uint64_t>> &queries,
                           Gatherer &g) {
    TreeDecommit d;
    d.queried.assign(t.cols.size(), {});
    std::vector<uint64_t> below;  // opened nodes of the layer below, sorted
    for (int l = (int)t.max_log; l >= 0; l--) {
        std::vector<size_t> lc;
        for (size_t i = 0; i < t.cols.size(); i++)
            if (t.cols[i].first == (uint32_t)l) lc.push_back(i);
        std::set<uint64_t> colq;
        auto it = queries.find((uint32_t)l);
        if (it != queries.end()) colq.insert(it->second.begin(), it->second.end());
        std::set<uint64_t> nodes(colq);
        for (uint64_t q : below) nodes.insert(q >> 1);
        const std::set<uint64_t> opened_below(below.begin(), below.end());
        for (uint64_t node : nodes) {
            if (l < (int)t.max_log) {
                for (uint64_t child : {2 * node, 2 * node + 1})
                    if (!opened_below.count(child))
                        for (int w = 0; w < 8; w++) d.hash_words.push_back(g.add(t.layers[l + 1], child * 8 + w));
            }
            const bool queried = colq.count(node) > 0;
            for (size_t ci : lc) {
                size_t gi = g.add(t.cols[ci].second, node);
                if (queried) d.queried[ci].push_back(gi);
                else d.column_witness.push_back(gi);
            }
        }
        below.assign(nodes.begin(), nodes.end());
    }
    return d;
}

// Proof byte stream.
struct Writer {
    std::vector<uint8_t> b;
    void u32(uint32_t v) { b.insert(b.end(), (uint8_t *)&v, (uint8_t *)&v + 4); }
    void u64(uint64_t v) { b.insert(b.end(), (uint8_t *)&v, (uint8_t *)&v + 8); }
    void bytes(const void *p, size_t n) { b.insert(b.end(), (const uint8_t *)p, (const uint8_t *)p + n); }
    void q(qm31 v) {
        u32(v.a.a);
        u32(v.a.b);
        u32(v.b.a);
        u32(v.b.b);
    }
};

void write_decommitment(Writer &w, const TreeDecommit &d, const std::vector<uint32_t> &vals) {
    w.u64(d.hash_words.size() / 8);
    for (size_t gi : d.hash_words) w.u32(vals[gi]);
    w.u64(d.column_witness.size());
    for (size_t gi : d.column_witness) w.u32(vals[gi]);
}

std::vector<uint64_t> fold_queries(const std::vector<uint64_t> &q, uint32_t n) {
    std::vector<uint64_t> r;
    for (uint64_t v : q) {
        uint64_t f = v >> n;
        if (r.empty() || r.back() != f) r.push_back(f);
    }
    return r;
}

// compute_decommitment_positions_and_witness_evals with fold step 1: every query
// opens its folding pair; the partner that is not itself a query is a witness.
void fri_positions(const std::vector<uint64_t> &queries, std::vector<uint64_t> &positions,
                   std::vector<uint64_t> &witness) {
    positions.clear();
    witness.clear();
    size_t i = 0;
    while (i < queries.size()) {
        const uint64_t start = queries[i] & ~1ull;
        size_t j = i;
        while (j < queries.size() && (queries[j] >> 1) == (queries[i] >> 1)) j++;
        for (uint64_t p = start; p < start + 2; p++) {
            positions.push_back(p);
            bool q = false;
            for (size_t k = i; k < j; k++) q = q || queries[k] == p;
            if (!q) witness.push_back(p);
        }
        i = j;
    }
}

struct Job {
    uint32_t L, N, B, n_queries, pow_bits;
};

int validate(const Job &j) {
    STWO_REQUIRE(j.N >= 3 && j.N <= WF_MAX_TRACE_COLS, STWO_ERR_UNSUPPORTED_SIZE,
                 "wide-Fibonacci proofs need 3..%u columns, got %u", WF_MAX_TRACE_COLS, j.N);
    STWO_REQUIRE(j.B >= 1 && j.B <= 4, STWO_ERR_UNSUPPORTED_SIZE, "log blowup %u unsupported (1..4)", j.B);
    STWO_REQUIRE(j.L >= 2 && j.L + 1 + j.B <= MAX_DOMAIN_LOG, STWO_ERR_UNSUPPORTED_SIZE,
                 "trace log size %u with log blowup %u unsupported", j.L, j.B);
    STWO_REQUIRE(j.n_queries >= 1 && j.n_queries <= MAX_QUERIES, STWO_ERR_UNSUPPORTED_SIZE, "%u queries unsupported",
                 j.n_queries);
    STWO_REQUIRE(j.pow_bits <= 32, STWO_ERR_UNSUPPORTED_SIZE, "pow_bits %u unsupported (0..32)", j.pow_bits);
    return STWO_OK;
}

// Device bytes one job allocates (an upper bound of the arena's total).
uint64_t job_device_bytes(const Job &j, bool own_twiddles) {
    auto r = [](uint64_t b) { return (std::max<uint64_t>(b, 16) + 255) & ~uint64_t(255); };
    const uint64_t n = 1ull << j.L, ne = n << 1, nb = n << j.B, neb = ne << j.B;
    auto tree = [&](uint32_t log) {
        uint64_t t = 0;
        for (uint32_t l = 0; l <= log; l++) t += r(32ull << l);
        return t;
    };
    uint64_t b = 0;
    if (own_twiddles) b += 2 * r(4 * nb);
    b += 2 * r(4 * n);                                    // a0, a1
    b += j.N * (r(4 * n) + r(4 * nb));                    // trace coefficients, trace evaluations
    if (j.B > 1) b += j.N * r(4 * ne);                    // trace on the composition domain
    b += tree(j.L + j.B) + tree(j.L + 1 + j.B);           // trace and composition trees
    b += 4 * r(4 * ne) + 4 * r(4 * neb);                  // composition, its evaluations
    b += r(16 * j.N);                                     // coefficient powers
    const uint64_t eap_blocks = (uint64_t)j.N * eval_at_point_blocks(j.L, 0) + 4 * eval_at_point_blocks(j.L + 1, 0);
    b += r(16 * eap_blocks);                              // eval_at_point partials
    b += 4 * r(4 * neb) + 4 * r(4 * nb);                  // quotients
    b += tree(j.L + 1 + j.B);                             // FRI first layer tree
    for (uint32_t l = j.B; l <= j.L + j.B; l++) b += 4 * r(4ull << l) + tree(l);  // FRI layers
    // the uploaded image: state and sampled values, tickets, quotient parameters, tables
    b += r(sizeof(ProofState) + 16 * (j.N + 4)) + r(4 * (j.N + 4)) + 2 * r(sizeof(QuotParamsDev));
    b += 2 * r(8 * j.N) + r(sizeof(EapDevPoly) * (j.N + 4)) + (2 * (j.L + j.B) + 8) * r(64) + r(8 * j.N);
    b += r(sizeof(TailParams));
    b += 3 * r(16 * j.N);                                 // FFT column tables (src, dst) of the trace
    auto tickets = [&](uint32_t log) { return r(4 * std::max<uint64_t>(merkle_tree_tickets(log), 1)); };
    b += tickets(j.L + j.B) + 2 * tickets(j.L + 1 + j.B);  // Merkle tree tickets
    for (uint32_t l = j.B; l <= j.L + j.B; l++) b += tickets(l);
    const uint64_t words = (uint64_t)j.n_queries * ((j.L + 2 + j.B) * 8 * 3 * 8 + 2 * (j.N + 16));
    b += r(words * sizeof(GatherReq)) + r(words * 4);     // decommitment gather
    return b;
}

// Timing events of one thread's proofs (reused; created on first use per device).
struct PhaseEvents {
    cudaEvent_t ev[5] = {};
    int device = -1;
    ~PhaseEvents() {
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
    }
    int ensure() {
        int dev = 0;
        STWO_CUDA_TRY(cudaGetDevice(&dev));
        if (device == dev) return STWO_OK;
        for (auto &e : ev) {
            if (e) cudaEventDestroy(e);
            e = nullptr;
            STWO_CUDA_TRY(cudaEventCreate(&e));
        }
        device = dev;
        return STWO_OK;
    }
};
thread_local PhaseEvents t_phase;

}  // namespace

void prove_cache_release(ProveCache *c, cudaStream_t st) {
    if (!c) return;
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->slab) cudaFreeAsync(c->slab, st);
    const uint64_t replays = c->replays;  // a running count over the cache's life
    *c = ProveCache{};
    c->replays = replays;
}

namespace {

// One job's device layout and host tables: everything a proof plans before its first
// launch. The plan depends only on the job's shape, so jobs of one shape planned into
// equal slabs lie at the same offsets, and job k's memory is job 0's moved by the slabs'
// distance: one launch sequence (jobs x stride) then serves all of them.
struct JobLayout {
    const uint32_t *tw = nullptr, *itw = nullptr;
    uint64_t tsz = 0;
    uint32_t *own_tw = nullptr, *own_itw = nullptr;
    uint32_t *a0 = nullptr, *a1 = nullptr;
    std::vector<uint32_t *> tpoly, tev, text, comp, cev, qc, qt;
    qm31 *powers = nullptr;
    uint32_t n_layers = 0;
    std::vector<std::vector<uint32_t *>> lay;
    uint32_t eap_n = 0, eap_total = 0, eap_iter = 0;
    qm31 *eap_partials = nullptr;
    Upload up;
    size_t off_state = 0, off_tickets = 0, off_qc = 0, off_qt = 0, off_tpoly = 0, off_text = 0, off_eap = 0;
    size_t off_fft_interp = 0, off_fft_eval = 0, off_fft_ext = 0, off_tail = 0;
    MerkleTree t_trace, t_comp, t_fri0;
    std::vector<MerkleTree> t_lay;
    uint32_t li0 = 0, li_circle = 0;
    uint8_t *dev_img = nullptr;
    ProofState *dstate = nullptr;
    qm31 *dsampled = nullptr;
    uint32_t *dtickets = nullptr;
    QuotParamsDev *dqc = nullptr, *dqt = nullptr;

    uint8_t *dev_at(size_t off) const { return dev_img + off; }

    int plan(const Job &j, Arena &ar, const uint32_t *tw_in, const uint32_t *itw_in, uint64_t tsz_in) {
        const uint32_t L = j.L, N = j.N, B = j.B, E = L + 1, D = E + B;
        const uint64_t rows = 1ull << L;
        // ---- buffers (all of the job's device memory, before the first launch)
        tw = tw_in;
        itw = itw_in;
        tsz = tsz_in;
        if (tw_in || itw_in) {
            STWO_REQUIRE(tw_in && itw_in && is_pow2(tsz_in) && tsz_in >= (1ull << (L + B)), STWO_ERR_INVALID_ARGUMENT,
                         "twiddle tree of %llu entries does not cover domain log size %u", (unsigned long long)tsz_in, D);
        } else {
            tsz = 1ull << (L + B);
            own_tw = ar.alloc<uint32_t>(tsz);
            own_itw = ar.alloc<uint32_t>(tsz);
            STWO_REQUIRE(own_tw && own_itw, STWO_ERR_OUT_OF_MEMORY, "twiddle allocation failed");
            tw = own_tw;
            itw = own_itw;
        }
        a0 = ar.alloc<uint32_t>(rows);
        a1 = ar.alloc<uint32_t>(rows);
        if (!a0 || !a1) return STWO_ERR_OUT_OF_MEMORY;  // pool_alloc recorded the message
        tpoly.assign(N, nullptr);
        tev.assign(N, nullptr);
        text.assign(N, nullptr);
        for (uint32_t c = 0; c < N; c++) {
            PV_ALLOC(p, uint32_t, rows);
            PV_ALLOC(e, uint32_t, rows << B);
            tpoly[c] = p;
            tev[c] = e;
            if (B == 1) {
                text[c] = e;  // the committed evaluations are already on CanonicCoset(L + 1)
            } else {
                PV_ALLOC(x, uint32_t, 1ull << E);
                text[c] = x;
            }
        }
        powers = ar.alloc<qm31>(N);
        if (!powers) return STWO_ERR_OUT_OF_MEMORY;
        comp.assign(4, nullptr);
        cev.assign(4, nullptr);
        qc.assign(4, nullptr);
        qt.assign(4, nullptr);
        for (int k = 0; k < 4; k++) {
            PV_ALLOC(c, uint32_t, 1ull << E);
            PV_ALLOC(e, uint32_t, 1ull << D);
            PV_ALLOC(a, uint32_t, 1ull << D);
            PV_ALLOC(b, uint32_t, 1ull << (L + B));
            comp[k] = c;
            cev[k] = e;
            qc[k] = a;
            qt[k] = b;
        }
        // FRI layers: inner logs D-1 .. B+1, then the last layer (log B)
        n_layers = D - 1 - B;
        STWO_REQUIRE(n_layers <= MAX_LAYERS && L + B - 1 > B, STWO_ERR_UNSUPPORTED_SIZE, "FRI layer count unsupported");
        lay.assign(n_layers + 1, std::vector<uint32_t *>(4));
        for (uint32_t li = 0; li <= n_layers; li++)
            for (int k = 0; k < 4; k++) {
                PV_ALLOC(c, uint32_t, 1ull << (D - 1 - li));
                lay[li][k] = c;
            }
        eap_n = N + 4;
        eap_total = 0;
        std::vector<EapDevPoly> eap(eap_n);
        std::vector<uint32_t> eap_logs(eap_n);
        for (uint32_t i = 0; i < eap_n; i++) eap_logs[i] = i < N ? L : E;
        eap_iter = eval_at_point_iter_log(eap_logs.data(), eap_n);
        for (uint32_t i = 0; i < eap_n; i++) {
            eap[i] = {i < N ? tpoly[i] : comp[i - N], eap_logs[i], eap_total};
            eap_total += eval_at_point_blocks(eap_logs[i], eap_iter);
        }
        eap_partials = ar.alloc<qm31>(eap_total);
        if (!eap_partials) return STWO_ERR_OUT_OF_MEMORY;

        // ---- the uploaded image: state (+ sampled values), tickets, quotient parameters, tables
        off_state = up.add(nullptr, sizeof(ProofState) + sizeof(qm31) * eap_n);
        up.at<ProofState>(off_state)->nonce = ~0ull;
        off_tickets = up.add(nullptr, 4 * eap_n);
        auto qpc = std::make_unique<QuotParamsDev>();
        auto qpt = std::make_unique<QuotParamsDev>();
        memset(qpc.get(), 0, sizeof(QuotParamsDev));
        memset(qpt.get(), 0, sizeof(QuotParamsDev));
        const cpoint *circle_tab = nullptr;
        PV_TRY(circle_point_table(&circle_tab));
        quot_init_static(*qpc, half_coset_init(D), half_coset_step(D), D, qc.data(), circle_tab);
        quot_init_static(*qpt, half_coset_init(L + B), half_coset_step(L + B), L + B, qt.data(), circle_tab);
        qpc->n_batches = qpt->n_batches = 1;
        qpc->batch_end[0] = 4;
        qpt->batch_end[0] = N;
        for (int k = 0; k < 4; k++) {
            qpc->cols[k] = cev[k];
            qpc->col_idx[k] = (uint16_t)k;
        }
        for (uint32_t c = 0; c < N; c++) {
            qpt->cols[c] = tev[c];
            qpt->col_idx[c] = (uint16_t)c;
        }
        off_qc = up.add(qpc.get(), sizeof(QuotParamsDev));
        off_qt = up.add(qpt.get(), sizeof(QuotParamsDev));
        off_tpoly = up.add(tpoly.data(), sizeof(void *) * N);
        off_text = up.add(text.data(), sizeof(void *) * N);
        off_eap = up.add(eap.data(), sizeof(EapDevPoly) * eap_n);
        // (src, dst) tables of the trace transforms: with more than 64 columns each pass is
        // one launch over its table.
        auto fft_table = [&](const std::vector<uint32_t *> &src, const std::vector<uint32_t *> &dst) {
            std::vector<const void *> t(2 * N);
            for (uint32_t c = 0; c < N; c++) {
                t[2 * c] = src[c];
                t[2 * c + 1] = dst[c];
            }
            return up.add(t.data(), sizeof(void *) * 2 * N);
        };
        off_fft_interp = fft_table(tpoly, tpoly);
        off_fft_eval = fft_table(tpoly, tev);
        off_fft_ext = B > 1 ? fft_table(tpoly, text) : 0;
        t_lay.assign(n_layers, MerkleTree{});
        {
            std::vector<std::pair<uint32_t, const uint32_t *>> cols;
            for (uint32_t c = 0; c < N; c++) cols.push_back({L + B, tev[c]});
            PV_TRY(plan_tree(t_trace, cols, ar, up));
            cols.clear();
            for (int k = 0; k < 4; k++) cols.push_back({D, cev[k]});
            PV_TRY(plan_tree(t_comp, cols, ar, up));
            cols.clear();
            for (int k = 0; k < 4; k++) cols.push_back({D, qc[k]});
            for (int k = 0; k < 4; k++) cols.push_back({L + B, qt[k]});
            PV_TRY(plan_tree(t_fri0, cols, ar, up));
            for (uint32_t li = 0; li < n_layers; li++) {
                cols.clear();
                for (int k = 0; k < 4; k++) cols.push_back({D - 1 - li, lay[li][k]});
                PV_TRY(plan_tree(t_lay[li], cols, ar, up));
            }
        }
        // The FRI tail: inner layers of log size <= TAIL_MAX_LOG (from li0 on) and the last
        // layer run in one launch. The trace quotient folds into layer 1 (log L + B - 1).
        li0 = D - 1 > TAIL_MAX_LOG ? D - 1 - TAIL_MAX_LOG : 0;
        li_circle = D - (L + B);
        off_tail = 0;
        {
            auto tp = std::make_unique<TailParams>();
            memset(tp.get(), 0, sizeof(TailParams));
            tp->li0 = li0;
            tp->n_tail = n_layers - li0;
            tp->lg0 = D - 1 - li0;
            tp->last_log = B;
            tp->circle_t = li_circle >= li0 ? li_circle - li0 : ~0u;
            for (int k = 0; k < 4; k++) tp->qt[k] = qt[k];
            tp->circle_tw = itw + (tsz - (1ull << (L + B - 1)));
            for (uint32_t t = 0; t <= tp->n_tail; t++)
                for (int k = 0; k < 4; k++) tp->lay[t][k] = lay[li0 + t][k];
            for (uint32_t t = 0; t < tp->n_tail; t++) {
                const uint32_t lg = tp->lg0 - t;
                for (uint32_t l = 0; l <= lg; l++) tp->nodes[t][l] = reinterpret_cast<uint4 *>(t_lay[li0 + t].layers[l]);
                tp->line_tw[t] = itw + (tsz - (1ull << lg));
            }
            off_tail = up.add(tp.get(), sizeof(TailParams));
        }
        dev_img = ar.alloc<uint8_t>(up.host.size());
        if (!dev_img) return STWO_ERR_OUT_OF_MEMORY;
        auto fix_tables = [&](MerkleTree &t) {
            for (auto &f : t.table_offsets)
                t.level_tables[f.second] = reinterpret_cast<const uint32_t *const *>(dev_at(f.first));
            t.tickets = reinterpret_cast<uint32_t *>(dev_at(t.ticket_offset));
        };
        fix_tables(t_trace);
        fix_tables(t_comp);
        fix_tables(t_fri0);
        for (auto &t : t_lay) fix_tables(t);
        dstate = reinterpret_cast<ProofState *>(dev_at(off_state));
        dsampled = reinterpret_cast<qm31 *>(dev_at(off_state) + sizeof(ProofState));
        dtickets = reinterpret_cast<uint32_t *>(dev_at(off_tickets));
        dqc = reinterpret_cast<QuotParamsDev *>(dev_at(off_qc));
        dqt = reinterpret_cast<QuotParamsDev *>(dev_at(off_qt));
        return STWO_OK;
    }
};

// K proofs of one shape (job j; inputs a0_in[k], a1_in[k]) in one launch sequence.
// K = 1 is the single proof, which may use a ProveCache; K > 1 takes the caller's
// twiddle tree and plans the jobs into K equal slabs. proofs[k] receive the proof
// bytes; job_rc[k] (K > 1) each job's status, and the call's own status is that of
// the launch sequence. With K = 1 the job's status is the call's.
int prove_jobs(const Job &j, uint32_t K, const uint32_t *const *a0_in, const uint32_t *const *a1_in,
               const uint32_t *tw_in, const uint32_t *itw_in, uint64_t tsz_in, std::vector<uint8_t> *proofs,
               int *job_rc, cudaStream_t st, stwo_prove_stats *stats, ProveCache *cache) {
    PV_TRY(validate(j));
    STWO_REQUIRE(K >= 1 && K <= MAX_JOBS_PER_LAUNCH, STWO_ERR_INVALID_ARGUMENT, "%u proofs in one launch sequence",
                 K);
    STWO_REQUIRE(K == 1 || (tw_in && itw_in && !cache), STWO_ERR_INVALID_ARGUMENT,
                 "several proofs in one launch sequence take the caller's twiddle tree and no proof cache");
    const uint32_t L = j.L, N = j.N, B = j.B, E = L + 1, D = E + B;
    const uint64_t rows = 1ull << L;
    const double t0 = now_ms();
    const uint64_t launches0 = t_kernel_launches;
    // A cache (a server worker's) keeps the job's slab after the proof, so that the next
    // proof of the same shape finds every buffer, table and parameter block at the same
    // address: its launch sequence is captured as a CUDA graph on that second proof
    // and replayed from the third on. Only for jobs with a caller's twiddle tree and
    // log_n_rows >= 3 (a 4-point transform reads a twiddle back to the host).
    int dev = 0;
    STWO_CUDA_TRY(cudaGetDevice(&dev));
    const bool cacheable = K == 1 && cache && tw_in && itw_in && L >= 3;
    const uint32_t key[5] = {j.L, j.N, j.B, j.n_queries, j.pow_bits};
    // Launch shapes (and the eval_at_point descriptors) follow the tunables, so a change
    // of any tunable retires the cache.
    const uint64_t tgen = tunables_generation();
    const bool hit = cacheable && cache->valid && cache->device == dev && cache->tw == tw_in &&
                     cache->itw == itw_in && cache->tsz == tsz_in && memcmp(cache->key, key, sizeof(key)) == 0 &&
                     cache->tunables_gen == tgen;
    if (cache && cache->valid && !hit) prove_cache_release(cache, st);
    // Phase events are recorded whenever the launch sequence may be captured, so that a
    // graph always carries them.
    const bool timing = stats || cacheable;
    if (timing) PV_TRY(t_phase.ensure());
    cudaEvent_t *ev = t_phase.ev;
    Arena ar(st);
    // One job's slab; K jobs take K equal slabs, and job k's memory is job 0's moved by k * S.
    const uint64_t S = (job_device_bytes(j, !(tw_in || itw_in)) + 255) & ~uint64_t(255);
    if (hit) ar.adopt(cache->slab, cache->cap);
    else PV_TRY(ar.reserve(K == 1 ? job_device_bytes(j, !(tw_in || itw_in)) : S * K));
    if (timing) STWO_CUDA_TRY(cudaEventRecord(ev[0], st));
    std::vector<JobLayout> jl(K);
    if (K == 1) {
        PV_TRY(jl[0].plan(j, ar, tw_in, itw_in, tsz_in));
    } else {
        uint64_t used0 = 0;
        for (uint32_t k = 0; k < K; k++) {
            Arena sub(st);
            sub.adopt(ar.slab + (size_t)k * S, S);
            PV_TRY(jl[k].plan(j, sub, tw_in, itw_in, tsz_in));
            if (k == 0) used0 = sub.used;
            STWO_REQUIRE(sub.extra.empty() && sub.used == used0, STWO_ERR_UNSUPPORTED_SIZE,
                         "a job of the batch does not fit its slab");
            ar.bytes += sub.bytes;
        }
        ar.used = ar.cap;  // the jobs' slabs are taken: later allocations (the gather) go past them
    }
    JobLayout &J = jl[0];
    const uint32_t *tw = J.tw, *itw = J.itw;
    const uint64_t tsz = J.tsz;
    uint32_t *own_tw = J.own_tw, *own_itw = J.own_itw;
    uint32_t *a0 = J.a0, *a1 = J.a1;
    std::vector<uint32_t *> &tpoly = J.tpoly, &tev = J.tev, &text = J.text, &comp = J.comp, &cev = J.cev,
                            &qc = J.qc, &qt = J.qt;
    std::vector<std::vector<uint32_t *>> &lay = J.lay;
    qm31 *powers = J.powers;
    const uint32_t n_layers = J.n_layers, eap_n = J.eap_n, eap_total = J.eap_total, eap_iter = J.eap_iter;
    qm31 *eap_partials = J.eap_partials;
    MerkleTree &t_trace = J.t_trace, &t_comp = J.t_comp, &t_fri0 = J.t_fri0;
    std::vector<MerkleTree> &t_lay = J.t_lay;
    const uint32_t li0 = J.li0, li_circle = J.li_circle;
    ProofState *dstate = J.dstate;
    qm31 *dsampled = J.dsampled;
    uint32_t *dtickets = J.dtickets;
    QuotParamsDev *dqc = J.dqc, *dqt = J.dqt;
    const size_t off_tpoly = J.off_tpoly, off_text = J.off_text, off_eap = J.off_eap, off_tail = J.off_tail;
    const size_t off_fft_interp = J.off_fft_interp, off_fft_eval = J.off_fft_eval, off_fft_ext = J.off_fft_ext;
    auto dev_at = [&](size_t off) { return J.dev_at(off); };
    (void)rows;

    {
        // the jobs' images, staged through pinned memory (the stage's next use comes after
        // a wait on st) and uploaded in one copy
        const size_t img = J.up.host.size();
        for (uint32_t k = 1; k < K; k++)
            STWO_REQUIRE(jl[k].up.host.size() == img, STWO_ERR_UNSUPPORTED_SIZE, "the batch's images differ");
        void *stage = nullptr;
        PV_TRY(host_stage(img * K, &stage));
        for (uint32_t k = 0; k < K; k++) memcpy(static_cast<uint8_t *>(stage) + img * k, jl[k].up.host.data(), img);
        if (K == 1) STWO_CUDA_TRY(cudaMemcpyAsync(J.dev_img, stage, img, cudaMemcpyHostToDevice, st));
        else STWO_CUDA_TRY(cudaMemcpy2DAsync(J.dev_img, S, stage, img, img, K, cudaMemcpyHostToDevice, st));
    }
    for (uint32_t k = 0; k < K; k++) {
        STWO_CUDA_TRY(cudaMemcpyAsync(jl[k].a0, a0_in[k], rows * 4, cudaMemcpyDefault, st));
        STWO_CUDA_TRY(cudaMemcpyAsync(jl[k].a1, a1_in[k], rows * 4, cudaMemcpyDefault, st));
    }

    // The launch sequence from the trace to the query words: device work only, no host
    // wait, every address inside the slab or the caller's twiddle tree.
    auto record = [&](int k, bool capturing) -> int {
        if (!timing) return STWO_OK;
        STWO_CUDA_TRY(capturing ? cudaEventRecordWithFlags(ev[k], st, cudaEventRecordExternal)
                                : cudaEventRecord(ev[k], st));
        return STWO_OK;
    };
    const size_t js = K > 1 ? S : 0;  // the jobs' memory stride
    // A transform over every job's columns: with one job the prover's own tables (in its
    // image, so the sequence stays capturable); with several, all jobs' columns in one
    // launch a pass (the call stages their table).
    auto fft_all = [&](const std::vector<uint32_t *> &src, const std::vector<uint32_t *> &dst, uint32_t n_log,
                       uint32_t coeff_log, const uint32_t *tree, bool inv, const void *table) -> int {
        std::vector<const uint32_t *> s;
        std::vector<uint32_t *> d;
        for (uint32_t k = 0; k < K; k++)
            for (size_t i = 0; i < src.size(); i++) {
                s.push_back(job_ptr<const uint32_t>(src[i], js, k));
                d.push_back(job_ptr(dst[i], js, k));
            }
        return fft_columns_tab(s.data(), d.data(), (uint32_t)s.size(), n_log, coeff_log, tree, tsz, inv, st,
                               K == 1 ? table : nullptr);
    };
    auto launch_all = [&](bool capturing) -> int {
        // ---- 1. trace: twiddles, generation, interpolation, evaluation, tree
        if (own_tw)
            PV_TRY(stwo_precompute_twiddles(half_coset_init(D), half_coset_step(D), L + B, own_tw, own_itw, st));
        {
            const uint32_t threads = rows < (uint64_t)device_sm_count() * 256 ? 64 : 256;
            const uint64_t blocks =
                std::min<uint64_t>((rows + threads - 1) / threads, (uint64_t)device_sm_count() * 16);
            wide_fib_trace_kernel<<<dim3((unsigned)blocks, K), threads, 0, st>>>(
                a0, a1, reinterpret_cast<uint32_t *const *>(dev_at(off_tpoly)), N, rows, js);
            STWO_LAUNCH_CHECK("wide_fib_trace_kernel");
        }
        // The trace columns are interpolated in place: they become the coefficient columns.
        PV_TRY(fft_all(tpoly, tpoly, L, L, itw, true, dev_at(off_fft_interp)));
        PV_TRY(fft_all(tpoly, tev, L + B, L, tw, false, dev_at(off_fft_eval)));
        auto commit = [&](MerkleTree &t) {
            return merkle_tree_dev_async(t.max_log, t.level_tables.data(), t.level_n.data(), t.layers.data(), t.tickets,
                                         t.n_tickets, K, js, st);
        };
        PV_TRY(commit(t_trace));
        fs_trace_kernel<<<K, 32, 0, st>>>(dstate, t_trace.layers[0], powers, N - 2, js);
        STWO_LAUNCH_CHECK("fs_trace_kernel");
        PV_TRY(record(1, capturing));

        // ---- 2. composition on CanonicCoset(L + 1), committed on CanonicCoset(L + 1 + B)
        if (B > 1) PV_TRY(fft_all(tpoly, text, E, L, tw, false, dev_at(off_fft_ext)));
        uint32_t den_half[2];
        vanishing_inverses(L, den_half);
        PV_TRY(wide_fib_dev_async(reinterpret_cast<const uint32_t *const *>(dev_at(off_text)), N, E,
                                  reinterpret_cast<const uint32_t *>(powers), den_half, comp.data(), K, js, st));
        PV_TRY(fft_all(comp, comp, E, E, itw, true, nullptr));  // in place -> coefficients
        PV_TRY(fft_all(comp, cev, D, E, tw, false, nullptr));
        PV_TRY(commit(t_comp));
        fs_comp_kernel<<<K, 1, 0, st>>>(dstate, t_comp.layers[0], js);
        STWO_LAUNCH_CHECK("fs_comp_kernel");
        PV_TRY(record(2, capturing));

        // ---- 3. out-of-domain sampling
        PV_TRY(eval_at_points_dev_async(dev_at(off_eap), eap_n, eap_iter, eap_total, dstate->oods, dsampled,
                                        eap_partials, dtickets, K, js, st));
        fs_oods_kernel<<<K, 256, 0, st>>>(dstate, dsampled, powers, N, L, vanishing_shift(L), dqc, dqt, js);
        STWO_LAUNCH_CHECK("fs_oods_kernel");
        PV_TRY(record(3, capturing));

        // ---- 4. DEEP quotients (largest columns first) and the FRI commitment
        PV_TRY(quotients_dev_async(dqc, D, 4, K, js, st));
        PV_TRY(quotients_dev_async(dqt, L + B, N, K, js, st));
        PV_TRY(commit(t_fri0));
        fs_layer_kernel<<<K, 1, 0, st>>>(dstate, t_fri0.layers[0], 2, 0, js);
        STWO_LAUNCH_CHECK("fs_layer_kernel");
        for (int k = 0; k < 4; k++) {
            if (K == 1) STWO_CUDA_TRY(cudaMemsetAsync(lay[0][k], 0, 4ull << (D - 1), st));
            else STWO_CUDA_TRY(cudaMemset2DAsync(lay[0][k], js, 0, 4ull << (D - 1), K, st));
        }
        {
            std::vector<const uint32_t *> s(qc.begin(), qc.end());
            PV_TRY(fold_async(s.data(), 1ull << D, stwo_qm31{}, itw, tsz - (1ull << (D - 1)), lay[0].data(), true, st,
                              &dstate->alphas[0], K, js));
        }
        for (uint32_t li = 0; li < li0; li++) {
            const uint32_t lg = D - 1 - li;
            if (li == li_circle) {
                // The trace quotient folds into this layer with the previous layer's alpha.
                std::vector<const uint32_t *> s(qt.begin(), qt.end());
                PV_TRY(fold_async(s.data(), 1ull << (L + B), stwo_qm31{}, itw, tsz - (1ull << lg), lay[li].data(), true,
                                  st, &dstate->alphas[li], K, js));
            }
            PV_TRY(commit(t_lay[li]));
            fs_layer_kernel<<<K, 1, 0, st>>>(dstate, t_lay[li].layers[0], 3 + li, li + 1, js);
            STWO_LAUNCH_CHECK("fs_layer_kernel");
            std::vector<const uint32_t *> s(lay[li].begin(), lay[li].end());
            PV_TRY(fold_async(s.data(), 1ull << lg, stwo_qm31{}, itw, tsz - (1ull << lg), lay[li + 1].data(), false, st,
                              &dstate->alphas[li + 1], K, js));
        }
        PV_TRY(launch_fri_tail(dstate, reinterpret_cast<const TailParams *>(dev_at(off_tail)), K, js, st));
        PV_TRY(record(4, capturing));

        // ---- 5. proof of work and query words, then the channel's record to the host
        {
            const uint64_t want = 1ull << std::min<uint32_t>(j.pow_bits + 2, 24);  // a few times the expected tries
            const uint64_t threads =
                std::max<uint64_t>(256, std::min<uint64_t>(want, (uint64_t)device_sm_count() * 1024));
            const uint64_t blocks = (threads + 255) / 256, grid = blocks * 256;
            const uint64_t max_k = ((1ull << (j.pow_bits + 6)) + grid - 1) / grid + 1;  // gives up after 2^(pow_bits+6)
            grind_kernel<<<dim3((unsigned)blocks, K), 256, 0, st>>>(dstate, j.pow_bits, max_k, js);
            STWO_LAUNCH_CHECK("grind_kernel");
            fs_finish_kernel<<<K, 1, 0, st>>>(dstate, j.n_queries, js);
            STWO_LAUNCH_CHECK("fs_finish_kernel");
        }
        return STWO_OK;
    };

    const bool cache_ok = cacheable && ar.extra.empty();
    if (cache_ok && hit && cache->exec) {
        STWO_CUDA_TRY(cudaGraphLaunch(cache->exec, st));
        count_launch(cache->launches);
        cache->replays++;
    } else if (cache_ok && hit && !cache->no_graph) {
        const uint64_t l0 = t_kernel_launches;
        // (the legacy default stream cannot be captured: the sequence then runs directly)
        const cudaError_t eb = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        const int rc_cap = eb == cudaSuccess ? launch_all(true) : (int)STWO_ERR_CUDA;
        cudaGraph_t graph = nullptr;
        const cudaError_t ec = eb == cudaSuccess ? cudaStreamEndCapture(st, &graph) : eb;
        cudaGraphExec_t exec = nullptr;
        cudaError_t ei = cudaSuccess;
        if (rc_cap == STWO_OK && ec == cudaSuccess) ei = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc_cap == STWO_OK && ec == cudaSuccess && ei == cudaSuccess) {
            cache->exec = exec;
            cache->launches = t_kernel_launches - l0;  // counted at capture, run now
            STWO_CUDA_TRY(cudaGraphLaunch(exec, st));
        } else {
            // The sequence did not capture: run it directly, now and for this shape.
            cudaGetLastError();
            clear_error();
            cache->no_graph = true;
            g_kernel_launches.fetch_sub(t_kernel_launches - l0, std::memory_order_relaxed);  // nothing ran
            t_kernel_launches = l0;
            PV_TRY(launch_all(false));
        }
    } else {
        PV_TRY(launch_all(false));
    }
    // ---- the jobs' records (channel state and sampled values), in one copy
    const size_t rec_bytes = sizeof(ProofState) + sizeof(qm31) * eap_n;
    std::vector<uint8_t> rec(rec_bytes * K);
    {
        void *rec_stage = nullptr;
        PV_TRY(host_stage(rec_bytes * K, &rec_stage));
        if (K == 1) STWO_CUDA_TRY(cudaMemcpyAsync(rec_stage, dstate, rec_bytes, cudaMemcpyDeviceToHost, st));
        else
            STWO_CUDA_TRY(
                cudaMemcpy2DAsync(rec_stage, rec_bytes, dstate, js, rec_bytes, K, cudaMemcpyDeviceToHost, st));
        PV_TRY(wait_stream(st));
        memcpy(rec.data(), rec_stage, rec_bytes * K);
    }
    // A job's status from the error bits its channel recorded.
    auto job_status = [&](const ProofState &ps) -> int {
        STWO_REQUIRE(!(ps.error & fs::ERR_DRAW), STWO_ERR_CUDA, "channel draw exceeded its retry bound");
        STWO_REQUIRE(!(ps.error & fs::ERR_CONSTRAINTS), STWO_ERR_INVALID_ARGUMENT,
                     "constraints not satisfied at the out-of-domain point");
        STWO_REQUIRE(!(ps.error & fs::ERR_LAST_LAYER), STWO_ERR_INVALID_ARGUMENT,
                     "FRI last layer exceeds its degree bound");
        STWO_REQUIRE(!(ps.error & fs::ERR_GRIND), STWO_ERR_INVALID_ARGUMENT,
                     "no proof-of-work nonce within 2^%u tries", j.pow_bits + 6);
        return STWO_OK;
    };

    // Per job: its queries and decommitments, planned as device reads that one gather
    // serves for all jobs.
    struct JobDecommit {
        int rc = STWO_OK;
        TreeDecommit d_trace, d_comp, d_fri0;
        std::vector<size_t> w_first;
        std::vector<std::vector<size_t>> w_inner;
        std::vector<TreeDecommit> d_inner;
    };
    std::vector<JobDecommit> jd(K);
    Gatherer g;
    for (uint32_t k = 0; k < K; k++) {
        JobLayout &Jk = jl[k];
        JobDecommit &o = jd[k];
        const ProofState &ps = *reinterpret_cast<const ProofState *>(rec.data() + rec_bytes * k);
        o.rc = job_status(ps);
        if (o.rc) {
            if (K == 1) return o.rc;
            continue;
        }
        // Queries::generate over the largest quotient domain (log D).
        std::vector<uint64_t> queries;
        {
            std::set<uint64_t> qs;
            const uint32_t mask = (uint32_t)((1ull << D) - 1);
            for (uint32_t i = 0; i < j.n_queries; i++) qs.insert(ps.query_words[i] & mask);
            queries.assign(qs.begin(), qs.end());
        }
        const std::map<uint32_t, std::vector<uint64_t>> tree_queries = {{D, queries},
                                                                        {L + B, fold_queries(queries, 1)}};
        o.d_trace = plan_decommit(Jk.t_trace, tree_queries, g);
        o.d_comp = plan_decommit(Jk.t_comp, tree_queries, g);
        // FRI first layer: per quotient column, its folding pairs; partners are witnesses.
        {
            std::map<uint32_t, std::vector<uint64_t>> pos;
            for (int grp = 0; grp < 2; grp++) {
                const uint32_t lg = grp == 0 ? D : L + B;
                const std::vector<uint32_t *> &col = grp == 0 ? Jk.qc : Jk.qt;
                std::vector<uint64_t> p, wv;
                fri_positions(fold_queries(queries, D - lg), p, wv);
                pos[lg] = p;
                for (uint64_t x : wv)
                    for (int c = 0; c < 4; c++) o.w_first.push_back(g.add(col[c], x));
            }
            o.d_fri0 = plan_decommit(Jk.t_fri0, pos, g);
        }
        o.w_inner.assign(n_layers, {});
        o.d_inner.assign(n_layers, {});
        {
            std::vector<uint64_t> lq = fold_queries(queries, 1);
            for (uint32_t li = 0; li < n_layers; li++) {
                std::vector<uint64_t> p, wv;
                fri_positions(lq, p, wv);
                for (uint64_t x : wv)
                    for (int c = 0; c < 4; c++) o.w_inner[li].push_back(g.add(Jk.lay[li][c], x));
                o.d_inner[li] = plan_decommit(Jk.t_lay[li], {{D - 1 - li, p}}, g);
                lq = fold_queries(lq, 1);
            }
        }
    }
    PV_TRY(g.run(ar, st));
    const std::vector<uint32_t> &vals = g.vals;

    // ---- serialisation
    uint64_t proof_bytes = 0;
    for (uint32_t k = 0; k < K; k++) {
        const JobDecommit &o = jd[k];
        if (job_rc) job_rc[k] = o.rc;
        if (o.rc) {
            proofs[k].clear();
            continue;
        }
        const ProofState &ps = *reinterpret_cast<const ProofState *>(rec.data() + rec_bytes * k);
        const qm31 *sampled = reinterpret_cast<const qm31 *>(rec.data() + rec_bytes * k + sizeof(ProofState));
        Writer w;
        w.u64(2);  // commitments
        w.bytes(ps.roots[0], 32);
        w.bytes(ps.roots[1], 32);
        w.u64(2);  // sampled_values
        w.u64(N);
        for (uint32_t c = 0; c < N; c++) {
            w.u64(1);
            w.q(sampled[c]);
        }
        w.u64(4);
        for (int c = 0; c < 4; c++) {
            w.u64(1);
            w.q(sampled[N + c]);
        }
        w.u64(2);  // decommitments
        write_decommitment(w, o.d_trace, vals);
        write_decommitment(w, o.d_comp, vals);
        w.u64(2);  // queried_values
        for (const TreeDecommit *d : {&o.d_trace, &o.d_comp}) {
            w.u64(d->queried.size());
            for (auto &col : d->queried) {
                w.u64(col.size());
                for (size_t gi : col) w.u32(vals[gi]);
            }
        }
        w.u64(ps.nonce);  // proof_of_work
        auto write_fri_layer = [&](const std::vector<size_t> &wit, const TreeDecommit &d, const uint32_t root[8]) {
            w.u64(wit.size() / 4);
            for (size_t gi : wit) w.u32(vals[gi]);
            write_decommitment(w, d, vals);
            w.bytes(root, 32);
        };
        write_fri_layer(o.w_first, o.d_fri0, ps.roots[2]);
        w.u64(n_layers);
        for (uint32_t li = 0; li < n_layers; li++) write_fri_layer(o.w_inner[li], o.d_inner[li], ps.roots[3 + li]);
        w.u64(1);  // last_layer_poly.coeffs
        w.q(ps.last_coeff);
        w.u32(0);  // last_layer_poly.log_size
        proofs[k] = std::move(w.b);
        proof_bytes += proofs[k].size();
    }
    const double t5 = now_ms();

    if (cacheable) {
        if (cache_ok && !hit) {
            cache->valid = true;
            memcpy(cache->key, key, sizeof(key));
            cache->tunables_gen = tgen;
            cache->tw = tw_in;
            cache->itw = itw_in;
            cache->tsz = tsz_in;
            cache->device = dev;
            cache->slab = ar.slab;
            cache->cap = ar.cap;
            ar.retain = true;
        } else if (!cache_ok && hit) {
            prove_cache_release(cache, st);  // the slab it holds was adopted: freed once, here
        }
    }
    if (stats) {
        float ms[4];
        for (int p = 0; p < 4; p++) STWO_CUDA_TRY(cudaEventElapsedTime(&ms[p], ev[p], ev[p + 1]));
        stats->trace_ms = ms[0];
        stats->composition_ms = ms[1];
        stats->oods_ms = ms[2];
        stats->fri_ms = ms[3];
        stats->total_ms = t5 - t0;
        stats->decommit_ms = std::max(0.0, stats->total_ms - (ms[0] + ms[1] + ms[2] + ms[3]));
        stats->device_bytes = ar.bytes;
        stats->kernel_launches = t_kernel_launches - launches0;
        stats->proof_bytes = proof_bytes;
    }
    return STWO_OK;
}

}  // namespace


// Shared with the batch server.
int wide_fib_prove(const stwo_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1, const uint32_t *tw,
                   const uint32_t *itw, uint64_t tree_size, std::vector<uint8_t> &proof, stwo_prove_stats *stats,
                   cudaStream_t st, ProveCache *cache) {
    STWO_REQUIRE(job && a0 && a1, STWO_ERR_INVALID_ARGUMENT, "null argument");
    Job j{job->log_n_rows, job->n_columns, job->log_blowup, job->n_queries, job->pow_bits};
    int rc = prove_jobs(j, 1, &a0, &a1, tw, itw, tree_size, &proof, nullptr, st, stats, cache);
    if (rc) cudaStreamSynchronize(st);  // the arena's frees are queued; leave the stream idle
    return rc;
}

// Several proofs of one shape in one launch sequence (the caller's twiddle tree);
// proofs[k] and job_rc[k] receive job k's bytes and status.
int wide_fib_prove_batch(const stwo_wide_fib_job *job, uint32_t n_jobs, const uint32_t *const *a0,
                         const uint32_t *const *a1, const uint32_t *tw, const uint32_t *itw, uint64_t tree_size,
                         std::vector<std::vector<uint8_t>> &proofs, int *job_rc, stwo_prove_stats *stats,
                         cudaStream_t st) {
    STWO_REQUIRE(job && a0 && a1 && job_rc && n_jobs >= 1, STWO_ERR_INVALID_ARGUMENT, "null argument");
    for (uint32_t k = 0; k < n_jobs; k++) STWO_REQUIRE(a0[k] && a1[k], STWO_ERR_INVALID_ARGUMENT, "null input");
    Job j{job->log_n_rows, job->n_columns, job->log_blowup, job->n_queries, job->pow_bits};
    proofs.assign(n_jobs, {});
    int rc = prove_jobs(j, n_jobs, a0, a1, tw, itw, tree_size, proofs.data(), job_rc, st, stats, nullptr);
    if (rc) {
        cudaStreamSynchronize(st);
        for (uint32_t k = 0; k < n_jobs; k++) job_rc[k] = rc;
    }
    return rc;
}

uint64_t wide_fib_job_device_bytes(const stwo_wide_fib_job *job, bool own_twiddles) {
    if (!job) return 0;
    Job j{job->log_n_rows, job->n_columns, job->log_blowup, job->n_queries, job->pow_bits};
    if (validate(j)) return 0;
    return job_device_bytes(j, own_twiddles);
}

}  // namespace stwo

using namespace stwo;

extern "C" {

uint64_t stwo_wide_fib_prove_device_bytes(const stwo_wide_fib_job *job, int with_own_twiddles) {
    return wide_fib_job_device_bytes(job, with_own_twiddles != 0);
}

int stwo_wide_fib_prove(const stwo_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1, const uint32_t *twiddles,
                        const uint32_t *itwiddles, uint64_t tree_size, uint8_t **proof_out, uint64_t *proof_len,
                        stwo_prove_stats *stats, void *stream) {
    STWO_REQUIRE(proof_out && proof_len, STWO_ERR_INVALID_ARGUMENT, "null proof output");
    *proof_out = nullptr;
    *proof_len = 0;
    std::vector<uint8_t> proof;
    int rc = wide_fib_prove(job, a0, a1, twiddles, itwiddles, tree_size, proof, stats, as_stream(stream));
    if (rc) return rc;
    *proof_out = static_cast<uint8_t *>(malloc(proof.size()));
    STWO_REQUIRE(*proof_out, STWO_ERR_OUT_OF_MEMORY, "proof buffer allocation failed");
    memcpy(*proof_out, proof.data(), proof.size());
    *proof_len = proof.size();
    return STWO_OK;
}

void stwo_free_proof(uint8_t *proof) { free(proof); }

int stwo_wide_fib_prove_batch(const stwo_wide_fib_job *job, uint32_t n_jobs, const uint32_t *const *a0,
                              const uint32_t *const *a1, const uint32_t *twiddles, const uint32_t *itwiddles,
                              uint64_t tree_size, uint8_t **proofs, uint64_t *proof_lens, int *job_status,
                              stwo_prove_stats *stats, void *stream) {
    STWO_REQUIRE(proofs && proof_lens && job_status && n_jobs >= 1 && n_jobs <= 256, STWO_ERR_INVALID_ARGUMENT,
                 "batch outputs");
    for (uint32_t k = 0; k < n_jobs; k++) {
        proofs[k] = nullptr;
        proof_lens[k] = 0;
    }
    std::vector<std::vector<uint8_t>> out;
    int rc = wide_fib_prove_batch(job, n_jobs, a0, a1, twiddles, itwiddles, tree_size, out, job_status, stats,
                                  as_stream(stream));
    if (rc) return rc;
    for (uint32_t k = 0; k < n_jobs; k++) {
        if (job_status[k] != STWO_OK) continue;
        proofs[k] = static_cast<uint8_t *>(malloc(out[k].size()));
        if (!proofs[k]) {
            for (uint32_t i = 0; i < k; i++) {
                free(proofs[i]);
                proofs[i] = nullptr;
            }
            return set_error(STWO_ERR_OUT_OF_MEMORY, "proof buffer allocation failed");
        }
        memcpy(proofs[k], out[k].data(), out[k].size());
        proof_lens[k] = out[k].size();
    }
    return STWO_OK;
}

struct stwo_prove_cache {
    ProveCache c;
};

stwo_prove_cache *stwo_prove_cache_create(void) { return new (std::nothrow) stwo_prove_cache(); }

int stwo_wide_fib_prove_cached(stwo_prove_cache *cache, const stwo_wide_fib_job *job, const uint32_t *a0,
                               const uint32_t *a1, const uint32_t *twiddles, const uint32_t *itwiddles,
                               uint64_t tree_size, uint8_t **proof_out, uint64_t *proof_len, stwo_prove_stats *stats,
                               void *stream) {
    STWO_REQUIRE(cache, STWO_ERR_INVALID_ARGUMENT, "null proof cache");
    STWO_REQUIRE(twiddles && itwiddles, STWO_ERR_INVALID_ARGUMENT, "a cached proof needs the caller's twiddle tree");
    STWO_REQUIRE(proof_out && proof_len, STWO_ERR_INVALID_ARGUMENT, "null proof output");
    *proof_out = nullptr;
    *proof_len = 0;
    std::vector<uint8_t> proof;
    int rc = wide_fib_prove(job, a0, a1, twiddles, itwiddles, tree_size, proof, stats, as_stream(stream), &cache->c);
    if (rc) return rc;
    *proof_out = static_cast<uint8_t *>(malloc(proof.size()));
    STWO_REQUIRE(*proof_out, STWO_ERR_OUT_OF_MEMORY, "proof buffer allocation failed");
    memcpy(*proof_out, proof.data(), proof.size());
    *proof_len = proof.size();
    return STWO_OK;
}

void stwo_prove_cache_stats(const stwo_prove_cache *cache, uint64_t *device_bytes, uint64_t *graph_replays) {
    if (device_bytes) *device_bytes = cache && cache->c.valid ? cache->c.cap : 0;
    if (graph_replays) *graph_replays = cache ? cache->c.replays : 0;
}

void stwo_prove_cache_destroy(stwo_prove_cache *cache, void *stream) {
    if (!cache) return;
    prove_cache_release(&cache->c, as_stream(stream));
    delete cache;
}

}  // extern "C"
