// Wide-Fibonacci STARK prover: stwo's prove() for the wide-Fibonacci AIR, driven on
// the host in C++ over this library's kernels.
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
// Everything that touches column data runs on the GPU; the channel, the query
// positions and the decommitted words live on the host. Each job runs on one stream
// and synchronises only where the channel needs a device result (tree roots, sampled
// values, the last FRI layer, the nonce, the gathered decommitment words), so jobs on
// other streams fill the device meanwhile.
//
// The proof bytes are the CommitmentSchemeProof fields in declaration order, little
// endian, vectors prefixed with a u64 length, hashes as 32 raw bytes, field elements as
// u32 words (a bincode-style layout):
//   commitments, sampled_values, decommitments, queried_values, proof_of_work,
//   fri_proof{first_layer, inner_layers, last_layer_poly{coeffs, log_size}}.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <vector>

#include "blake2s.cuh"
#include "blake2s_host.h"
#include "common.cuh"

namespace stwo {

int fft_columns(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st);
int merkle_layer_async(uint32_t log_size, const uint32_t *prev, const uint32_t *const *cols, uint32_t n_cols,
                       bool cols_on_device, uint32_t *out, cudaStream_t st);
int merkle_top_async(uint32_t prev_log, uint32_t *const *layers, cudaStream_t st);
int quotients_async(uint32_t half_init, uint32_t half_step, uint32_t log_size, const uint32_t *const *cols,
                    uint32_t n_cols, bool cols_on_device, stwo_qm31 rc_c, const stwo_spoint *pts, const uint32_t *bsz,
                    const uint32_t *cidx, const stwo_qm31 *vals, uint32_t n_batches, uint32_t *const *out4,
                    cudaStream_t st);
int fold_async(const uint32_t *const *src4, uint64_t n, stwo_qm31 alpha_c, const uint32_t *itw, uint64_t off,
               uint32_t *const *dst4, bool circle, cudaStream_t st);
int wide_fib_async(const uint32_t *const *trace, uint32_t n_cols, uint32_t log_size, const stwo_qm31 *powers_host,
                   const uint32_t *powers_dev, const uint32_t *den_inv, uint32_t *const *out4, cudaStream_t st);
int batch_inverse_m31_async(const uint32_t *src, uint32_t *dst, uint64_t n, cudaStream_t st);
size_t eval_at_points_scratch_bytes(const uint32_t *log_sizes, uint32_t n_polys);
int eval_at_points_async(const uint32_t *const *coeffs, const uint32_t *log_sizes, uint32_t n_polys,
                         const stwo_spoint *points, stwo_qm31 *results, void *scratch, size_t scratch_bytes,
                         bool tickets_zeroed, cudaStream_t st);

namespace {

constexpr uint32_t WF_MAX_TRACE_COLS = 1024;
constexpr uint32_t MAX_DOMAIN_LOG = 27;  // largest committed domain CanonicCoset(L+1+B)

// ------------------------------------------------------------------ device kernels

// Trace rows (write_trace_row, wide_fibonacci.rs:196-203): a_0 = a0[r], a_1 = a1[r],
// a_{j+2} = a_j^2 + a_{j+1}^2. Row r is position r of every column, the bit-reversed
// storage order of the trace evaluations.
struct TraceCols {
    uint32_t *c[WF_MAX_TRACE_COLS];
};

__global__ void __launch_bounds__(256) wide_fib_trace_kernel(const uint32_t *__restrict__ a0,
                                                             const uint32_t *__restrict__ a1,
                                                             const __grid_constant__ TraceCols t, uint32_t n_cols,
                                                             uint64_t rows) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t x = a0[r], y = a1[r];
        t.c[0][r] = x;
        t.c[1][r] = y;
        for (uint32_t j = 2; j < n_cols; j++) {
            uint32_t z = m31_add(m31_sqr(x), m31_sqr(y));
            t.c[j][r] = z;
            x = y;
            y = z;
        }
    }
}

// Vanishing polynomial of CanonicCoset(L).coset at every point of the circle domain
// CanonicCoset(E) in bit-reversed order (coset_vanishing as wide_fibonacci.rs:99-117
// calls it): p -> p - initial + step/2, then the x coordinate doubled L-1 times.
struct VanishingParams {
    cpoint gen_pows[31];  // GEN^(2^b)
    cpoint shift;         // -initial + step/2 of the vanishing coset
    uint32_t half_init, half_step, ext_log, doublings;
};

__global__ void __launch_bounds__(256) vanishing_kernel(uint32_t *__restrict__ out,
                                                        const __grid_constant__ VanishingParams p) {
    const uint64_t n = 1ull << p.ext_log, half = n >> 1;
    for (uint64_t pos = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; pos < n; pos += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = bit_reverse_bits((uint32_t)pos, p.ext_log);
        uint32_t idx = p.half_init + p.half_step * (uint32_t)(i < half ? i : i - half);
        if (i >= half) idx = 0x80000000u - (idx & 0x7fffffffu);  // the conjugate half
        cpoint r = {1, 0};
#pragma unroll 1
        for (int b = 0; b < 31; b++)
            if ((idx >> b) & 1u) r = point_mul(r, p.gen_pows[b]);
        r = point_mul(r, p.shift);
        uint32_t x = r.x;
        for (uint32_t d = 0; d < p.doublings; d++) {
            uint32_t s = m31_sqr(x);
            x = m31_sub(m31_add(s, s), 1);
        }
        out[pos] = x;
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

// Proof-of-work search (GrindOps::grind): nonce k is valid when the channel digest
// mixed with k (one BLAKE2s compression of the digest with message [lo(k), hi(k), 0...])
// has at least pow_bits trailing zero bits as a little-endian u128. Thread t tries the
// nonces base + t + k * (grid size), k < per_thread, and records the least valid one.
struct GrindParams {
    uint32_t h[8];
    uint32_t pow_bits;
};

__device__ __forceinline__ uint32_t ctz128(const uint32_t w[4]) {
    if (w[0]) return __ffs(w[0]) - 1;
    if (w[1]) return 32 + __ffs(w[1]) - 1;
    if (w[2]) return 64 + __ffs(w[2]) - 1;
    if (w[3]) return 96 + __ffs(w[3]) - 1;
    return 128;
}

__global__ void __launch_bounds__(256) grind_kernel(const GrindParams p, uint64_t base, uint32_t per_thread,
                                                    unsigned long long *__restrict__ best) {
    const uint32_t one = 1;
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint32_t k = 0; k < per_thread; k++) {
        const uint64_t nonce = base + t + k * stride;
        uint32_t h[8], m[16] = {0};
#pragma unroll
        for (int i = 0; i < 8; i++) h[i] = p.h[i];
        m[0] = (uint32_t)nonce;
        m[1] = (uint32_t)(nonce >> 32);
        blake::compress(h, m, one);
        if (ctz128(h) >= p.pow_bits) {
            atomicMin(best, (unsigned long long)nonce);
            return;
        }
    }
}

// ------------------------------------------------------------------ host plumbing

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Stream-ordered device allocations of one job, all released when the job ends.
struct Arena {
    cudaStream_t st;
    std::vector<void *> ptrs;
    uint64_t bytes = 0;
    explicit Arena(cudaStream_t s) : st(s) {}
    ~Arena() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
    template <typename T = uint32_t>
    T *alloc(size_t count) {
        void *p = nullptr;
        size_t b = std::max<size_t>(count * sizeof(T), 16);
        b = (b + 255) & ~size_t(255);
        if (pool_alloc(&p, b, st) != STWO_OK) return nullptr;
        ptrs.push_back(p);
        bytes += b;
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

inline qm31 to_q(stwo_qm31 v) { return {{v.a, v.b}, {v.c, v.d}}; }
inline stwo_qm31 from_q(qm31 v) { return {v.a.a, v.a.b, v.b.a, v.b.b}; }

// Half coset {initial index, step index} of CanonicCoset(log).circle_domain().
inline uint32_t half_coset_init(uint32_t log) { return 1u << (30 - log); }
inline uint32_t half_coset_step(uint32_t log) { return (uint32_t)((1ull << (32 - log)) & 0x7fffffffu); }

// Blake2sChannel (stwo core/channel/blake2s.rs): a 32-byte digest, the number of
// digest updates and the number of draws since the last update.
struct Channel {
    uint8_t digest[32] = {0};
    uint64_t n_challenges = 0, n_sent = 0;

    void update(const uint8_t d[32]) {
        memcpy(digest, d, 32);
        n_challenges++;
        n_sent = 0;
    }
    // Blake2sMerkleChannel::mix_root: digest = H(digest || root).
    void mix_root(const uint8_t root[32]) {
        uint8_t buf[64], out[32];
        memcpy(buf, digest, 32);
        memcpy(buf + 32, root, 32);
        host_blake2s::hash(buf, 64, out);
        update(out);
    }
    // digest = H(digest || felts as u32 LE words).
    void mix_felts(const std::vector<qm31> &f) {
        std::vector<uint8_t> buf(32 + 16 * f.size());
        memcpy(buf.data(), digest, 32);
        for (size_t i = 0; i < f.size(); i++) {
            uint32_t w[4] = {f[i].a.a, f[i].a.b, f[i].b.a, f[i].b.b};
            memcpy(buf.data() + 32 + 16 * i, w, 16);
        }
        uint8_t out[32];
        host_blake2s::hash(buf.data(), buf.size(), out);
        update(out);
    }
    // digest = compress(digest as chaining state, [lo, hi, 0, ...]) with zero counter and flags.
    void mix_nonce(uint64_t nonce) {
        uint32_t h[8], m[16] = {0};
        memcpy(h, digest, 32);
        m[0] = (uint32_t)nonce;
        m[1] = (uint32_t)(nonce >> 32);
        host_blake2s::compress(h, m, 0, 0);
        uint8_t out[32];
        memcpy(out, h, 32);
        update(out);
    }
    // H(digest || n_sent as u64 LE, zero-padded to 32 bytes).
    void draw_random_bytes(uint8_t out[32]) {
        uint8_t buf[64] = {0};
        memcpy(buf, digest, 32);
        memcpy(buf + 32, &n_sent, 8);
        n_sent++;
        host_blake2s::hash(buf, 64, out);
    }
    // Eight base field elements; redrawn until every u32 is below 2P.
    void draw_base_felts(uint32_t f[8]) {
        for (;;) {
            uint8_t b[32];
            draw_random_bytes(b);
            uint32_t u[8];
            memcpy(u, b, 32);
            bool ok = true;
            for (int i = 0; i < 8; i++) ok = ok && u[i] < 2 * P;
            if (!ok) continue;
            for (int i = 0; i < 8; i++) f[i] = u[i] >= P ? u[i] - P : u[i];
            return;
        }
    }
    qm31 draw_felt() {
        uint32_t f[8];
        draw_base_felts(f);
        return {{f[0], f[1]}, {f[2], f[3]}};
    }
};

// Merkle tree of columns of power-of-two sizes (MerkleProver::commit): the columns in
// decreasing size order (stable); layer l hashes the children (below the top) and the
// columns of size 2^l. All layers stay on the device for decommitment.
struct MerkleTree {
    std::vector<uint32_t *> layers;  // layers[l]: 2^l nodes of 8 words
    std::vector<std::pair<uint32_t, const uint32_t *>> cols;
    uint32_t max_log = 0;
    uint8_t root[32];
};

// Layers of at most 2^MERKLE_TOP_LOG nodes that hash children only are hashed by one
// single-CTA launch.
constexpr uint32_t MERKLE_TOP_LOG = 10;

int commit_tree(MerkleTree &t, std::vector<std::pair<uint32_t, const uint32_t *>> cols, Arena &ar,
                cudaStream_t st) {
    std::stable_sort(cols.begin(), cols.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    t.cols = cols;
    t.max_log = cols[0].first;
    const uint32_t min_col_log = cols.back().first;
    t.layers.assign(t.max_log + 1, nullptr);
    for (int l = (int)t.max_log; l >= 0; l--) {
        PV_ALLOC(layer, uint32_t, (size_t)8 << l);
        t.layers[l] = layer;
    }
    for (int l = (int)t.max_log; l >= 0; l--) {
        if ((uint32_t)l < min_col_log && (uint32_t)l <= MERKLE_TOP_LOG) {
            PV_TRY(merkle_top_async((uint32_t)l + 1, t.layers.data(), st));  // layers l .. 0
            break;
        }
        std::vector<const uint32_t *> lc;
        for (auto &c : cols)
            if (c.first == (uint32_t)l) lc.push_back(c.second);
        const uint32_t *prev = l < (int)t.max_log ? t.layers[l + 1] : nullptr;
        PV_TRY(merkle_layer_async((uint32_t)l, prev, lc.data(), (uint32_t)lc.size(), false, t.layers[l], st));
    }
    void *stage = nullptr;
    PV_TRY(host_stage(32, &stage));
    STWO_CUDA_TRY(cudaMemcpyAsync(stage, t.layers[0], 32, cudaMemcpyDeviceToHost, st));
    PV_TRY(wait_stream(st));
    memcpy(t.root, stage, 32);
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
    void bytes(const uint8_t *p, size_t n) { b.insert(b.end(), p, p + n); }
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

// LineEvaluation::interpolate of the last FRI layer (2^log values in bit-reversed order
// over the line domain Coset(init, step, log)); coefficients in natural order.
std::vector<qm31> interpolate_line(const std::vector<qm31> &evals, uint32_t init, uint32_t step, uint32_t log) {
    const size_t n = evals.size();
    std::vector<qm31> v(n);
    for (size_t i = 0; i < n; i++) v[bit_reverse_bits((uint32_t)i, log)] = evals[i];
    uint32_t di = init, ds = step;
    for (size_t size = n; size > 1; size >>= 1) {
        for (size_t c = 0; c < n; c += size)
            for (size_t i = 0; i < size / 2; i++) {
                const uint32_t x = index_to_point((uint32_t)((di + (uint64_t)ds * i) & 0x7fffffffu)).x;
                const uint32_t xi = m31_inv(x);
                qm31 a = v[c + i], b = v[c + i + size / 2];
                v[c + i] = qm31_add(a, b);
                v[c + i + size / 2] = qm31_scale(qm31_sub(a, b), xi);
            }
        di = (di * 2) & 0x7fffffffu;
        ds = (ds * 2) & 0x7fffffffu;
    }
    const uint32_t ninv = m31_inv((uint32_t)n);
    std::vector<qm31> coeffs(n);  // bit-reversed (LinePoly storage) -> natural order
    for (size_t i = 0; i < n; i++) coeffs[bit_reverse_bits((uint32_t)i, log)] = qm31_scale(v[i], ninv);
    return coeffs;
}

// Circle point over QM31 and its group operation with a base-field point.
struct qpoint {
    qm31 x, y;
};
inline qpoint qpoint_mul_base(qpoint p, cpoint s) {
    return {qm31_sub(qm31_scale(p.x, s.x), qm31_scale(p.y, s.y)), qm31_add(qm31_scale(p.x, s.y), qm31_scale(p.y, s.x))};
}

// -initial + step/2 of CanonicCoset(log).coset (initial index 2^(30-log), step 2^(31-log)).
cpoint vanishing_shift(uint32_t log) {
    cpoint init = index_to_point(1u << (30 - log));
    cpoint half_step = index_to_point(1u << (30 - log));
    return point_mul(point_conj(init), half_step);
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
    STWO_REQUIRE(j.n_queries >= 1 && j.n_queries <= 1024, STWO_ERR_UNSUPPORTED_SIZE, "%u queries unsupported",
                 j.n_queries);
    STWO_REQUIRE(j.pow_bits <= 40, STWO_ERR_UNSUPPORTED_SIZE, "pow_bits %u unsupported (0..40)", j.pow_bits);
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
    b += 2 * r(4 * ne) + 4 * r(4 * ne) + 4 * r(4 * neb);  // denominators, composition, its evaluations
    b += r(16 * (j.N - 2));                               // coefficient powers
    b += r(1 << 20);                                      // eval_at_point scratch and results (bound)
    b += 4 * r(4 * neb) + 4 * r(4 * nb);                  // quotients
    b += tree(j.L + 1 + j.B);                             // FRI first layer tree
    for (uint32_t l = j.B; l <= j.L + j.B; l++) b += 4 * r(4ull << l) + tree(l);  // FRI layers
    b += r(64);                                           // nonce
    const uint64_t words = (uint64_t)j.n_queries * ((j.L + 2 + j.B) * 8 * 3 * 8 + 2 * (j.N + 16));
    b += r(words * sizeof(GatherReq)) + r(words * 4);     // decommitment gather
    return b;
}

int prove_impl(const Job &j, const uint32_t *a0_in, const uint32_t *a1_in, const uint32_t *tw_in,
               const uint32_t *itw_in, uint64_t tsz_in, std::vector<uint8_t> &proof, cudaStream_t st,
               stwo_prove_stats *stats) {
    PV_TRY(validate(j));
    const uint32_t L = j.L, N = j.N, B = j.B, E = L + 1;
    const uint64_t rows = 1ull << L;
    const double t0 = now_ms();
    const uint64_t launches0 = t_kernel_launches;
    Arena ar(st);
    Channel ch;

    // Twiddles: the caller's tree, or one for CanonicCoset(L + 1 + B).half_coset
    // (wide_fibonacci.rs:216-220). Any canonic tree at least that large serves.
    const uint32_t *tw = tw_in, *itw = itw_in;
    uint64_t tsz = tsz_in;
    if (tw_in || itw_in) {
        STWO_REQUIRE(tw_in && itw_in && is_pow2(tsz_in) && tsz_in >= (1ull << (L + B)), STWO_ERR_INVALID_ARGUMENT,
                     "twiddle tree of %llu entries does not cover domain log size %u", (unsigned long long)tsz_in,
                     L + 1 + B);
    } else {
        const uint32_t D = L + 1 + B;
        tsz = 1ull << (L + B);
        PV_ALLOC(t, uint32_t, tsz);
        PV_ALLOC(it, uint32_t, tsz);
        PV_TRY(stwo_precompute_twiddles(half_coset_init(D), half_coset_step(D), L + B, t, it, st));
        tw = t;
        itw = it;
    }

    // ---- 1. trace: generation, interpolation, evaluation on CanonicCoset(L + B), tree
    PV_ALLOC(a0, uint32_t, rows);
    PV_ALLOC(a1, uint32_t, rows);
    STWO_CUDA_TRY(cudaMemcpyAsync(a0, a0_in, rows * 4, cudaMemcpyDefault, st));
    STWO_CUDA_TRY(cudaMemcpyAsync(a1, a1_in, rows * 4, cudaMemcpyDefault, st));
    std::vector<uint32_t *> tpoly(N), tev(N);
    auto tc = std::make_unique<TraceCols>();
    for (uint32_t c = 0; c < N; c++) {
        PV_ALLOC(p, uint32_t, rows);
        PV_ALLOC(e, uint32_t, rows << B);
        tpoly[c] = p;
        tev[c] = e;
        tc->c[c] = p;
    }
    {
        const uint64_t blocks = std::min<uint64_t>((rows + 255) / 256, (uint64_t)device_sm_count() * 8);
        wide_fib_trace_kernel<<<(unsigned)blocks, 256, 0, st>>>(a0, a1, *tc, N, rows);
        STWO_LAUNCH_CHECK("wide_fib_trace_kernel");
    }
    // The trace columns are interpolated in place: they become the coefficient columns.
    PV_TRY(fft_columns(tpoly.data(), tpoly.data(), N, L, L, itw, tsz, true, st));
    {
        std::vector<const uint32_t *> src(tpoly.begin(), tpoly.end());
        PV_TRY(fft_columns(src.data(), tev.data(), N, L + B, L, tw, tsz, false, st));
    }
    MerkleTree t_trace;
    {
        std::vector<std::pair<uint32_t, const uint32_t *>> cols;
        for (uint32_t c = 0; c < N; c++) cols.push_back({L + B, tev[c]});
        PV_TRY(commit_tree(t_trace, cols, ar, st));
    }
    ch.mix_root(t_trace.root);
    const double t1 = now_ms();

    // ---- 2. composition polynomial on CanonicCoset(L + 1), committed on CanonicCoset(L + 1 + B)
    const qm31 rc = ch.draw_felt();
    std::vector<const uint32_t *> text(N);
    if (B == 1) {
        for (uint32_t c = 0; c < N; c++) text[c] = tev[c];  // already on CanonicCoset(L + 1)
    } else {
        std::vector<uint32_t *> dst(N);
        for (uint32_t c = 0; c < N; c++) {
            PV_ALLOC(e, uint32_t, 1ull << E);
            dst[c] = e;
            text[c] = e;
        }
        std::vector<const uint32_t *> src(tpoly.begin(), tpoly.end());
        PV_TRY(fft_columns(src.data(), dst.data(), N, E, L, tw, tsz, false, st));
    }
    PV_ALLOC(den, uint32_t, 1ull << E);
    PV_ALLOC(den_inv, uint32_t, 1ull << E);
    {
        VanishingParams vp{};
        cpoint g = {CIRCLE_GEN_X, CIRCLE_GEN_Y};
        for (int b = 0; b < 31; b++) {
            vp.gen_pows[b] = g;
            g = point_mul(g, g);
        }
        vp.shift = vanishing_shift(L);
        vp.half_init = half_coset_init(E);
        vp.half_step = half_coset_step(E);
        vp.ext_log = E;
        vp.doublings = L - 1;
        const uint64_t blocks = std::min<uint64_t>(((1ull << E) + 255) / 256, (uint64_t)device_sm_count() * 8);
        vanishing_kernel<<<(unsigned)blocks, 256, 0, st>>>(den, vp);
        STWO_LAUNCH_CHECK("vanishing_kernel");
    }
    PV_TRY(batch_inverse_m31_async(den, den_inv, 1ull << E, st));
    // DomainEvaluationAccumulator: powers [1, r, ..., r^(N-3)]; constraint i takes r^(N-3-i).
    std::vector<stwo_qm31> powers(N - 2);
    {
        qm31 p = qm31_one();
        for (uint32_t k = 0; k + 2 < N; k++) {
            powers[k] = from_q(p);
            p = qm31_mul(p, rc);
        }
    }
    PV_ALLOC(powers_dev, stwo_qm31, N - 2);
    {
        // staged through pinned memory; the stage's next reuse is after a wait on this stream
        void *stage = nullptr;
        PV_TRY(host_stage(sizeof(stwo_qm31) * (N - 2), &stage));
        memcpy(stage, powers.data(), sizeof(stwo_qm31) * (N - 2));
        STWO_CUDA_TRY(cudaMemcpyAsync(powers_dev, stage, sizeof(stwo_qm31) * (N - 2), cudaMemcpyHostToDevice, st));
    }
    std::vector<uint32_t *> comp(4), cev(4);
    for (int k = 0; k < 4; k++) {
        PV_ALLOC(c, uint32_t, 1ull << E);
        PV_ALLOC(e, uint32_t, 1ull << (E + B));
        comp[k] = c;
        cev[k] = e;
    }
    PV_TRY(wide_fib_async(text.data(), N, E, nullptr, reinterpret_cast<const uint32_t *>(powers_dev), den_inv,
                          comp.data(), st));
    PV_TRY(fft_columns(comp.data(), comp.data(), 4, E, E, itw, tsz, true, st));  // in place -> coefficients
    {
        std::vector<const uint32_t *> src(comp.begin(), comp.end());
        PV_TRY(fft_columns(src.data(), cev.data(), 4, E + B, E, tw, tsz, false, st));
    }
    MerkleTree t_comp;
    {
        std::vector<std::pair<uint32_t, const uint32_t *>> cols;
        for (int k = 0; k < 4; k++) cols.push_back({E + B, cev[k]});
        PV_TRY(commit_tree(t_comp, cols, ar, st));
    }
    ch.mix_root(t_comp.root);
    const double t2 = now_ms();

    // ---- 3. out-of-domain sampling (CirclePoint::get_random_point)
    qpoint oods;
    {
        const qm31 t = ch.draw_felt(), t2q = qm31_mul(t, t);
        const qm31 inv = qm31_inv(qm31_add(t2q, qm31_one()));
        oods = {qm31_mul(qm31_sub(qm31_one(), t2q), inv), qm31_mul(qm31_add(t, t), inv)};
    }
    std::vector<qm31> sampled(N + 4);
    {
        std::vector<const uint32_t *> polys;
        std::vector<uint32_t> logs;
        for (uint32_t c = 0; c < N; c++) {
            polys.push_back(tpoly[c]);
            logs.push_back(L);
        }
        for (int k = 0; k < 4; k++) {
            polys.push_back(comp[k]);
            logs.push_back(E);
        }
        std::vector<stwo_spoint> pts(polys.size(), stwo_spoint{from_q(oods.x), from_q(oods.y)});
        const size_t sb = eval_at_points_scratch_bytes(logs.data(), (uint32_t)polys.size());
        PV_ALLOC(scratch, uint8_t, sb);
        PV_ALLOC(res, stwo_qm31, polys.size());
        PV_TRY(eval_at_points_async(polys.data(), logs.data(), (uint32_t)polys.size(), pts.data(), res, scratch, sb,
                                    false, st));
        void *stage = nullptr;
        PV_TRY(host_stage(polys.size() * sizeof(stwo_qm31), &stage));
        STWO_CUDA_TRY(cudaMemcpyAsync(stage, res, polys.size() * sizeof(stwo_qm31), cudaMemcpyDeviceToHost, st));
        PV_TRY(wait_stream(st));
        const stwo_qm31 *hv = static_cast<const stwo_qm31 *>(stage);
        for (size_t i = 0; i < polys.size(); i++) sampled[i] = to_q(hv[i]);
    }
    ch.mix_felts(sampled);
    {
        // The composition's sampled value (from_partial_evals over the basis 1, i, u, iu)
        // must equal the constraints evaluated on the sampled trace values.
        const qm31 basis[4] = {{{1, 0}, {0, 0}}, {{0, 1}, {0, 0}}, {{0, 0}, {1, 0}}, {{0, 0}, {0, 1}}};
        qm31 comp_val = qm31_zero();
        for (int k = 0; k < 4; k++) comp_val = qm31_add(comp_val, qm31_mul(sampled[N + k], basis[k]));
        qm31 x = qpoint_mul_base(oods, vanishing_shift(L)).x;
        for (uint32_t d = 0; d + 1 < L; d++) {
            qm31 s = qm31_mul(x, x);
            x = qm31_sub(qm31_add(s, s), qm31_one());
        }
        qm31 acc = qm31_zero();
        for (uint32_t i = 0; i + 2 < N; i++) {
            qm31 cons = qm31_sub(qm31_add(qm31_mul(sampled[i], sampled[i]), qm31_mul(sampled[i + 1], sampled[i + 1])),
                                 sampled[i + 2]);
            acc = qm31_add(qm31_mul(acc, rc), cons);
        }
        acc = qm31_mul(acc, qm31_inv(x));
        STWO_REQUIRE(qm31_eq(acc, comp_val), STWO_ERR_INVALID_ARGUMENT,
                     "constraints not satisfied at the out-of-domain point");
    }
    const double t3 = now_ms();

    // ---- 4. DEEP quotients (largest columns first) and the FRI commitment
    const qm31 qrc = ch.draw_felt();
    std::vector<uint32_t *> qc(4), qt(4);
    for (int k = 0; k < 4; k++) {
        PV_ALLOC(a, uint32_t, 1ull << (E + B));
        PV_ALLOC(b, uint32_t, 1ull << (L + B));
        qc[k] = a;
        qt[k] = b;
    }
    {
        const stwo_spoint sp = {from_q(oods.x), from_q(oods.y)};
        std::vector<uint32_t> idx4 = {0, 1, 2, 3}, sz4 = {4};
        std::vector<stwo_qm31> v4;
        for (int k = 0; k < 4; k++) v4.push_back(from_q(sampled[N + k]));
        std::vector<const uint32_t *> cc(cev.begin(), cev.end());
        PV_TRY(quotients_async(half_coset_init(E + B), half_coset_step(E + B), E + B, cc.data(), 4, false, from_q(qrc),
                               &sp, sz4.data(), idx4.data(), v4.data(), 1, qc.data(), st));
        std::vector<uint32_t> idxn(N), szn = {N};
        std::vector<stwo_qm31> vn(N);
        for (uint32_t c = 0; c < N; c++) {
            idxn[c] = c;
            vn[c] = from_q(sampled[c]);
        }
        std::vector<const uint32_t *> tcols(tev.begin(), tev.end());
        PV_TRY(quotients_async(half_coset_init(L + B), half_coset_step(L + B), L + B, tcols.data(), N, false,
                               from_q(qrc), &sp, szn.data(), idxn.data(), vn.data(), 1, qt.data(), st));
    }
    MerkleTree t_fri0;
    {
        std::vector<std::pair<uint32_t, const uint32_t *>> cols;
        for (int k = 0; k < 4; k++) cols.push_back({E + B, qc[k]});
        for (int k = 0; k < 4; k++) cols.push_back({L + B, qt[k]});
        PV_TRY(commit_tree(t_fri0, cols, ar, st));
    }
    ch.mix_root(t_fri0.root);
    struct Layer {
        uint32_t log;
        std::vector<uint32_t *> v;
        MerkleTree tree;
    };
    std::vector<Layer> layers;
    uint32_t cur_log = E + B - 1;  // LineDomain(Coset::half_odds(E + B - 1))
    std::vector<uint32_t *> cur(4);
    for (int k = 0; k < 4; k++) {
        PV_ALLOC(c, uint32_t, 1ull << cur_log);
        cur[k] = c;
        STWO_CUDA_TRY(cudaMemsetAsync(c, 0, 4ull << cur_log, st));
    }
    qm31 alpha = ch.draw_felt();
    {
        std::vector<const uint32_t *> s(qc.begin(), qc.end());
        PV_TRY(fold_async(s.data(), 1ull << (E + B), from_q(alpha), itw, tsz - (1ull << cur_log), cur.data(), true, st));
    }
    bool trace_folded = false;
    while (cur_log > B) {  // last layer domain: 2^(log_last_layer_degree_bound + log_blowup) = 2^B
        if (!trace_folded && cur_log == L + B - 1) {
            // The trace quotient folds into this layer with the previous layer's alpha.
            std::vector<const uint32_t *> s(qt.begin(), qt.end());
            PV_TRY(fold_async(s.data(), 1ull << (L + B), from_q(alpha), itw, tsz - (1ull << cur_log), cur.data(), true,
                              st));
            trace_folded = true;
        }
        Layer lay;
        lay.log = cur_log;
        lay.v = cur;
        std::vector<std::pair<uint32_t, const uint32_t *>> cols;
        for (int k = 0; k < 4; k++) cols.push_back({cur_log, cur[k]});
        PV_TRY(commit_tree(lay.tree, cols, ar, st));
        ch.mix_root(lay.tree.root);
        alpha = ch.draw_felt();
        std::vector<uint32_t *> nxt(4);
        for (int k = 0; k < 4; k++) {
            PV_ALLOC(c, uint32_t, 1ull << (cur_log - 1));
            nxt[k] = c;
        }
        std::vector<const uint32_t *> s(cur.begin(), cur.end());
        PV_TRY(fold_async(s.data(), 1ull << cur_log, from_q(alpha), itw, tsz - (1ull << cur_log), nxt.data(), false, st));
        layers.push_back(std::move(lay));
        cur = nxt;
        cur_log--;
    }
    STWO_REQUIRE(trace_folded, STWO_ERR_UNSUPPORTED_SIZE, "trace quotient not folded (trace too small)");
    // Last layer: 2^B evaluations over Coset(2^(29-B), 2^(31-B)) -> line polynomial of degree bound 1.
    qm31 last_coeff;
    {
        const size_t n = 1ull << B;
        void *stage = nullptr;
        PV_TRY(host_stage(16 * n, &stage));
        uint32_t *hv = static_cast<uint32_t *>(stage);
        for (int k = 0; k < 4; k++)
            STWO_CUDA_TRY(cudaMemcpyAsync(hv + k * n, cur[k], 4 * n, cudaMemcpyDeviceToHost, st));
        PV_TRY(wait_stream(st));
        std::vector<qm31> ev(n);
        for (size_t i = 0; i < n; i++) ev[i] = {{hv[i], hv[n + i]}, {hv[2 * n + i], hv[3 * n + i]}};
        std::vector<qm31> coeffs = interpolate_line(ev, 1u << (29 - B), 1u << (31 - B), B);
        for (size_t i = 1; i < n; i++)
            STWO_REQUIRE(qm31_eq(coeffs[i], qm31_zero()), STWO_ERR_INVALID_ARGUMENT,
                         "FRI last layer exceeds its degree bound");
        last_coeff = coeffs[0];
        ch.mix_felts({last_coeff});
    }
    const double t4 = now_ms();

    // ---- 5. proof of work, queries, decommitments
    uint64_t nonce = 0;
    {
        PV_ALLOC(best, unsigned long long, 1);
        GrindParams gp{};
        memcpy(gp.h, ch.digest, 32);
        gp.pow_bits = j.pow_bits;
        const uint32_t blocks = (uint32_t)device_sm_count() * 4, threads = 256, per_thread = 16;
        const uint64_t chunk = (uint64_t)blocks * threads * per_thread;
        unsigned long long found = ~0ull;
        // Expected work 2^pow_bits tries; the search gives up after 2^(pow_bits + 8).
        const uint64_t limit = std::max<uint64_t>(1ull << (j.pow_bits + 8), chunk);
        for (uint64_t base = 0; found == ~0ull && base < limit; base += chunk) {
            STWO_CUDA_TRY(cudaMemsetAsync(best, 0xff, 8, st));
            grind_kernel<<<blocks, threads, 0, st>>>(gp, base, per_thread, best);
            STWO_LAUNCH_CHECK("grind_kernel");
            void *stage = nullptr;
            PV_TRY(host_stage(8, &stage));
            STWO_CUDA_TRY(cudaMemcpyAsync(stage, best, 8, cudaMemcpyDeviceToHost, st));
            PV_TRY(wait_stream(st));
            memcpy(&found, stage, 8);
        }
        STWO_REQUIRE(found != ~0ull, STWO_ERR_INVALID_ARGUMENT, "no proof-of-work nonce found");
        nonce = found;
    }
    ch.mix_nonce(nonce);

    // Queries::generate over the largest quotient domain (log E + B).
    std::vector<uint64_t> queries;
    {
        std::set<uint64_t> qs;
        uint32_t cnt = 0;
        const uint32_t mask = (uint32_t)((1ull << (E + B)) - 1);
        while (cnt < j.n_queries) {
            uint8_t b[32];
            ch.draw_random_bytes(b);
            for (int i = 0; i < 8 && cnt < j.n_queries; i++, cnt++) {
                uint32_t u;
                memcpy(&u, b + 4 * i, 4);
                qs.insert(u & mask);
            }
        }
        queries.assign(qs.begin(), qs.end());
    }
    const std::map<uint32_t, std::vector<uint64_t>> tree_queries = {{E + B, queries},
                                                                     {L + B, fold_queries(queries, 1)}};

    Gatherer g;
    TreeDecommit d_trace = plan_decommit(t_trace, tree_queries, g);
    TreeDecommit d_comp = plan_decommit(t_comp, tree_queries, g);
    // FRI first layer: per quotient column, its folding pairs; partners are witnesses.
    std::vector<size_t> w_first;
    TreeDecommit d_fri0;
    {
        std::map<uint32_t, std::vector<uint64_t>> pos;
        for (int grp = 0; grp < 2; grp++) {
            const uint32_t lg = grp == 0 ? E + B : L + B;
            const std::vector<uint32_t *> &col = grp == 0 ? qc : qt;
            std::vector<uint64_t> p, wv;
            fri_positions(fold_queries(queries, E + B - lg), p, wv);
            pos[lg] = p;
            for (uint64_t x : wv)
                for (int k = 0; k < 4; k++) w_first.push_back(g.add(col[k], x));
        }
        d_fri0 = plan_decommit(t_fri0, pos, g);
    }
    std::vector<std::vector<size_t>> w_inner(layers.size());
    std::vector<TreeDecommit> d_inner(layers.size());
    {
        std::vector<uint64_t> lq = fold_queries(queries, 1);
        for (size_t li = 0; li < layers.size(); li++) {
            std::vector<uint64_t> p, wv;
            fri_positions(lq, p, wv);
            for (uint64_t x : wv)
                for (int k = 0; k < 4; k++) w_inner[li].push_back(g.add(layers[li].v[k], x));
            d_inner[li] = plan_decommit(layers[li].tree, {{layers[li].log, p}}, g);
            lq = fold_queries(lq, 1);
        }
    }
    PV_TRY(g.run(ar, st));
    const std::vector<uint32_t> &vals = g.vals;

    // ---- serialisation
    Writer w;
    w.u64(2);  // commitments
    w.bytes(t_trace.root, 32);
    w.bytes(t_comp.root, 32);
    w.u64(2);  // sampled_values
    w.u64(N);
    for (uint32_t c = 0; c < N; c++) {
        w.u64(1);
        w.q(sampled[c]);
    }
    w.u64(4);
    for (int k = 0; k < 4; k++) {
        w.u64(1);
        w.q(sampled[N + k]);
    }
    w.u64(2);  // decommitments
    write_decommitment(w, d_trace, vals);
    write_decommitment(w, d_comp, vals);
    w.u64(2);  // queried_values
    for (const TreeDecommit *d : {&d_trace, &d_comp}) {
        w.u64(d->queried.size());
        for (auto &col : d->queried) {
            w.u64(col.size());
            for (size_t gi : col) w.u32(vals[gi]);
        }
    }
    w.u64(nonce);  // proof_of_work
    auto write_fri_layer = [&](const std::vector<size_t> &wit, const TreeDecommit &d, const uint8_t root[32]) {
        w.u64(wit.size() / 4);
        for (size_t gi : wit) w.u32(vals[gi]);
        write_decommitment(w, d, vals);
        w.bytes(root, 32);
    };
    write_fri_layer(w_first, d_fri0, t_fri0.root);
    w.u64(layers.size());
    for (size_t li = 0; li < layers.size(); li++) write_fri_layer(w_inner[li], d_inner[li], layers[li].tree.root);
    w.u64(1);  // last_layer_poly.coeffs
    w.q(last_coeff);
    w.u32(0);  // last_layer_poly.log_size
    proof = std::move(w.b);
    const double t5 = now_ms();

    if (stats) {
        stats->trace_ms = t1 - t0;
        stats->composition_ms = t2 - t1;
        stats->oods_ms = t3 - t2;
        stats->fri_ms = t4 - t3;
        stats->decommit_ms = t5 - t4;
        stats->total_ms = t5 - t0;
        stats->device_bytes = ar.bytes;
        stats->kernel_launches = t_kernel_launches - launches0;
        stats->proof_bytes = proof.size();
    }
    return STWO_OK;
}

}  // namespace

// Shared with the batch server.
int wide_fib_prove(const stwo_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1, const uint32_t *tw,
                   const uint32_t *itw, uint64_t tree_size, std::vector<uint8_t> &proof, stwo_prove_stats *stats,
                   cudaStream_t st) {
    STWO_REQUIRE(job && a0 && a1, STWO_ERR_INVALID_ARGUMENT, "null argument");
    Job j{job->log_n_rows, job->n_columns, job->log_blowup, job->n_queries, job->pow_bits};
    int rc = prove_impl(j, a0, a1, tw, itw, tree_size, proof, st, stats);
    if (rc) cudaStreamSynchronize(st);  // the arena's frees are queued; leave the stream idle
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

}  // extern "C"
