// MerkleOps<Blake2sMerkleHasher>::commit_on_layer.
//
// Node hash (cuda/src/blake2s.cu:97-151, stwo_gpu_backend/src/blake2s.rs:19-97):
// the chaining state starts at zero; if the layer has children, one compression
// of (left hash || right hash); then the layer's columns, 16 words per
// compression, the last chunk zero-padded. The compression is BLAKE2s's with the
// IV in v[8..15] and zero counter and flags.
//
// One thread per node; the 16-word message and the 16-word working state stay in
// registers (the round permutation is resolved at compile time). Column reads are
// coalesced across the threads of a warp (consecutive nodes, consecutive words).
#include <algorithm>
#include <vector>

#include "blake2s.cuh"
#include "common.cuh"

namespace stwo {
namespace {

using blake::compress;

constexpr int MERKLE_MAX_COLS = 2048;

// Column pointers by value, in a parameter block sized to the call (a launch copies
// its whole parameter block, so small calls use a small one).
template <int CAP>
struct MerkleCols {
    const uint32_t *c[CAP];
};

// Hashes node i of a layer: children (if prev) then n_cols column words, 16 per
// compression, the last chunk zero-padded.
template <class ColAt>
__device__ __forceinline__ void merkle_node(uint32_t i, const uint4 *prev, ColAt col_at, uint32_t n_cols, uint4 *out,
                                            uint32_t one) {
    uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t m[16];
    if (prev) {
        const uint4 *p = prev + 4 * (size_t)i;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint4 v = p[q];
            m[4 * q] = v.x; m[4 * q + 1] = v.y; m[4 * q + 2] = v.z; m[4 * q + 3] = v.w;
        }
        compress(h, m, one);
    }
    uint32_t c0 = 0;
    for (; c0 + 16 <= n_cols; c0 += 16) {  // full chunks: no per-word bound checks
#pragma unroll
        for (int j = 0; j < 16; j++) m[j] = __ldg(col_at(c0 + j) + i);
        compress(h, m, one);
    }
    if (c0 < n_cols) {  // the zero-padded last chunk
#pragma unroll
        for (int j = 0; j < 16; j++) {
            uint32_t cj = c0 + j;
            m[j] = cj < n_cols ? __ldg(col_at(cj) + i) : 0u;
        }
        compress(h, m, one);
    }
    out[2 * (size_t)i] = make_uint4(h[0], h[1], h[2], h[3]);
    out[2 * (size_t)i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// One layer, one thread per node. COLS_ON_DEVICE: column pointers come from a device
// array (reference ABI); otherwise from the parameter block.
template <bool COLS_ON_DEVICE, int CAP>
__global__ void __launch_bounds__(256) merkle_layer_kernel(uint32_t log_size, const uint4 *__restrict__ prev,
                                                           const __grid_constant__ MerkleCols<CAP> cols,
                                                           const uint32_t *const *__restrict__ dev_cols,
                                                           uint32_t n_cols, uint4 *__restrict__ out, uint32_t one) {
    // 32-bit node indices: at most 2^31 nodes, and i + the grid's stride stays below 2^32
    const uint32_t n = 1u << log_size;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (COLS_ON_DEVICE)
            merkle_node(i, prev, [&](uint32_t c) { return dev_cols[c]; }, n_cols, out, one);
        else
            merkle_node(i, prev, [&](uint32_t c) { return cols.c[c]; }, n_cols, out, one);
    }
}

// A whole tree in one launch. The layers are cut into bands of at most
// log2(THREADS) + 1 + spread layers; a band is a grid of units, and unit u of a band
// hashes the (THREADS << spread) >> j nodes of its level j that start at
// u * ((THREADS << spread) >> j): the parents of the nodes it hashed one level down,
// so a barrier is the only synchronisation inside a unit. A unit of every band but the
// last ends in a single node. The band above needs 2 * (THREADS << spread') such
// nodes per unit: the CTA that finishes the last of them (a per-unit ticket, counted
// with an atomic add after a device-scope fence) hashes that unit next, so no CTA ever
// waits and the tree's upper layers need no launch of their own. Tickets are reset by
// the CTA that takes them: the array is zero again when the tree is done.
//
// Levels of at most THREADS nodes keep each node's hash in shared memory as well, and
// their parents read it from there instead of from L2: these levels are short of
// warps and bound by the latency of one compression plus its loads.
//
// With spread s a thread hashes 2^s bottom-level nodes, so a unit stays dense for s + 1
// levels before its upper levels thin out.
constexpr int MERKLE_MAX_BANDS = 6;

struct TreeBand {
    uint32_t top;          // the band's lowest level (largest layer)
    uint32_t levels;       // layers top .. top - levels + 1
    uint32_t spread;       // a unit's first level has THREADS << spread nodes (fewer for a single unit)
    uint32_t has_prev;     // the first level hashes children
    uint32_t units;
    uint32_t fan;          // units of the band below per unit of this one (every band but the first)
    uint32_t ticket_base;  // this band's tickets, one per unit (every band but the first)
};

struct TreeParams {
    uint4 *layer[31];                     // layer[l]: 2^l nodes
    const uint32_t *const *cols[31];      // device column table per layer
    uint32_t n_cols[31];
    TreeBand band[MERKLE_MAX_BANDS];
    uint32_t n_bands;
    uint32_t *tickets;
    size_t js;  // jobs' memory stride: blockIdx.y's tree is job 0's moved by blockIdx.y * js
};


template <int THREADS>
__device__ __forceinline__ void merkle_unit(const TreeParams &p, const TreeBand &bd, uint32_t u,
                                            uint4 (*thin)[THREADS][2], uint32_t one) {
    const uint32_t job = blockIdx.y;
    // node indices fit 32 bits: a layer has at most 2^30 nodes
    const uint32_t per0 = (uint32_t)THREADS << bd.spread;
    for (uint32_t j = 0; j < bd.levels; j++) {
        const uint32_t l = bd.top - j;
        const uint32_t per = per0 >> j, first = u * per, n_l = 1u << l;
        const uint32_t *const *ct = job_ptr(p.cols[l], p.js, job);
        const uint32_t nc = p.n_cols[l];
        // children: none (a leaf layer), this CTA's shared memory (when the level below
        // had at most THREADS nodes), or global memory: other CTAs' nodes on a band's
        // first level (read from L2, since this SM's L1 never held them), else this CTA's
        // own nodes of a dense level below
        const bool kids = j > 0 || bd.has_prev;
        const bool kids_shared = j > 0 && (per0 >> (j - 1)) <= (uint32_t)THREADS;
        const bool to_shared = per <= (uint32_t)THREADS && j + 1 < bd.levels;
        const uint4 *below = kids ? job_ptr(p.layer[l + 1], p.js, job) : nullptr;
        uint4 *out = job_ptr(p.layer[l], p.js, job);
        for (uint32_t k = threadIdx.x; k < per && first + k < n_l; k += THREADS) {
            const uint32_t i = first + k;
            uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t m[16];
            if (kids) {
                uint4 v[4];
                if (kids_shared) {
                    const uint4 *s = &thin[(j - 1) & 1][2 * k][0];
#pragma unroll
                    for (int q = 0; q < 4; q++) v[q] = s[q];
                } else if (j == 0) {  // other CTAs' nodes: from L2
#pragma unroll
                    for (int q = 0; q < 4; q++) v[q] = __ldcg(below + 4 * i + q);
                } else {  // this CTA's nodes of the level below
#pragma unroll
                    for (int q = 0; q < 4; q++) v[q] = below[4 * i + q];
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    m[4 * q] = v[q].x; m[4 * q + 1] = v[q].y; m[4 * q + 2] = v[q].z; m[4 * q + 3] = v[q].w;
                }
                compress(h, m, one);
            }
            uint32_t c0 = 0;
            for (; c0 + 16 <= nc; c0 += 16) {  // full chunks: no per-word bound checks
#pragma unroll
                for (int w = 0; w < 16; w++) m[w] = __ldg(ct[c0 + w] + i);
                compress(h, m, one);
            }
            if (c0 < nc) {  // the zero-padded last chunk
#pragma unroll
                for (int w = 0; w < 16; w++) {
                    const uint32_t cw = c0 + w;
                    m[w] = cw < nc ? __ldg(ct[cw] + i) : 0u;
                }
                compress(h, m, one);
            }
            const uint4 lo = make_uint4(h[0], h[1], h[2], h[3]), hi = make_uint4(h[4], h[5], h[6], h[7]);
            out[2 * i] = lo;
            out[2 * i + 1] = hi;
            if (to_shared) {
                thin[j & 1][k][0] = lo;
                thin[j & 1][k][1] = hi;
            }
        }
        __syncthreads();  // this level's nodes are visible to the whole CTA
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) merkle_tree_kernel(const __grid_constant__ TreeParams p, uint32_t one) {
    __shared__ uint4 thin[2][THREADS][2];
    __shared__ uint32_t next;
    uint32_t b = 0, u = blockIdx.x;
    for (;;) {
        merkle_unit<THREADS>(p, p.band[b], u, thin, one);
        if (b + 1 >= p.n_bands) return;
        const TreeBand &up = p.band[b + 1];
        const uint32_t parent = u / up.fan;
        // The unit's last level is its one node, written by thread 0 (the barrier that
        // ends merkle_unit is behind it): only that store needs to be visible to other
        // CTAs before the ticket.
        if (threadIdx.x == 0) {
            __threadfence();
            uint32_t *t = job_ptr(p.tickets, p.js, blockIdx.y) + up.ticket_base + parent;
            const uint32_t want = up.fan < p.band[b].units ? up.fan : p.band[b].units;
            const uint32_t arrived = atomicAdd(t, 1u) + 1;
            next = arrived == want;
            if (arrived == want) *t = 0;
        }
        __syncthreads();
        if (!next) return;
        __threadfence();  // the other units' nodes, after their tickets
        u = parent;
        b++;
    }
}

// The band partition of a tree of 2^max_log leaves under the current launch tunables.
struct TreePlan {
    int threads = 256;
    TreeBand band[MERKLE_MAX_BANDS];
    uint32_t n_bands = 0;
    uint32_t n_tickets = 0;
};

int plan_tree_bands(uint32_t max_log, TreePlan &tp) {
    STWO_REQUIRE(max_log <= 30, STWO_ERR_UNSUPPORTED_SIZE, "merkle tree of log size %u", max_log);
    // CTA size (tunable): 128, 256 or 512 threads, i.e. 8, 9 or 10 layers per band,
    // plus `spread` more (tunable, 0..5) while a band still fills every SM with 1024
    // threads (the CTAs that are resident at once: four of 256 threads at 64 registers).
    // Requiring 2048 capped the spread of mid-size trees and so their units' size: at 4
    // columns x 2^19..2^21 leaves 0.0995 / 0.150 / 0.242 ms against 0.0884 / 0.137 /
    // 0.227 ms now.
    const int threads = tunable(TUNE_MERKLE_SUB_THREADS);
    tp.threads = threads;
    const int tlog = threads == 512 ? 9 : threads == 128 ? 7 : 8;
    const int max_spread = tunable(TUNE_MERKLE_SUB_SPREAD);
    const uint64_t min_blocks = (uint64_t)device_sm_count() * 1024 / threads;
    tp.n_bands = 0;
    tp.n_tickets = 0;
    int top = (int)max_log;
    while (top >= 0) {
        STWO_REQUIRE(tp.n_bands < (uint32_t)MERKLE_MAX_BANDS, STWO_ERR_UNSUPPORTED_SIZE, "merkle tree bands");
        int spread = max_spread;
        while (spread > 0 && (top < tlog + spread || ((1ull << top) >> (tlog + spread)) < min_blocks)) spread--;
        const int max_levels = tlog + 1 + spread;
        const uint32_t levels = (uint32_t)std::min(top + 1, max_levels);
        const uint64_t nodes = 1ull << top, per = (uint64_t)threads << spread;
        const uint64_t units = nodes > per ? nodes / per : 1;
        STWO_REQUIRE(levels == (uint32_t)max_levels || units == 1, STWO_ERR_UNSUPPORTED_SIZE, "merkle subtree partition");
        TreeBand &bd = tp.band[tp.n_bands];
        bd.top = (uint32_t)top;
        bd.levels = levels;
        bd.spread = (uint32_t)spread;
        bd.has_prev = top < (int)max_log;
        bd.units = (uint32_t)units;
        bd.fan = tp.n_bands > 0 ? (uint32_t)(2 * per) : 0;
        bd.ticket_base = tp.n_bands > 0 ? tp.n_tickets : 0;
        if (tp.n_bands > 0) tp.n_tickets += (uint32_t)units;
        tp.n_bands++;
        top -= (int)levels;
    }
    return STWO_OK;
}

template <int THREADS>
void launch_tree(const TreeParams &p, uint32_t blocks, uint32_t jobs, cudaStream_t st) {
    merkle_tree_kernel<THREADS><<<dim3(blocks, jobs), THREADS, 0, st>>>(p, 1u);
}

template <int CAP>
void launch_layer(uint32_t log_size, const uint32_t *prev, const uint32_t *const *cols, uint32_t n_cols,
                  bool cols_on_device, uint32_t *out, unsigned blocks, cudaStream_t st) {
    MerkleCols<CAP> mc;  // parameter block (host stack)
    if (!cols_on_device)
        for (uint32_t i = 0; i < n_cols; i++) mc.c[i] = cols[i];
    if (cols_on_device)
        merkle_layer_kernel<true, CAP><<<blocks, 256, 0, st>>>(log_size, reinterpret_cast<const uint4 *>(prev), mc,
                                                               cols, n_cols, reinterpret_cast<uint4 *>(out), 1u);
    else
        merkle_layer_kernel<false, CAP><<<blocks, 256, 0, st>>>(log_size, reinterpret_cast<const uint4 *>(prev), mc,
                                                                nullptr, n_cols, reinterpret_cast<uint4 *>(out), 1u);
}

}  // namespace

uint32_t merkle_tree_tickets(uint32_t max_log) {
    TreePlan tp;
    return plan_tree_bands(max_log, tp) == STWO_OK ? tp.n_tickets : 0;
}

// A whole tree whose per-layer columns are device pointer tables: level_cols[l],
// level_ncols[l] for layer l (table may be null when the count is 0); layers[l] the
// 2^l-node outputs. With `tickets` (n_tickets zeroed words, at least
// merkle_tree_tickets(max_log); left zeroed) one launch; otherwise one launch per band.
// jobs trees of one shape at once: tree k's layers, tables and tickets are tree 0's
// moved by k * js bytes.
int merkle_tree_dev_async(uint32_t max_log, const uint32_t *const *const *level_cols, const uint32_t *level_ncols,
                          uint32_t *const *layers, uint32_t *tickets, uint32_t n_tickets, uint32_t jobs, size_t js,
                          cudaStream_t st) {
    TreePlan tp;
    int rc = plan_tree_bands(max_log, tp);
    if (rc) return rc;
    TreeParams p{};
    for (uint32_t l = 0; l <= max_log; l++) {
        STWO_REQUIRE(((uintptr_t)layers[l] & 15) == 0, STWO_ERR_INVALID_ARGUMENT, "hash buffers must be 16-byte aligned");
        p.layer[l] = reinterpret_cast<uint4 *>(layers[l]);
        p.cols[l] = level_cols[l];
        p.n_cols[l] = level_ncols[l];
    }
    STWO_REQUIRE(jobs >= 1 && jobs <= 65535, STWO_ERR_INVALID_ARGUMENT, "merkle trees per launch: %u", jobs);
    p.js = js;
    auto launch = [&](uint32_t blocks) {
        if (tp.threads == 512) launch_tree<512>(p, blocks, jobs, st);
        else if (tp.threads == 128) launch_tree<128>(p, blocks, jobs, st);
        else launch_tree<256>(p, blocks, jobs, st);
    };
    if (tickets && n_tickets >= tp.n_tickets) {
        for (uint32_t b = 0; b < tp.n_bands; b++) p.band[b] = tp.band[b];
        p.n_bands = tp.n_bands;
        p.tickets = tickets;
        launch(tp.band[0].units);
        STWO_LAUNCH_CHECK("merkle_tree_kernel");
        return STWO_OK;
    }
    p.n_bands = 1;
    for (uint32_t b = 0; b < tp.n_bands; b++) {
        p.band[0] = tp.band[b];
        launch(tp.band[b].units);
        STWO_LAUNCH_CHECK("merkle_tree_kernel");
    }
    return STWO_OK;
}

int merkle_layer_async(uint32_t log_size, const uint32_t *prev, const uint32_t *const *cols, uint32_t n_cols,
                       bool cols_on_device, uint32_t *out, cudaStream_t st) {
    STWO_REQUIRE(log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "merkle layer of log size %u", log_size);
    STWO_REQUIRE(cols_on_device || n_cols <= (uint32_t)MERKLE_MAX_COLS, STWO_ERR_UNSUPPORTED_SIZE,
                 "at most %d columns per merkle layer call", MERKLE_MAX_COLS);
    STWO_REQUIRE(((uintptr_t)out & 15) == 0 && ((uintptr_t)prev & 15) == 0, STWO_ERR_INVALID_ARGUMENT,
                 "hash buffers must be 16-byte aligned");
    uint64_t n = 1ull << log_size;
    uint64_t blocks = (n + 255) / 256;
    uint64_t cap = (uint64_t)device_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    if (cols_on_device || n_cols <= 16) launch_layer<16>(log_size, prev, cols, n_cols, cols_on_device, out, (unsigned)blocks, st);
    else if (n_cols <= 256) launch_layer<256>(log_size, prev, cols, n_cols, false, out, (unsigned)blocks, st);
    else launch_layer<MERKLE_MAX_COLS>(log_size, prev, cols, n_cols, false, out, (unsigned)blocks, st);
    STWO_LAUNCH_CHECK("merkle_layer_kernel");
    return STWO_OK;
}

}  // namespace stwo

using namespace stwo;

extern "C" {

int stwo_merkle_commit_layer(uint32_t log_size, const uint32_t *prev_layer, const uint32_t *const *columns,
                             uint32_t n_columns, uint32_t *out, void *stream) {
    return merkle_layer_async(log_size, prev_layer, columns, n_columns, false, out, as_stream(stream));
}

int stwo_merkle_commit_tree(const uint32_t *const *columns, const uint32_t *log_sizes, uint32_t n_columns,
                            uint32_t max_log, uint32_t *const *layers, void *stream) {
    STWO_REQUIRE(max_log <= 30 && layers && (n_columns == 0 || (columns && log_sizes)), STWO_ERR_INVALID_ARGUMENT,
                 "merkle tree arguments");
    cudaStream_t st = as_stream(stream);
    // Per-layer column tables, in one staged device buffer: layer l's columns in the
    // caller's order.
    std::vector<const uint32_t *> flat;
    std::vector<uint32_t> start(max_log + 1, 0), count(max_log + 1, 0);
    for (int l = (int)max_log; l >= 0; l--) {
        start[l] = (uint32_t)flat.size();
        for (uint32_t i = 0; i < n_columns; i++) {
            STWO_REQUIRE(log_sizes[i] <= max_log, STWO_ERR_INVALID_ARGUMENT, "column %u of log size %u above the tree's %u",
                         i, log_sizes[i], max_log);
            STWO_REQUIRE(columns[i], STWO_ERR_INVALID_ARGUMENT, "null column pointer");
            if (log_sizes[i] == (uint32_t)l) flat.push_back(columns[i]);
        }
        count[l] = (uint32_t)flat.size() - start[l];
    }
    // The tree kernel's tickets (zeroed words) follow the tables in the same buffer.
    const uint32_t n_tickets = merkle_tree_tickets(max_log);
    const size_t tick_words = ((size_t)n_tickets + 1) / 2;  // in pointer-sized words
    const size_t table_words = flat.size();
    flat.resize(table_words + tick_words + 1, nullptr);  // (never an empty allocation)
    void *table = nullptr;
    int arc = pool_alloc(&table, sizeof(void *) * flat.size(), st);
    if (arc) return arc;
    // from pageable memory: the copy has read `flat` when it returns
    cudaError_t e = cudaMemcpyAsync(table, flat.data(), sizeof(void *) * flat.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(table, st);
        return set_error(STWO_ERR_CUDA, "merkle column table: %s", cudaGetErrorString(e));
    }
    std::vector<const uint32_t *const *> level_cols(max_log + 1, nullptr);
    for (uint32_t l = 0; l <= max_log; l++)
        if (count[l]) level_cols[l] = static_cast<const uint32_t *const *>(table) + start[l];
    uint32_t *tickets = reinterpret_cast<uint32_t *>(static_cast<const uint32_t **>(table) + table_words);
    int rc = merkle_tree_dev_async(max_log, level_cols.data(), count.data(), layers, tickets, n_tickets, 1, 0, st);
    cudaFreeAsync(table, st);
    return rc;
}

void commit_on_first_layer(size_t size, size_t amount_of_columns, uint32_t *const *columns, stwo_blake2s_hash *result) {
    if (!is_pow2(size)) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "layer size %zu is not a power of two", size);
        return;
    }
    sync_default_stream(merkle_layer_async(log2_u64(size), nullptr, const_cast<const uint32_t *const *>(columns),
                                           (uint32_t)amount_of_columns, true, reinterpret_cast<uint32_t *>(result), 0));
}

void commit_on_layer_with_previous(size_t size, size_t amount_of_columns, uint32_t *const *columns,
                                   const stwo_blake2s_hash *previous_layer, stwo_blake2s_hash *result) {
    if (!is_pow2(size)) {
        set_error(STWO_ERR_INVALID_ARGUMENT, "layer size %zu is not a power of two", size);
        return;
    }
    sync_default_stream(merkle_layer_async(log2_u64(size), reinterpret_cast<const uint32_t *>(previous_layer),
                                           const_cast<const uint32_t *const *>(columns), (uint32_t)amount_of_columns,
                                           true, reinterpret_cast<uint32_t *>(result), 0));
}

}  // extern "C"
