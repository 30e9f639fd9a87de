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
__device__ __forceinline__ void merkle_node(uint64_t i, const uint4 *prev, ColAt col_at, uint32_t n_cols, uint4 *out,
                                            uint32_t one) {
    uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t m[16];
    if (prev) {
        const uint4 *p = prev + 4 * i;
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
    out[2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
    out[2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
}

// One layer, one thread per node. COLS_ON_DEVICE: column pointers come from a device
// array (reference ABI); otherwise from the parameter block.
template <bool COLS_ON_DEVICE, int CAP>
__global__ void __launch_bounds__(256) merkle_layer_kernel(uint32_t log_size, const uint4 *__restrict__ prev,
                                                           const __grid_constant__ MerkleCols<CAP> cols,
                                                           const uint32_t *const *__restrict__ dev_cols,
                                                           uint32_t n_cols, uint4 *__restrict__ out, uint32_t one) {
    const uint64_t n = 1ull << log_size;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (COLS_ON_DEVICE)
            merkle_node(i, prev, [&](uint32_t c) { return dev_cols[c]; }, n_cols, out, one);
        else
            merkle_node(i, prev, [&](uint32_t c) { return cols.c[c]; }, n_cols, out, one);
    }
}

// Up to log2(THREADS) + 1 + spread layers in one launch. CTA c owns the
// (THREADS << spread) >> j nodes of level j (layer top_log - j) that start at
// c * ((THREADS << spread) >> j): exactly the parents of the nodes it owned one level
// down, which it wrote itself before the barrier. Level j hashes the children (absent
// on the leaf layer) and the layer's columns (device pointer tables, one per level).
// With spread s a thread hashes 2^s nodes of the bottom level, so the CTA stays dense
// for s + 1 levels before its upper levels thin out.
constexpr int MERKLE_SUB_MAX_LEVELS = 15;  // 512 threads, spread 5: 16384 nodes -> 1 node

struct SubtreeParams {
    uint4 *layer[32];                                   // layer[l]: 2^l nodes
    const uint32_t *const *cols[MERKLE_SUB_MAX_LEVELS];  // device column tables per level
    uint32_t n_cols[MERKLE_SUB_MAX_LEVELS];
    uint32_t top_log, levels, has_prev, spread;
};

template <int THREADS>
__global__ void __launch_bounds__(THREADS) merkle_subtree_kernel(const __grid_constant__ SubtreeParams p, uint32_t one) {
    for (uint32_t j = 0; j < p.levels; j++) {
        const uint32_t l = p.top_log - j;
        const uint64_t per_cta = ((uint64_t)THREADS << p.spread) >> j;
        const uint64_t first = blockIdx.x * per_cta, n_l = 1ull << l;
        const uint4 *prev = (j > 0 || p.has_prev) ? p.layer[l + 1] : nullptr;
        const uint32_t *const *ct = p.cols[j];
        for (uint64_t k = threadIdx.x; k < per_cta && first + k < n_l; k += blockDim.x)
            merkle_node(first + k, prev, [&](uint32_t c) { return ct[c]; }, p.n_cols[j], p.layer[l], one);
        __syncthreads();  // this level's global writes are visible to the whole CTA
    }
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

// A whole tree whose per-layer columns are device pointer tables: level_cols[l],
// level_ncols[l] for layer l (table may be null when the count is 0); layers[l] the
// 2^l-node outputs. ceil((max_log + 1) / (log2(CTA size) + 1)) launches.
int merkle_tree_dev_async(uint32_t max_log, const uint32_t *const *const *level_cols, const uint32_t *level_ncols,
                          uint32_t *const *layers, cudaStream_t st) {
    STWO_REQUIRE(max_log <= 30, STWO_ERR_UNSUPPORTED_SIZE, "merkle tree of log size %u", max_log);
    SubtreeParams p{};
    for (uint32_t l = 0; l <= max_log; l++) {
        p.layer[l] = reinterpret_cast<uint4 *>(layers[l]);
        STWO_REQUIRE(((uintptr_t)layers[l] & 15) == 0, STWO_ERR_INVALID_ARGUMENT, "hash buffers must be 16-byte aligned");
    }
    // CTA size (tunable): 128, 256 or 512 threads, i.e. 8, 9 or 10 layers per launch,
    // plus `spread` more (tunable, 0..5) while the launch still fills every SM with
    // 2048 threads.
    const int threads = tunable(TUNE_MERKLE_SUB_THREADS);
    const int tlog = threads == 512 ? 9 : threads == 128 ? 7 : 8;
    const int max_spread = tunable(TUNE_MERKLE_SUB_SPREAD);
    const uint64_t min_blocks = (uint64_t)device_sm_count() * 2048 / threads;
    int top = (int)max_log;
    while (top >= 0) {
        int spread = max_spread;
        while (spread > 0 && (top < tlog + spread || ((1ull << top) >> (tlog + spread)) < min_blocks)) spread--;
        const int max_levels = tlog + 1 + spread;
        const uint32_t levels = (uint32_t)std::min(top + 1, max_levels);
        p.top_log = (uint32_t)top;
        p.levels = levels;
        p.has_prev = top < (int)max_log;
        p.spread = (uint32_t)spread;
        for (uint32_t j = 0; j < levels; j++) {
            p.cols[j] = level_cols[top - j];
            p.n_cols[j] = level_ncols[top - j];
        }
        const uint64_t nodes = 1ull << top, per_cta = (uint64_t)threads << spread;
        const uint64_t blocks = nodes > per_cta ? nodes / per_cta : 1;
        STWO_REQUIRE(levels == (uint32_t)max_levels || blocks == 1, STWO_ERR_UNSUPPORTED_SIZE, "merkle subtree partition");
        if (threads == 512) merkle_subtree_kernel<512><<<(unsigned)blocks, 512, 0, st>>>(p, 1u);
        else if (threads == 128) merkle_subtree_kernel<128><<<(unsigned)blocks, 128, 0, st>>>(p, 1u);
        else merkle_subtree_kernel<256><<<(unsigned)blocks, 256, 0, st>>>(p, 1u);
        STWO_LAUNCH_CHECK("merkle_subtree_kernel");
        top -= (int)levels;
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
    void *table = nullptr;
    if (!flat.empty()) {
        int arc = pool_alloc(&table, sizeof(void *) * flat.size(), st);
        if (arc) return arc;
        // from pageable memory: the copy has read `flat` when it returns
        cudaError_t e = cudaMemcpyAsync(table, flat.data(), sizeof(void *) * flat.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            cudaFreeAsync(table, st);
            return set_error(STWO_ERR_CUDA, "merkle column table: %s", cudaGetErrorString(e));
        }
    }
    std::vector<const uint32_t *const *> level_cols(max_log + 1, nullptr);
    for (uint32_t l = 0; l <= max_log; l++)
        if (count[l]) level_cols[l] = static_cast<const uint32_t *const *>(table) + start[l];
    int rc = merkle_tree_dev_async(max_log, level_cols.data(), count.data(), layers, st);
    if (table) cudaFreeAsync(table, st);
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
