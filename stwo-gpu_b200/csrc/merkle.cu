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
#include "blake2s.cuh"
#include "common.cuh"

namespace stwo {
namespace {

using blake::compress;

constexpr int MERKLE_MAX_COLS = 2048;

struct MerkleCols {
    const uint32_t *c[MERKLE_MAX_COLS];
};

// COLS_ON_DEVICE: column pointers come from a device array (reference ABI);
// otherwise from the kernel parameter block.
template <bool COLS_ON_DEVICE>
__global__ void __launch_bounds__(256) merkle_layer_kernel(uint32_t log_size, const uint4 *__restrict__ prev,
                                                           const __grid_constant__ MerkleCols cols,
                                                           const uint32_t *const *__restrict__ dev_cols,
                                                           uint32_t n_cols, uint4 *__restrict__ out, uint32_t one) {
    const uint64_t n = 1ull << log_size;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        uint32_t m[16];
        if (prev) {
            const uint4 *p = prev + 4 * i;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint4 v = __ldg(p + q);
                m[4 * q] = v.x; m[4 * q + 1] = v.y; m[4 * q + 2] = v.z; m[4 * q + 3] = v.w;
            }
            compress(h, m, one);
        }
        for (uint32_t c0 = 0; c0 < n_cols; c0 += 16) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                uint32_t cj = c0 + j;
                const uint32_t *col = nullptr;
                if (cj < n_cols) col = COLS_ON_DEVICE ? dev_cols[cj] : cols.c[cj];
                m[j] = col ? __ldg(col + i) : 0u;
            }
            compress(h, m, one);
        }
        out[2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
        out[2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
    }
}

// The column-free top of a tree in one launch of one CTA: layers top_log .. 0, each
// node the compression of its two children. The children of layer top_log come from
// `prev`; later layers read the layer this CTA wrote before the barrier.
struct TopLayers {
    uint4 *layer[32];  // layer[l]: 2^l nodes (2 uint4 each)
};

constexpr int MERKLE_TOP_THREADS = 512;

__global__ void __launch_bounds__(MERKLE_TOP_THREADS) merkle_top_kernel(const uint4 *prev,
                                                                       const __grid_constant__ TopLayers t,
                                                                       uint32_t top_log, uint32_t one) {
    const uint4 *src = prev;
    for (int l = (int)top_log; l >= 0; l--) {
        uint4 *dst = t.layer[l];
        for (uint32_t i = threadIdx.x; i < (1u << l); i += blockDim.x) {
            uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint32_t m[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint4 v = src[4 * i + q];
                m[4 * q] = v.x; m[4 * q + 1] = v.y; m[4 * q + 2] = v.z; m[4 * q + 3] = v.w;
            }
            compress(h, m, one);
            dst[2 * i] = make_uint4(h[0], h[1], h[2], h[3]);
            dst[2 * i + 1] = make_uint4(h[4], h[5], h[6], h[7]);
        }
        __syncthreads();  // this layer's global writes are visible to the whole CTA
        src = dst;
    }
}

}  // namespace

// Hashes layers prev_log-1 .. 0 of a tree whose layers (host array of device
// pointers, indexed by log size) are all column-free below prev_log.
int merkle_top_async(uint32_t prev_log, uint32_t *const *layers, cudaStream_t st) {
    STWO_REQUIRE(prev_log >= 1 && prev_log <= 16, STWO_ERR_UNSUPPORTED_SIZE, "merkle top from log size %u", prev_log);
    TopLayers t{};
    for (uint32_t l = 0; l < prev_log; l++) {
        t.layer[l] = reinterpret_cast<uint4 *>(layers[l]);
        STWO_REQUIRE(((uintptr_t)layers[l] & 15) == 0, STWO_ERR_INVALID_ARGUMENT, "hash buffers must be 16-byte aligned");
    }
    STWO_REQUIRE(((uintptr_t)layers[prev_log] & 15) == 0, STWO_ERR_INVALID_ARGUMENT,
                 "hash buffers must be 16-byte aligned");
    merkle_top_kernel<<<1, MERKLE_TOP_THREADS, 0, st>>>(reinterpret_cast<const uint4 *>(layers[prev_log]), t,
                                                         prev_log - 1, 1u);
    STWO_LAUNCH_CHECK("merkle_top_kernel");
    return STWO_OK;
}

int merkle_layer_async(uint32_t log_size, const uint32_t *prev, const uint32_t *const *cols, uint32_t n_cols,
                       bool cols_on_device, uint32_t *out, cudaStream_t st) {
    STWO_REQUIRE(log_size <= 31, STWO_ERR_UNSUPPORTED_SIZE, "merkle layer of log size %u", log_size);
    STWO_REQUIRE(cols_on_device || n_cols <= (uint32_t)MERKLE_MAX_COLS, STWO_ERR_UNSUPPORTED_SIZE,
                 "at most %d columns per merkle layer call", MERKLE_MAX_COLS);
    STWO_REQUIRE(((uintptr_t)out & 15) == 0 && ((uintptr_t)prev & 15) == 0, STWO_ERR_INVALID_ARGUMENT,
                 "hash buffers must be 16-byte aligned");
    MerkleCols mc;  // parameter block (host stack)
    if (!cols_on_device)
        for (uint32_t i = 0; i < n_cols; i++) mc.c[i] = cols[i];
    uint64_t n = 1ull << log_size;
    uint64_t blocks = (n + 255) / 256;
    uint64_t cap = (uint64_t)device_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    if (cols_on_device)
        merkle_layer_kernel<true><<<(unsigned)blocks, 256, 0, st>>>(log_size, reinterpret_cast<const uint4 *>(prev), mc,
                                                                    cols, n_cols, reinterpret_cast<uint4 *>(out), 1u);
    else
        merkle_layer_kernel<false><<<(unsigned)blocks, 256, 0, st>>>(log_size, reinterpret_cast<const uint4 *>(prev), mc,
                                                                     nullptr, n_cols, reinterpret_cast<uint4 *>(out), 1u);
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
