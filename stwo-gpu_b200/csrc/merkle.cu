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
#include "common.cuh"

namespace stwo {
namespace {

constexpr int MERKLE_MAX_COLS = 2048;

__device__ __forceinline__ uint32_t rotr(uint32_t x, uint32_t c) { return __funnelshift_r(x, x, c); }

__device__ constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                            0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

// c + d as an integer multiply-add by a runtime 1: it issues to the FMA pipe,
// which the rotate/xor/add-heavy compression otherwise leaves idle while the ALU
// pipe saturates.
__device__ __forceinline__ uint32_t add_on_fma(uint32_t c, uint32_t d, uint32_t one) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(d), "r"(one), "r"(c));
    return r;
}

#define STWO_G(a, b, c, d, x, y)    \
    a = a + b + (x);                \
    d = rotr(d ^ a, 16);            \
    c = add_on_fma(c, d, one);      \
    b = rotr(b ^ c, 12);            \
    a = a + b + (y);                \
    d = rotr(d ^ a, 8);             \
    c = add_on_fma(c, d, one);      \
    b = rotr(b ^ c, 7);

// One BLAKE2s round with message permutation s0..s15 (RFC 7693 SIGMA rows).
#define STWO_ROUND(s0, s1, s2, s3, s4, s5, s6, s7, s8, s9, s10, s11, s12, s13, s14, s15) \
    { STWO_G(v0, v4, v8, v12, m[s0], m[s1])                                            \
      STWO_G(v1, v5, v9, v13, m[s2], m[s3])                                            \
      STWO_G(v2, v6, v10, v14, m[s4], m[s5])                                           \
      STWO_G(v3, v7, v11, v15, m[s6], m[s7])                                           \
      STWO_G(v0, v5, v10, v15, m[s8], m[s9])                                           \
      STWO_G(v1, v6, v11, v12, m[s10], m[s11])                                         \
      STWO_G(v2, v7, v8, v13, m[s12], m[s13])                                          \
      STWO_G(v3, v4, v9, v14, m[s14], m[s15]) }

__device__ __forceinline__ void compress(uint32_t h[8], const uint32_t m[16], uint32_t one) {
    uint32_t v0 = h[0], v1 = h[1], v2 = h[2], v3 = h[3], v4 = h[4], v5 = h[5], v6 = h[6], v7 = h[7];
    uint32_t v8 = IV[0], v9 = IV[1], v10 = IV[2], v11 = IV[3], v12 = IV[4], v13 = IV[5], v14 = IV[6], v15 = IV[7];
    STWO_ROUND(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15)
    STWO_ROUND(14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3)
    STWO_ROUND(11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4)
    STWO_ROUND(7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8)
    STWO_ROUND(9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13)
    STWO_ROUND(2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9)
    STWO_ROUND(12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11)
    STWO_ROUND(13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10)
    STWO_ROUND(6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5)
    STWO_ROUND(10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0)
    h[0] ^= v0 ^ v8;
    h[1] ^= v1 ^ v9;
    h[2] ^= v2 ^ v10;
    h[3] ^= v3 ^ v11;
    h[4] ^= v4 ^ v12;
    h[5] ^= v5 ^ v13;
    h[6] ^= v6 ^ v14;
    h[7] ^= v7 ^ v15;
}

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

}  // namespace

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
