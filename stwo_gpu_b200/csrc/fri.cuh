// FRI fold arithmetic shared by the fold kernels (fri.cu) and the prover's fused FRI
// tail (prover.cu): fold_line / fold_circle_into_line of one pair of values
// (cuda/src/fri/fold_line.cu:15-33, fold_circle_into_line.cu:19-45).
#pragma once
#include <cstdint>

#include "field.cuh"

namespace stwo {

// The circle fold's inverse twiddle for output h: from the first line layer's pairs
// [x, y] of the inverse-twiddle tree suffix lt0, in the pattern [y, -y, -x, x].
__device__ __forceinline__ uint32_t circle_itw(const uint32_t *__restrict__ lt0, uint64_t h) {
    uint64_t q = h >> 2;
    uint32_t r = (uint32_t)(h & 3u);
    uint32_t v = __ldg(lt0 + 2 * q + ((r >> 1) ^ 1u));
    return (r == 1u || r == 2u) ? m31_neg(v) : v;
}

// (a + b) + alpha * (a - b) * t
__host__ __device__ __forceinline__ qm31 fold_pair(qm31 a, qm31 b, uint32_t t, qm31 alpha) {
    qm31 s = qm31_add(a, b);
    qm31 d = qm31_scale(qm31_sub(a, b), t);
    return qm31_add(s, qm31_mul(alpha, d));
}

}  // namespace stwo
