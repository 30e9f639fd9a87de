// M31 / CM31 / QM31 field arithmetic and circle-group points for sm_100a.
//
// p = 2^31 - 1. Every function returns a canonical value in [0, p); inputs must be
// canonical. The field tower follows the reference (cuda/include/fields.cuh:5-19):
// CM31 = M31[i]/(i^2 + 1), QM31 = CM31[u]/(u^2 - (2 + i)); the coordinate order
// of a QM31 (a.a, a.b, b.a, b.b) is the reference's repr(C) CudaSecureField
// {a, b, c, d} (stwo_gpu_backend/src/cuda/bindings.rs:8-14).
//
// Multiplication: for a < 2^31 and b2 = 2*b (b < 2^31), the 64-bit product a*b2
// splits as hi = floor(a*b / 2^31) and lo>>1 = (a*b) mod 2^31, so
// a*b = hi*2^31 + lo>>1 == hi + lo>>1 (mod p) with hi + lo>>1 <= 2p; one
// conditional subtraction finishes. Operands that are reused (twiddles) are kept
// pre-doubled so the doubling is paid once.
#pragma once
#include <cstdint>

namespace stwo {

constexpr uint32_t P = 0x7fffffffu;

struct cm31 { uint32_t a, b; };
struct qm31 { cm31 a, b; };
struct cpoint { uint32_t x, y; };

__host__ __device__ __forceinline__ uint32_t reduce_once(uint32_t s) {
    // s in [0, 2p]  ->  [0, p)
#ifdef __CUDA_ARCH__
    return min(s, s - P);
#else
    return s >= P ? s - P : s;
#endif
}

__host__ __device__ __forceinline__ uint32_t m31_add(uint32_t a, uint32_t b) { return reduce_once(a + b); }

__host__ __device__ __forceinline__ uint32_t m31_sub(uint32_t a, uint32_t b) {
    uint32_t d = a - b;
#ifdef __CUDA_ARCH__
    return min(d, d + P);
#else
    return a >= b ? d : d + P;
#endif
}

__host__ __device__ __forceinline__ uint32_t m31_neg(uint32_t a) { return a ? P - a : 0u; }

// a * b where b2 = 2*b (pre-doubled operand).
__host__ __device__ __forceinline__ uint32_t m31_mul2(uint32_t a, uint32_t b2) {
#ifdef __CUDA_ARCH__
    uint64_t w = (uint64_t)a * b2;
    uint32_t lo = (uint32_t)w, hi = (uint32_t)(w >> 32);
    return reduce_once(hi + (lo >> 1));
#else
    uint64_t w = (uint64_t)a * b2;
    return reduce_once((uint32_t)(w >> 32) + ((uint32_t)w >> 1));
#endif
}

__host__ __device__ __forceinline__ uint32_t m31_mul(uint32_t a, uint32_t b) { return m31_mul2(a, b << 1); }

// Unreduced dot products: acc += a * b for canonical a, b (< P), one 32x32->64-bit
// multiply-add per term. Each product is below 2^62, and a folded accumulator below
// 2^34, so three terms fit between folds.
__host__ __device__ __forceinline__ uint64_t mac64(uint64_t acc, uint32_t a, uint32_t b) {
    return acc + (uint64_t)a * b;
}
// A value congruent to acc mod P, below 2^34.
__host__ __device__ __forceinline__ uint64_t fold64(uint64_t acc) { return (acc & P) + (acc >> 31); }
#ifdef __CUDACC__
// fold64 as one wide multiply-add on the FMA pipe: acc = hi * 2^32 + lo = 2 hi + lo
// (mod P), below 3 * 2^32 (so below 2^34 like fold64). After it, four products of
// values below 2^31 still fit: 3 * 2^32 + 4 (2^31 - 1)^2 < 2^64. `two` must be 2,
// passed at run time so that the compiler keeps the multiply-add instead of turning
// it into shifts and adds on the ALU pipe, which the surrounding field arithmetic
// already keeps busy.
__device__ __forceinline__ uint64_t fold64_fma(uint64_t acc, uint32_t two) {
    uint64_t r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"((uint32_t)(acc >> 32)), "r"(two), "l"(acc & 0xffffffffull));
    return r;
}
#endif
// acc mod P, canonical.
__host__ __device__ __forceinline__ uint32_t reduce64_p(uint64_t acc) {
    uint64_t s = (acc & P) + (acc >> 31);
    s = (s & P) + (s >> 31);
    return reduce_once((uint32_t)s);
}

__host__ __device__ __forceinline__ uint32_t m31_sqr(uint32_t a) { return m31_mul(a, a); }

__host__ __device__ inline uint32_t m31_pow(uint32_t a, uint64_t e) {
    uint32_t r = 1;
    while (e) {
        if (e & 1) r = m31_mul(r, a);
        a = m31_mul(a, a);
        e >>= 1;
    }
    return r;
}

__host__ __device__ __forceinline__ uint32_t m31_sqr_n(uint32_t a, int n) {
    for (int i = 0; i < n; i++) a = m31_sqr(a);
    return a;
}

// Inverse by Fermat, a^(p-2) with p - 2 = 4 (2^29 - 1) + 1, through the chain of
// a^(2^k - 1) for k = 1, 2, 3, 6, 12, 24, 27, 29: 30 squarings and 8 products.
__host__ __device__ inline uint32_t m31_inv(uint32_t a) {
    const uint32_t a2 = m31_mul(m31_sqr(a), a);            // 2^2 - 1
    const uint32_t a3 = m31_mul(m31_sqr(a2), a);           // 2^3 - 1
    const uint32_t a6 = m31_mul(m31_sqr_n(a3, 3), a3);     // 2^6 - 1
    const uint32_t a12 = m31_mul(m31_sqr_n(a6, 6), a6);    // 2^12 - 1
    const uint32_t a24 = m31_mul(m31_sqr_n(a12, 12), a12); // 2^24 - 1
    const uint32_t a27 = m31_mul(m31_sqr_n(a24, 3), a3);   // 2^27 - 1
    const uint32_t a29 = m31_mul(m31_sqr_n(a27, 2), a2);   // 2^29 - 1
    return m31_mul(m31_sqr_n(a29, 2), a);                  // 2^31 - 3
}

// 2^-k mod p = 2^(31-k) for 0 <= k <= 31.
__host__ __device__ __forceinline__ uint32_t m31_inv_pow2(uint32_t k) { return k == 0 ? 1u : (1u << (31 - k)); }

// ---------------------------------------------------------------- CM31
__host__ __device__ __forceinline__ cm31 cm31_add(cm31 x, cm31 y) { return {m31_add(x.a, y.a), m31_add(x.b, y.b)}; }
__host__ __device__ __forceinline__ cm31 cm31_sub(cm31 x, cm31 y) { return {m31_sub(x.a, y.a), m31_sub(x.b, y.b)}; }
__host__ __device__ __forceinline__ cm31 cm31_neg(cm31 x) { return {m31_neg(x.a), m31_neg(x.b)}; }
__host__ __device__ __forceinline__ cm31 cm31_mul(cm31 x, cm31 y) {
    return {m31_sub(m31_mul(x.a, y.a), m31_mul(x.b, y.b)), m31_add(m31_mul(x.a, y.b), m31_mul(x.b, y.a))};
}
__host__ __device__ __forceinline__ cm31 cm31_scale(cm31 x, uint32_t s) { return {m31_mul(x.a, s), m31_mul(x.b, s)}; }
// (a + b i)^2 = (a + b)(a - b) + 2ab i: two products.
__host__ __device__ __forceinline__ cm31 cm31_sqr(cm31 x) {
    const uint32_t ab = m31_mul(x.a, x.b);
    return {m31_mul(m31_add(x.a, x.b), m31_sub(x.a, x.b)), m31_add(ab, ab)};
}
__host__ __device__ inline cm31 cm31_inv(cm31 x) {
    uint32_t f = m31_inv(m31_add(m31_mul(x.a, x.a), m31_mul(x.b, x.b)));
    return {m31_mul(x.a, f), m31_mul(m31_neg(x.b), f)};
}

// ---------------------------------------------------------------- QM31
__host__ __device__ __forceinline__ qm31 qm31_zero() { return {{0, 0}, {0, 0}}; }
__host__ __device__ __forceinline__ qm31 qm31_one() { return {{1, 0}, {0, 0}}; }
__host__ __device__ __forceinline__ qm31 qm31_from_m31(uint32_t v) { return {{v, 0}, {0, 0}}; }
__host__ __device__ __forceinline__ qm31 qm31_add(qm31 x, qm31 y) { return {cm31_add(x.a, y.a), cm31_add(x.b, y.b)}; }
__host__ __device__ __forceinline__ qm31 qm31_sub(qm31 x, qm31 y) { return {cm31_sub(x.a, y.a), cm31_sub(x.b, y.b)}; }
__host__ __device__ __forceinline__ qm31 qm31_neg(qm31 x) { return {cm31_neg(x.a), cm31_neg(x.b)}; }
__host__ __device__ __forceinline__ qm31 qm31_scale(qm31 x, uint32_t s) {
    uint32_t s2 = s << 1;
    return {{m31_mul2(x.a.a, s2), m31_mul2(x.a.b, s2)}, {m31_mul2(x.b.a, s2), m31_mul2(x.b.b, s2)}};
}
__host__ __device__ __forceinline__ qm31 qm31_mul_cm31(qm31 x, cm31 s) { return {cm31_mul(x.a, s), cm31_mul(x.b, s)}; }
// x y with x = (x0 + x1 i) + (x2 + x3 i) u, y likewise, u^2 = 2 + i, i^2 = -1:
//   (x0 + x1 i)(y0 + y1 i) + (2 + i)(x2 + x3 i)(y2 + y3 i)
//     + ((x0 + x1 i)(y2 + y3 i) + (x2 + x3 i)(y0 + y1 i)) u,
// i.e. per output coordinate a dot product of x with four coefficients derived from y:
//   r0 = x0 y0 - x1 y1 + x2 (2 y2 - y3) - x3 (y2 + 2 y3)
//   r1 = x0 y1 + x1 y0 + x2 (y2 + 2 y3) + x3 (2 y2 - y3)
//   r2 = x0 y2 - x1 y3 + x2 y0 - x3 y1
//   r3 = x0 y3 + x1 y2 + x2 y1 + x3 y0
// Negated coefficients are taken as P - c (in (0, P]), so every term is a product of
// values below 2^31; each coordinate accumulates its four 64-bit products (below 2^64)
// and is reduced once.
__host__ __device__ __forceinline__ qm31 qm31_mul(qm31 x, qm31 y) {
    const uint32_t y0 = y.a.a, y1 = y.a.b, y2 = y.b.a, y3 = y.b.b;
    const uint32_t ny1 = P - y1, ny3 = P - y3;
    const uint32_t e = m31_sub(m31_add(y2, y2), y3);  // 2 y2 - y3
    const uint32_t f = m31_add(y2, m31_add(y3, y3));  // y2 + 2 y3
    const uint32_t nf = P - f;
    const uint32_t x0 = x.a.a, x1 = x.a.b, x2 = x.b.a, x3 = x.b.b;
    const uint64_t r0 = mac64(mac64(mac64((uint64_t)x0 * y0, x1, ny1), x2, e), x3, nf);
    const uint64_t r1 = mac64(mac64(mac64((uint64_t)x0 * y1, x1, y0), x2, f), x3, e);
    const uint64_t r2 = mac64(mac64(mac64((uint64_t)x0 * y2, x1, ny3), x2, y0), x3, ny1);
    const uint64_t r3 = mac64(mac64(mac64((uint64_t)x0 * y3, x1, y2), x2, y1), x3, y0);
    return {{reduce64_p(r0), reduce64_p(r1)}, {reduce64_p(r2), reduce64_p(r3)}};
}
__host__ __device__ inline qm31 qm31_inv(qm31 x) {
    cm31 b2 = cm31_mul(x.b, x.b);
    cm31 rb2 = {m31_sub(m31_add(b2.a, b2.a), b2.b), m31_add(m31_add(b2.b, b2.b), b2.a)};
    cm31 d = cm31_inv(cm31_sub(cm31_mul(x.a, x.a), rb2));
    return {cm31_mul(x.a, d), cm31_neg(cm31_mul(x.b, d))};
}
__host__ __device__ inline qm31 qm31_pow(qm31 x, uint64_t e) {
    qm31 r = qm31_one();
    while (e) {
        if (e & 1) r = qm31_mul(r, x);
        x = qm31_mul(x, x);
        e >>= 1;
    }
    return r;
}
__host__ __device__ __forceinline__ qm31 qm31_conj(qm31 x) { return {x.a, cm31_neg(x.b)}; }
__host__ __device__ __forceinline__ bool qm31_eq(qm31 x, qm31 y) {
    return x.a.a == y.a.a && x.a.b == y.a.b && x.b.a == y.b.a && x.b.b == y.b.b;
}

// ---------------------------------------------------------------- circle group
// Generator of the order-2^31 circle group over M31 (cuda/include/point.cuh:17).
constexpr uint32_t CIRCLE_GEN_X = 2u, CIRCLE_GEN_Y = 1268011823u;

__host__ __device__ __forceinline__ cpoint point_mul(cpoint p, cpoint q) {
    return {m31_sub(m31_mul(p.x, q.x), m31_mul(p.y, q.y)), m31_add(m31_mul(p.x, q.y), m31_mul(p.y, q.x))};
}
__host__ __device__ __forceinline__ cpoint point_conj(cpoint p) { return {p.x, m31_neg(p.y)}; }

// GEN^(index mod 2^31).
__host__ __device__ inline cpoint index_to_point(uint32_t index) {
    index &= 0x7fffffffu;
    cpoint r = {1, 0}, b = {CIRCLE_GEN_X, CIRCLE_GEN_Y};
    while (index) {
        if (index & 1) r = point_mul(r, b);
        b = point_mul(b, b);
        index >>= 1;
    }
    return r;
}

__host__ __device__ __forceinline__ uint32_t bit_reverse_bits(uint32_t i, uint32_t log_size) {
#ifdef __CUDA_ARCH__
    return log_size == 0 ? i : (__brev(i) >> (32 - log_size));
#else
    if (log_size == 0) return i;
    uint32_t r = 0;
    for (uint32_t k = 0; k < log_size; k++) r |= ((i >> k) & 1u) << (log_size - 1 - k);
    return r;
#endif
}

}  // namespace stwo
