// BLAKE2s compression on the device, as the Merkle hasher and the proof-of-work search
// use it: the message and the 16-word working state in registers, the round
// permutation resolved at compile time, counter and flags zero (RFC 7693 with
// t = 0, f = 0).
#pragma once
#include <cstdint>

namespace stwo {
namespace blake {

__device__ __forceinline__ uint32_t rotr(uint32_t x, uint32_t c) { return __funnelshift_r(x, x, c); }

#ifndef STWO_B2S_PRMT
#define STWO_B2S_PRMT 1
#endif
// Byte-aligned rotations as byte permutes.
__device__ __forceinline__ uint32_t rotr16(uint32_t x) {
#if STWO_B2S_PRMT
    return __byte_perm(x, 0, 0x1032);
#else
    return rotr(x, 16);
#endif
}
__device__ __forceinline__ uint32_t rotr8(uint32_t x) {
#if STWO_B2S_PRMT
    return __byte_perm(x, 0, 0x0321);
#else
    return rotr(x, 8);
#endif
}

__device__ constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                            0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

// c + d as an integer multiply-add by a runtime 1: it issues to the FMA pipe,
// which the rotate/xor/add-heavy compression otherwise leaves idle while the ALU
// pipe saturates. Every addition of G goes there (measured on B200: 19.2 G
// compressions/s against 18.4 with the three-input a + b + m on the ALU pipe).
__device__ __forceinline__ uint32_t add_on_fma(uint32_t c, uint32_t d, uint32_t one) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(d), "r"(one), "r"(c));
    return r;
}

// FMA: the additions as multiply-adds on the FMA pipe, for many threads hashing at
// once (the xors and rotations keep the ALU pipe busy). Otherwise the three-input
// a + b + m and c + d on the ALU pipe: two instructions fewer a G, for one thread
// hashing alone (the device channel), whose time is its own instruction stream.
template <bool FMA>
__device__ __forceinline__ uint32_t add3(uint32_t a, uint32_t x, uint32_t b, uint32_t one) {
    if (FMA) return add_on_fma(add_on_fma(a, x, one), b, one);
    return a + x + b;
}
template <bool FMA>
__device__ __forceinline__ uint32_t add2(uint32_t c, uint32_t d, uint32_t one) {
    if (FMA) return add_on_fma(c, d, one);
    return c + d;
}

#define STWO_G(a, b, c, d, x, y)    \
    a = add3<FMA>(a, (x), b, one);  \
    d = rotr16(d ^ a);              \
    c = add2<FMA>(c, d, one);       \
    b = rotr(b ^ c, 12);            \
    a = add3<FMA>(a, (y), b, one);  \
    d = rotr8(d ^ a);               \
    c = add2<FMA>(c, d, one);       \
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

// Compression with byte counter t (low word) and finalisation flag f0; the Merkle
// hasher and the nonce mixing use t = f0 = 0.
template <bool FMA = true>
__device__ __forceinline__ void compress_tf(uint32_t h[8], const uint32_t m[16], uint32_t t, uint32_t f0,
                                            uint32_t one) {
    uint32_t v0 = h[0], v1 = h[1], v2 = h[2], v3 = h[3], v4 = h[4], v5 = h[5], v6 = h[6], v7 = h[7];
    uint32_t v8 = IV[0], v9 = IV[1], v10 = IV[2], v11 = IV[3], v12 = IV[4] ^ t, v13 = IV[5], v14 = IV[6] ^ f0,
             v15 = IV[7];
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

template <bool FMA = true>
__device__ __forceinline__ void compress(uint32_t h[8], const uint32_t m[16], uint32_t one) {
    compress_tf<FMA>(h, m, 0u, 0u, one);
}

}  // namespace blake
}  // namespace stwo
