// The Fiat-Shamir channel on the device: stwo's Blake2sChannel
// (core/channel/blake2s.rs) with Blake2sMerkleChannel's root mixing
// (core/vcs/blake2_merkle.rs), run by one thread so that a proof's challenges are
// drawn where the committed data already is, without a round trip to the host.
//
//   mix_root(r):    digest = BLAKE2s(digest || r)
//   mix_felts(f):   digest = BLAKE2s(digest || f as u32 LE words)
//   mix_nonce(k):   digest = compress(digest, [lo(k), hi(k), 0...]) (zero counter, flags)
//   draw:           BLAKE2s(digest || n_sent as u64 LE || 24 zero bytes), n_sent += 1
//   draw_felt:      first four of eight u32s, redrawn unless all eight are < 2P
// Every update of the digest resets n_sent.
#pragma once
#include <cstdint>

#include "blake2s.cuh"
#include "field.cuh"

namespace stwo {
namespace fs {

// Error bits a proof's device state records (the host reads them after the run).
constexpr uint32_t ERR_DRAW = 1;         // a felt draw needed more than 64 tries
constexpr uint32_t ERR_CONSTRAINTS = 2;  // the OODS composition check failed
constexpr uint32_t ERR_LAST_LAYER = 4;   // the last FRI layer exceeds its degree bound
constexpr uint32_t ERR_GRIND = 8;        // no proof-of-work nonce within the search bound

struct DevChannel {
    uint32_t digest[8];
    uint32_t n_sent_lo, n_sent_hi;
};

// BLAKE2s-256 (RFC 7693, unkeyed, 32-byte digest) of the words word(0..n_words-1),
// little endian. One thread runs the channel, so its compressions take the
// short-chain form (additions on the ALU pipe).
template <class W>
__device__ void blake2s_words(W word, uint32_t n_words, uint32_t out[8]) {
    const uint32_t one = 1;
    uint32_t h[8];
#pragma unroll
    for (int i = 0; i < 8; i++) h[i] = blake::IV[i];
    h[0] ^= 0x01010020u;  // digest length 32, fanout 1, depth 1
    uint32_t off = 0, m[16];
    while (n_words - off > 16) {
        for (int k = 0; k < 16; k++) m[k] = word(off + k);
        off += 16;
        blake::compress_tf<false>(h, m, off * 4, 0u, one);
    }
    for (uint32_t k = 0; k < 16; k++) m[k] = off + k < n_words ? word(off + k) : 0u;
    blake::compress_tf<false>(h, m, n_words * 4, 0xffffffffu, one);
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = h[i];
}

__device__ inline void ch_update(DevChannel &c, const uint32_t d[8]) {
    for (int i = 0; i < 8; i++) c.digest[i] = d[i];
    c.n_sent_lo = c.n_sent_hi = 0;
}

__device__ inline void ch_mix_root(DevChannel &c, const uint32_t *root) {
    uint32_t d[8];
    blake2s_words([&](uint32_t i) { return i < 8 ? c.digest[i] : root[i - 8]; }, 16, d);
    ch_update(c, d);
}

__device__ inline void ch_mix_felts(DevChannel &c, const qm31 *f, uint32_t n) {
    uint32_t d[8];
    blake2s_words(
        [&](uint32_t i) {
            if (i < 8) return c.digest[i];
            const qm31 &v = f[(i - 8) >> 2];
            switch ((i - 8) & 3u) {
                case 0: return v.a.a;
                case 1: return v.a.b;
                case 2: return v.b.a;
                default: return v.b.b;
            }
        },
        8 + 4 * n, d);
    ch_update(c, d);
}

__device__ inline void ch_mix_nonce(DevChannel &c, uint64_t nonce) {
    uint32_t h[8], m[16] = {0};
    for (int i = 0; i < 8; i++) h[i] = c.digest[i];
    m[0] = (uint32_t)nonce;
    m[1] = (uint32_t)(nonce >> 32);
    blake::compress<false>(h, m, 1u);
    ch_update(c, h);
}

__device__ inline void ch_draw_words(DevChannel &c, uint32_t out[8]) {
    blake2s_words(
        [&](uint32_t i) {
            if (i < 8) return c.digest[i];
            if (i == 8) return c.n_sent_lo;
            if (i == 9) return c.n_sent_hi;
            return 0u;
        },
        16, out);
    if (++c.n_sent_lo == 0) c.n_sent_hi++;
}

__device__ inline qm31 ch_draw_felt(DevChannel &c, uint32_t &error) {
    for (int tries = 0; tries < 64; tries++) {
        uint32_t u[8];
        ch_draw_words(c, u);
        bool ok = true;
        for (int i = 0; i < 8; i++) ok = ok && u[i] < 2 * P;
        if (!ok) continue;
        for (int i = 0; i < 4; i++) u[i] = u[i] >= P ? u[i] - P : u[i];
        return {{u[0], u[1]}, {u[2], u[3]}};
    }
    error |= ERR_DRAW;
    return qm31_zero();
}

}  // namespace fs
}  // namespace stwo
