// Circle FFT (evaluate / interpolate) over M31 columns in bit-reversed order.
//
// Semantics follow PolyOps::evaluate / interpolate of the reference
// (cuda/src/poly/rfft.cu:5-141, ifft.cu:3-163, poly/utils.cu:3-22): layer k >= 1
// of a size-2^N transform pairs indices that differ in bit k, with twiddle
// line_twiddles[k-1][i >> (k+1)] read from the suffix of the twiddle tree that
// belongs to the domain; layer 0 (the circle layer) derives its twiddle from the
// first line layer's pairs [x, y] as [y, -y, -x, x]. Evaluate runs layers N-1..0
// with butterfly (a + t b, a - t b); interpolate runs 0..N-1 with
// (a + b, (a - b) t) and rescales by 2^-N.
//
// B200 design (not the reference's one-launch-per-layer scheme):
//  * A pass applies a contiguous range of layers [lo, hi) to tiles of up to 2^15
//    elements (128 KB) held in shared memory. The bottom pass works on contiguous
//    tiles; passes for higher layers use "strided" tiles of 2^(hi-lo) rows x 2^c
//    contiguous words (c >= 5, full 128-byte lines), so every HBM access is a
//    coalesced 16-byte vector access. A 2^24 column takes 2 passes, not 24.
//  * Inside a tile each thread owns 2^e elements (e <= 6) and applies up to e
//    layers per round in registers, touching shared memory once per round.
//    The XOR swizzle S(j) = j ^ ((j>>5 ^ j>>10) & 31) keeps every access pattern
//    used here (consecutive lanes on any 5-bit window below bit 15) free of bank
//    conflicts.
//  * Twiddles are read from the tree through the read-only path and doubled once
//    for the shift-free M31 product (field.cuh).
//  * Zero extension for evaluate is fused into the first pass (the upper layers
//    of a zero-padded input only copy it), the 2^-N rescale into the last pass.
//  * One launch serves every column of one size: up to 64 columns travel by value
//    in the parameter block; above that a device table of (src, dst) pointers
//    (staged by the call, or resident in the caller's device memory) serves them
//    all, so 2^16 columns take one launch per pass instead of 1024. Columns of
//    different sizes use separate launches on the same stream.
#include <algorithm>
#include <cstdlib>
#include <utility>
#include <vector>

#include "common.cuh"

namespace stwo {
namespace {

constexpr int MAX_TILE_LOG = 15;
constexpr int MAX_THREADS_LOG = 9;
constexpr int MAX_COLS_PER_LAUNCH = 64;

struct FftColumn {
    const uint32_t *src;
    uint32_t *dst;
};

struct FftLaunch {
    FftColumn cols[MAX_COLS_PER_LAUNCH];
    const FftColumn *table;  // device (src, dst) of every column, or null: cols[] above
    uint32_t src_from_dst;   // with a table: this pass reads table[col].dst (passes after the first)
    const uint32_t *tw;   // suffix of the tree for a size-2^N domain (2^(N-1) entries)
    uint32_t N;           // log size of the (virtual) transform
    uint32_t lo, hi;      // layers [lo, hi) applied by this pass
    uint32_t c;           // low global bits [0, c) spanned by a tile row
    uint32_t tile_log;    // log2 of tile elements = c + (hi - lo)
    uint32_t src_mask;    // src index mask (2^L - 1 for an extension read, else all ones)
    uint32_t scale2;      // 2 * scale factor applied on store, 0 = none
};

__device__ __forceinline__ uint32_t swz(uint32_t j) { return j ^ (((j >> 5) ^ (j >> 10)) & 31u); }

// Source and destination of column `col` of a launch.
__device__ __forceinline__ FftColumn fft_col(const FftLaunch &p, uint32_t col) {
    if (p.table) {
        const ulonglong2 t = __ldg(reinterpret_cast<const ulonglong2 *>(p.table) + col);
        FftColumn c{reinterpret_cast<const uint32_t *>(p.src_from_dst ? t.y : t.x), reinterpret_cast<uint32_t *>(t.y)};
        return c;
    }
    return p.cols[col];
}

// Doubled twiddle for layer k, group h.
__device__ __forceinline__ uint32_t twiddle2(const uint32_t *__restrict__ tw, uint32_t N, uint32_t k, uint32_t h) {
    if (k == 0) {
        uint32_t q = h >> 2, r = h & 3u;
        uint32_t v = __ldg(tw + 2 * q + ((r >> 1) ^ 1u));
        if (r == 1u || r == 2u) v = m31_neg(v);
        return v << 1;
    }
    uint32_t off = (1u << (N - 1)) - (1u << (N - k));
    return __ldg(tw + off + h) << 1;
}

template <bool INV>
__device__ __forceinline__ void butterfly(uint32_t &a, uint32_t &b, uint32_t t2) {
    if (INV) {
        uint32_t s = m31_add(a, b), d = m31_sub(a, b);
        a = s;
        b = m31_mul2(d, t2);
    } else {
        uint32_t t = m31_mul2(b, t2);
        b = m31_sub(a, t);
        a = m31_add(a, t);
    }
}

struct TileGeom {
    uint32_t gfix, cmask, c, lo;
    __device__ __forceinline__ uint32_t gidx(uint32_t j) const { return gfix | (j & cmask) | ((j >> c) << lo); }
};

// One round: each thread applies the RB layers of tile bits [a, a+RB) to its
// 2^LOG_E elements (2^(LOG_E-RB) groups of 2^RB).
template <int RB, int LOG_E, bool INV>
__device__ __forceinline__ void fft_round(uint32_t *sm, const FftLaunch &p, const TileGeom &g, uint32_t a,
                                          uint32_t W) {
    constexpr int R = 1 << RB;
    constexpr int GROUPS = 1 << (LOG_E - RB);
    const uint32_t amask = (1u << a) - 1u;
    const uint32_t k0 = p.lo + (a - p.c);  // global layer of bit a
#pragma unroll 1
    for (int grp = 0; grp < GROUPS; grp++) {
        uint32_t x = threadIdx.x | ((uint32_t)grp << W);
        uint32_t jb = (x & amask) | ((x >> a) << (a + RB));
        uint32_t gb = g.gidx(jb);
        uint32_t v[R];
#pragma unroll
        for (int m = 0; m < R; m++) v[m] = sm[swz(jb | ((uint32_t)m << a))];
#pragma unroll
        for (int uu = 0; uu < RB; uu++) {
            const int u = INV ? uu : RB - 1 - uu;
            const uint32_t k = k0 + u;
            const uint32_t hb = gb >> (k + 1);
#pragma unroll
            for (int q = 0; q < (R >> (u + 1)); q++) {
                uint32_t t2 = twiddle2(p.tw, p.N, k, hb + q);
#pragma unroll
                for (int l = 0; l < (1 << u); l++) {
                    const int m0 = (q << (u + 1)) | l;
                    butterfly<INV>(v[m0], v[m0 | (1 << u)], t2);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < R; m++) sm[swz(jb | ((uint32_t)m << a))] = v[m];
    }
}

template <int LOG_E, bool INV>
__device__ __forceinline__ void fft_round_dispatch(int rb, uint32_t *sm, const FftLaunch &p, const TileGeom &g,
                                                   uint32_t a, uint32_t W) {
    switch (rb) {
    case 1: fft_round<1, LOG_E, INV>(sm, p, g, a, W); break;
    case 2: if constexpr (LOG_E >= 2) fft_round<2, LOG_E, INV>(sm, p, g, a, W); break;
    case 3: if constexpr (LOG_E >= 3) fft_round<3, LOG_E, INV>(sm, p, g, a, W); break;
    case 4: if constexpr (LOG_E >= 4) fft_round<4, LOG_E, INV>(sm, p, g, a, W); break;
    case 5: if constexpr (LOG_E >= 5) fft_round<5, LOG_E, INV>(sm, p, g, a, W); break;
    case 6: if constexpr (LOG_E >= 6) fft_round<6, LOG_E, INV>(sm, p, g, a, W); break;
    default: break;
    }
}

template <int LOG_E, bool INV>
__global__ void __launch_bounds__(1 << MAX_THREADS_LOG) fft_pass_kernel(const __grid_constant__ FftLaunch p) {
    extern __shared__ uint32_t sm[];
    const uint32_t tile = 1u << p.tile_log;
    const uint32_t W = p.tile_log - LOG_E;  // log2(threads)
    const uint32_t tiles_log = p.N - p.tile_log;
    const uint32_t col = blockIdx.x >> tiles_log;
    const uint32_t T = blockIdx.x & ((1u << tiles_log) - 1u);
    const uint32_t low_fixed = p.lo - p.c;  // fixed bits [c, lo)
    TileGeom g;
    g.c = p.c;
    g.lo = p.lo;
    g.cmask = (1u << p.c) - 1u;
    g.gfix = ((T & ((1u << low_fixed) - 1u)) << p.c) | ((T >> low_fixed) << p.hi);

    const FftColumn fc = fft_col(p, col);
    const uint32_t *__restrict__ src = fc.src;
    uint32_t *__restrict__ dst = fc.dst;

    // Global -> shared: 4 consecutive tile elements are 4 consecutive words.
    for (uint32_t j = threadIdx.x * 4; j < tile; j += blockDim.x * 4) {
        uint32_t gi = g.gidx(j) & p.src_mask;
        uint4 v = __ldg(reinterpret_cast<const uint4 *>(src + gi));
        sm[swz(j)] = v.x;
        sm[swz(j + 1)] = v.y;
        sm[swz(j + 2)] = v.z;
        sm[swz(j + 3)] = v.w;
    }
    __syncthreads();

    const int g_bits = (int)(p.hi - p.lo);
    if (INV) {
        for (int s = 0; s < g_bits; s += LOG_E) {
            int rb = min(LOG_E, g_bits - s);
            fft_round_dispatch<LOG_E, INV>(rb, sm, p, g, p.c + s, W);
            __syncthreads();
        }
    } else {
        for (int top = g_bits; top > 0; top -= LOG_E) {
            int rb = min(LOG_E, top);
            fft_round_dispatch<LOG_E, INV>(rb, sm, p, g, p.c + (top - rb), W);
            __syncthreads();
        }
    }

    for (uint32_t j = threadIdx.x * 4; j < tile; j += blockDim.x * 4) {
        uint4 v;
        v.x = sm[swz(j)];
        v.y = sm[swz(j + 1)];
        v.z = sm[swz(j + 2)];
        v.w = sm[swz(j + 3)];
        if (p.scale2) {
            v.x = m31_mul2(v.x, p.scale2);
            v.y = m31_mul2(v.y, p.scale2);
            v.z = m31_mul2(v.z, p.scale2);
            v.w = m31_mul2(v.w, p.scale2);
        }
        *reinterpret_cast<uint4 *>(dst + g.gidx(j)) = v;
    }
}

// ---------------------------------------------------------------------------
// Specialised pass over 2^14-element tiles: 256 threads x 64 elements (or 512 x 32),
// three CTAs per SM so that one CTA's global loads and stores overlap the others'
// butterflies (the transform is bound by integer issue, not by HBM).
//
// Tile index bits: [0, C) columns of a strided tile (consecutive global words),
// [C, C+G) the G layer bits of the pass, [C+G, 14) "slots": for a single-pass
// transform of a 2^G column (G < 14) a CTA holds 2^(14-G) independent tiles.
// The round structure is compile-time: the first round loads straight from global
// memory into registers, the last round stores straight back, and only the rounds
// in between go through shared memory, where the swizzled address is one XOR with
// a constant (S is linear over GF(2); a round's own bits are disjoint from the
// others). Middle rounds map warp lanes onto 5 tile bits whose bank images under
// S are independent, so every shared-memory access is conflict free.
// CTA order: contiguous passes run the same tile position of all columns back to
// back (their twiddles are then L2 hits); strided passes run the 2^(N-hi) copies of
// an extension read back to back (the coefficient tile is then an L2 hit).
// ---------------------------------------------------------------------------
constexpr int TT = 14;  // tile = 2^14 elements; a thread owns 2^E of them (E = 5 or 6)

__host__ __device__ constexpr uint32_t swz_c(uint32_t j) { return j ^ (((j >> 5) ^ (j >> 10)) & 31u); }

template <int G, bool INV, int R, int E>
struct RoundT {
    static constexpr int NR = (G + E - 1) / E;
    // balanced split of the G bits into NR rounds
    static constexpr int before(int r) { return r == 0 ? 0 : before(r - 1) + (G - before(r - 1) + (NR - r)) / (NR - r + 1); }
    static constexpr int RB = before(R + 1) - before(R);
    static constexpr int A = INV ? before(R) : G - before(R + 1);  // first owned layer (row) bit
};

// Bank-bit image of tile bit b under S.
__host__ __device__ constexpr uint32_t bank_vec(int b) {
    return (b < 5 ? 1u << b : 0u) ^ (b >= 5 && b < 10 ? 1u << (b - 5) : 0u) ^ (b >= 10 && b < 15 ? 1u << (b - 10) : 0u);
}

struct BitMap { int pos[TT]; };

// Positions (tile bits) of the thread-index bits of a round owning [OA, OA+RB):
// lanes first (the lowest other bits, or for middle rounds the lowest bits with
// independent bank images), then the remaining other bits in increasing order.
__host__ __device__ constexpr BitMap make_map(int OA, int RB, bool pick_lanes) {
    BitMap m{};
    int other[TT] = {};
    int n = 0;
    for (int b = 0; b < TT; b++)
        if (b < OA || b >= OA + RB) other[n++] = b;
    bool used[TT] = {};
    int k = 0;
    if (pick_lanes) {
        uint32_t basis[5] = {0, 0, 0, 0, 0};
        int nb = 0;
        for (int i = 0; i < n && k < 5; i++) {
            uint32_t v = bank_vec(other[i]);
            for (int t = 0; t < nb; t++)
                if ((v ^ basis[t]) < v) v ^= basis[t];
            if (v) {
                basis[nb++] = v;
                // keep the basis sorted by leading bit for the reduction above
                for (int t = nb - 1; t > 0 && basis[t] > basis[t - 1]; t--) {
                    uint32_t tmp = basis[t]; basis[t] = basis[t - 1]; basis[t - 1] = tmp;
                }
                m.pos[k++] = other[i];
                used[i] = true;
            }
        }
    }
    for (int i = 0; i < n; i++)
        if (!used[i]) m.pos[k++] = other[i];
    return m;
}

template <int N_BITS>
__device__ __forceinline__ uint32_t deposit(uint32_t x, const BitMap &m) {
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < N_BITS; i++) r |= ((x >> i) & 1u) << m.pos[i];
    return r;
}

struct GeoT {
    const FftLaunch *p;
    uint32_t tiles_log, low_fixed, n_high, n_cols;
};

template <int G, int C>
__device__ __forceinline__ void tile_locate(const GeoT &geo, uint32_t jb, uint32_t &col, uint32_t &gidx) {
    constexpr int SLOT_BITS = TT - C - G;
    const uint32_t tile_id = (blockIdx.x << SLOT_BITS) | (jb >> (C + G));
    const uint32_t jl = jb & ((1u << (C + G)) - 1u);
    if constexpr (C == 0) {
        // contiguous pass: tile position major, column minor
        const uint32_t T = tile_id / geo.n_cols;
        col = tile_id - T * geo.n_cols;
        gidx = (T << G) | jl;
    } else {
        col = tile_id >> geo.tiles_log;
        const uint32_t t = tile_id & ((1u << geo.tiles_log) - 1u);
        const uint32_t th = t & ((1u << geo.n_high) - 1u), tl = t >> geo.n_high;
        gidx = (tl << C) | (th << geo.p->hi) | (jl & ((1u << C) - 1u)) | ((jl >> C) << geo.p->lo);
    }
}

// The butterflies of one layer (bit u of the round) on one group of 2^RB registers.
template <int C, int A, int RB, bool INV, int U>
__device__ __forceinline__ void layer_butterflies(uint32_t (&v)[1 << RB], const FftLaunch &p, uint32_t gb,
                                                  uint32_t sh) {
    constexpr int RR = 1 << RB;
    constexpr int NQ = RR >> (U + 1);  // twiddles of this layer: consecutive and aligned to NQ
    constexpr bool CIRCLE = (C == 0 && A + U == 0);
    const uint32_t k = sh + U;
    const uint32_t hb = gb >> (k + 1);
    uint32_t tws[NQ];
    if constexpr (CIRCLE) {
#pragma unroll
        for (int q = 0; q < NQ; q++) tws[q] = twiddle2(p.tw, p.N, 0, hb + q);
    } else {
        const uint32_t *tk = p.tw + ((1u << (p.N - 1)) - (1u << (p.N - k))) + hb;
        if constexpr (NQ >= 4) {
#pragma unroll
            for (int q = 0; q < NQ; q += 4) {
                uint4 t = __ldg(reinterpret_cast<const uint4 *>(tk + q));
                tws[q] = t.x << 1; tws[q + 1] = t.y << 1; tws[q + 2] = t.z << 1; tws[q + 3] = t.w << 1;
            }
        } else if constexpr (NQ == 2) {
            uint2 t = __ldg(reinterpret_cast<const uint2 *>(tk));
            tws[0] = t.x << 1;
            tws[1] = t.y << 1;
        } else {
            tws[0] = __ldg(tk) << 1;
        }
    }
#pragma unroll
    for (int q = 0; q < NQ; q++) {
#pragma unroll
        for (int l = 0; l < (1 << U); l++) {
            const int m0 = (q << (U + 1)) | l;
            butterfly<INV>(v[m0], v[m0 | (1 << U)], tws[q]);
        }
    }
}

// All layers of one round on one group: evaluate runs them top-down, interpolate
// bottom-up. gb is the global index of the group's first element and sh the
// global bit of the round's first layer.
template <int C, int A, int RB, bool INV, int... Us>
__device__ __forceinline__ void round_butterflies_seq(uint32_t (&v)[1 << RB], const FftLaunch &p, uint32_t gb,
                                                      uint32_t sh, std::integer_sequence<int, Us...>) {
    (layer_butterflies<C, A, RB, INV, INV ? Us : RB - 1 - Us>(v, p, gb, sh), ...);
}

template <int C, int A, int RB, bool INV>
__device__ __forceinline__ void round_butterflies(uint32_t (&v)[1 << RB], const FftLaunch &p, uint32_t gb,
                                                  uint32_t sh) {
    round_butterflies_seq<C, A, RB, INV>(v, p, gb, sh, std::make_integer_sequence<int, RB>{});
}

template <int C, int A, int RB, bool INV>
__device__ __forceinline__ void store_global(uint32_t (&v)[1 << RB], const FftLaunch &p, uint32_t *__restrict__ dst,
                                             uint32_t gb, uint32_t sh) {
    constexpr int RR = 1 << RB;
    if (INV && p.scale2) {
#pragma unroll
        for (int m = 0; m < RR; m++) v[m] = m31_mul2(v[m], p.scale2);
    }
    if constexpr (C == 0 && A == 0 && RR >= 4) {
#pragma unroll
        for (int m = 0; m < RR; m += 4)
            *reinterpret_cast<uint4 *>(dst + gb + m) = make_uint4(v[m], v[m + 1], v[m + 2], v[m + 3]);
    } else {
#pragma unroll
        for (int m = 0; m < RR; m++) dst[gb + ((uint32_t)m << sh)] = v[m];
    }
}

template <int G, int C, bool INV, int R, int E>
__device__ __forceinline__ void roundT(uint32_t *sm, const GeoT &geo) {
    using RI = RoundT<G, INV, R, E>;
    constexpr int RB = RI::RB, A = RI::A, OA = C + A, RR = 1 << RB, GROUPS = 1 << (E - RB), W = TT - E;
    constexpr bool FIRST = R == 0, LAST = R == RI::NR - 1;
    constexpr int XBITS = TT - RB;
    constexpr BitMap M = make_map(OA, RB, !FIRST && !LAST);
    const FftLaunch &p = *geo.p;
    const uint32_t lo = (C == 0) ? 0u : p.lo;
    const uint32_t sh = lo + A;  // global bit of the round's first owned bit
    const uint32_t jt = deposit<W>(threadIdx.x, M);
    if constexpr (FIRST) {
        // Issue every global load of the round before the first butterfly.
        uint32_t v[GROUPS][RR];
        uint32_t gbs[GROUPS], cols[GROUPS];
#pragma unroll
        for (int grp = 0; grp < GROUPS; grp++) {
            const uint32_t jb = jt | deposit<XBITS>((uint32_t)grp << W, M);
            tile_locate<G, C>(geo, jb, cols[grp], gbs[grp]);
            const uint32_t *__restrict__ src = fft_col(p, cols[grp]).src;
            const uint32_t base = gbs[grp] & p.src_mask;
            if constexpr (C == 0 && A == 0 && RR >= 4) {
#pragma unroll
                for (int m = 0; m < RR; m += 4) {
                    uint4 t = __ldg(reinterpret_cast<const uint4 *>(src + base + m));
                    v[grp][m] = t.x; v[grp][m + 1] = t.y; v[grp][m + 2] = t.z; v[grp][m + 3] = t.w;
                }
            } else {
#pragma unroll
                for (int m = 0; m < RR; m++) v[grp][m] = __ldg(src + base + ((uint32_t)m << sh));
            }
        }
#pragma unroll
        for (int grp = 0; grp < GROUPS; grp++) {
            round_butterflies<C, A, RB, INV>(v[grp], p, gbs[grp], sh);
            if constexpr (LAST) {
                store_global<C, A, RB, INV>(v[grp], p, fft_col(p, cols[grp]).dst, gbs[grp], sh);
            } else {
                const uint32_t sj = swz_c(jt | deposit<XBITS>((uint32_t)grp << W, M));
#pragma unroll
                for (int m = 0; m < RR; m++) sm[sj ^ swz_c((uint32_t)m << OA)] = v[grp][m];
            }
        }
    } else {
#pragma unroll 1
        for (int grp = 0; grp < GROUPS; grp++) {
            const uint32_t jb = jt | deposit<XBITS>((uint32_t)grp << W, M);
            uint32_t col, gb;
            tile_locate<G, C>(geo, jb, col, gb);
            uint32_t v[RR];
            const uint32_t sj = swz_c(jb);
#pragma unroll
            for (int m = 0; m < RR; m++) v[m] = sm[sj ^ swz_c((uint32_t)m << OA)];
            round_butterflies<C, A, RB, INV>(v, p, gb, sh);
            if constexpr (LAST) {
                store_global<C, A, RB, INV>(v, p, fft_col(p, col).dst, gb, sh);
            } else {
#pragma unroll
                for (int m = 0; m < RR; m++) sm[sj ^ swz_c((uint32_t)m << OA)] = v[m];
            }
        }
    }
}

template <int G, int C, bool INV, int E, int... Rs>
__device__ __forceinline__ void roundsT(uint32_t *sm, const GeoT &geo, std::integer_sequence<int, Rs...>) {
    (
        [&] {
            roundT<G, C, INV, Rs, E>(sm, geo);
            if constexpr (Rs + 1 < RoundT<G, INV, 0, E>::NR) __syncthreads();
        }(),
        ...);
}

// 2^6 elements a thread: three CTAs per SM (at most 80 registers a thread, 192 KB of
// shared memory), measured 2292 vs 2231 columns/s at log 24 against two CTAs per SM
// with 112-128 registers, and 2132 with four CTAs per SM (64 registers). 2^5 elements
// a thread (512 threads): two CTAs per SM (64 registers; at three it spills).
template <int G, int C, bool INV, int E>
__global__ void __launch_bounds__(1 << (TT - E), E == 6 ? 3 : 2) fftT_kernel(const __grid_constant__ FftLaunch p, uint32_t n_cols) {
    extern __shared__ uint32_t sm[];
    GeoT geo;
    geo.p = &p;
    geo.tiles_log = p.N - (C + G);
    geo.low_fixed = (C == 0) ? 0u : p.lo - C;
    geo.n_high = p.N - p.hi;
    geo.n_cols = n_cols;
    roundsT<G, C, INV, E>(sm, geo, std::make_integer_sequence<int, RoundT<G, INV, 0, E>::NR>{});
}

template <int G, int C, bool INV, int E>
int launchT_e(const FftLaunch &p, uint32_t n_cols, cudaStream_t st) {
    constexpr int NR = RoundT<G, INV, 0, E>::NR;
    const size_t smem = NR > 1 ? (sizeof(uint32_t) << TT) : 0;
    auto kern = fftT_kernel<G, C, INV, E>;
    static std::atomic<uint64_t> attr_set{0};
    int rc = once_per_device(attr_set, [&] {
        STWO_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(sizeof(uint32_t) << TT)));
        return (int)STWO_OK;
    });
    if (rc) return rc;
    const uint64_t tiles = (uint64_t)n_cols << (p.N - C - G);
    const uint64_t per_cta = 1ull << (TT - C - G);
    STWO_REQUIRE(tiles % per_cta == 0, STWO_ERR_UNSUPPORTED_SIZE, "fft tile packing");
    STWO_REQUIRE(tiles < (1ull << 32), STWO_ERR_UNSUPPORTED_SIZE, "fft launch of %llu tiles", (unsigned long long)tiles);
    const uint64_t blocks = tiles / per_cta;
    kern<<<(unsigned)blocks, 1 << (TT - E), smem, st>>>(p, n_cols);
    STWO_LAUNCH_CHECK("fftT_kernel");
    return STWO_OK;
}

// Elements per thread, 2^6 (256 threads per CTA) or 2^5 (512 threads): a tunable per
// pass kind and domain size (stwo_autotune); 2^6 by default, measured faster at log 24
// (2222 vs 2125 columns/s). STWO_FFT_EPT_LOG=5 sets every pass kind to 2^5.
inline int fft_ept_log(bool contiguous, uint32_t N) {
    static const int forced = [] {
        const char *e = getenv("STWO_FFT_EPT_LOG");
        return e ? atoi(e) : 0;
    }();
    if (forced == 5 || forced == 6) return forced;
    return tunable(!contiguous ? TUNE_FFT_EPT_STRIDED : N <= 20 ? TUNE_FFT_EPT_CONTIG_SMALL : TUNE_FFT_EPT_CONTIG_LARGE);
}

template <int G, int C, bool INV>
int launchT_t(const FftLaunch &p, uint32_t n_cols, cudaStream_t st) {
    return fft_ept_log(C == 0, p.N) == 5 ? launchT_e<G, C, INV, 5>(p, n_cols, st) : launchT_e<G, C, INV, 6>(p, n_cols, st);
}

// Dispatch over (G, C): contiguous passes G = 11..14 (C = 0), strided passes
// G = 1..10 with C = 14 - G.
template <bool INV>
int launchT(const FftLaunch &p, uint32_t n_cols, uint32_t G, uint32_t C, cudaStream_t st) {
    if (C == 0) {
        switch (G) {
        case 11: return launchT_t<11, 0, INV>(p, n_cols, st);
        case 12: return launchT_t<12, 0, INV>(p, n_cols, st);
        case 13: return launchT_t<13, 0, INV>(p, n_cols, st);
        case 14: return launchT_t<14, 0, INV>(p, n_cols, st);
        default: break;
        }
    } else if (C + G == TT) {
        switch (G) {
        case 1: return launchT_t<1, 13, INV>(p, n_cols, st);
        case 2: return launchT_t<2, 12, INV>(p, n_cols, st);
        case 3: return launchT_t<3, 11, INV>(p, n_cols, st);
        case 4: return launchT_t<4, 10, INV>(p, n_cols, st);
        case 5: return launchT_t<5, 9, INV>(p, n_cols, st);
        case 6: return launchT_t<6, 8, INV>(p, n_cols, st);
        case 7: return launchT_t<7, 7, INV>(p, n_cols, st);
        case 8: return launchT_t<8, 6, INV>(p, n_cols, st);
        case 9: return launchT_t<9, 5, INV>(p, n_cols, st);
        case 10: return launchT_t<10, 4, INV>(p, n_cols, st);
        default: break;
        }
    }
    return set_error(STWO_ERR_UNSUPPORTED_SIZE, "no specialised fft pass for G=%u C=%u", G, C);
}

// Transforms of 2 and 4 elements. The circle twiddle is y of the half coset's
// first point, which the tree does not store for these sizes; it is derived from
// the first line layer of the next larger domain ([x', y'] with y = 2 x' y'), so
// the tree must cover at least an 8-element domain.
struct TinyLaunch {
    FftColumn cols[MAX_COLS_PER_LAUNCH];
    uint32_t N;
    uint32_t t_x, t_y;   // (i)twiddles: x and y of the first half-coset point (or inverses)
    uint32_t scale;
};

template <bool INV>
__global__ void fft_tiny_kernel(const __grid_constant__ TinyLaunch p) {
    uint32_t col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= gridDim.x * blockDim.x) return;
    if (p.cols[col].src == nullptr) return;
    const uint32_t *src = p.cols[col].src;
    uint32_t *dst = p.cols[col].dst;
    uint32_t y2 = p.t_y << 1, ny2 = m31_neg(p.t_y) << 1, x2 = p.t_x << 1;
    if (p.N == 1) {
        uint32_t a = src[0], b = src[1];
        butterfly<INV>(a, b, y2);
        if (INV) { a = m31_mul(a, p.scale); b = m31_mul(b, p.scale); }
        dst[0] = a;
        dst[1] = b;
    } else {
        uint32_t v0 = src[0], v1 = src[1], v2 = src[2], v3 = src[3];
        if (INV) {
            butterfly<true>(v0, v1, y2);
            butterfly<true>(v2, v3, ny2);
            butterfly<true>(v0, v2, x2);
            butterfly<true>(v1, v3, x2);
            v0 = m31_mul(v0, p.scale); v1 = m31_mul(v1, p.scale);
            v2 = m31_mul(v2, p.scale); v3 = m31_mul(v3, p.scale);
        } else {
            butterfly<false>(v0, v2, x2);
            butterfly<false>(v1, v3, x2);
            butterfly<false>(v0, v1, y2);
            butterfly<false>(v2, v3, ny2);
        }
        dst[0] = v0; dst[1] = v1; dst[2] = v2; dst[3] = v3;
    }
}

template <int LOG_E, bool INV>
int launch_pass_t(const FftLaunch &p, uint32_t n_cols, cudaStream_t st) {
    const uint32_t threads = 1u << (p.tile_log - LOG_E);
    const size_t smem = sizeof(uint32_t) << p.tile_log;
    auto kern = fft_pass_kernel<LOG_E, INV>;
    static std::atomic<uint64_t> attr_set{0};
    int rc = once_per_device(attr_set, [&] {
        STWO_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)(sizeof(uint32_t) << MAX_TILE_LOG)));
        return (int)STWO_OK;
    });
    if (rc) return rc;
    const uint64_t blocks = (uint64_t)n_cols << (p.N - p.tile_log);
    STWO_REQUIRE(blocks < (1ull << 31), STWO_ERR_UNSUPPORTED_SIZE, "fft grid too large");
    kern<<<(unsigned)blocks, threads, smem, st>>>(p);
    STWO_LAUNCH_CHECK("fft_pass_kernel");
    return STWO_OK;
}

int launch_pass(const FftLaunch &p, uint32_t n_cols, bool inv, cudaStream_t st) {
    // Threads per tile: up to 512, at least 4 elements per thread.
    uint32_t W = std::min<uint32_t>(MAX_THREADS_LOG, p.tile_log >= 2 ? p.tile_log - 2 : 0);
    int log_e = (int)(p.tile_log - W);
    switch (log_e) {
#define STWO_FFT_CASE(E) \
    case E: return inv ? launch_pass_t<E, true>(p, n_cols, st) : launch_pass_t<E, false>(p, n_cols, st);
        STWO_FFT_CASE(2)
        STWO_FFT_CASE(3)
        STWO_FFT_CASE(4)
        STWO_FFT_CASE(5)
        STWO_FFT_CASE(6)
#undef STWO_FFT_CASE
    default:
        return set_error(STWO_ERR_UNSUPPORTED_SIZE, "fft tile of 2^%u elements unsupported", p.tile_log);
    }
}

struct PassSpec { uint32_t lo, hi, c, tile_log; };

// Layer ranges for a transform whose non-trivial layers are [0, L): a bottom
// contiguous pass of up to 14 layers and strided passes above, each over 2^14-element
// tiles (rows of >= 16 contiguous words). The radix split of the upper layers — how
// many a strided pass takes at most, 4..10, spread evenly over the passes — is a
// tunable (fft_max_strided_layers, measured by stwo_autotune): fewer layers a pass
// means wider contiguous tile rows but one more round trip through HBM.
std::vector<PassSpec> plan_passes(uint32_t L) {
    std::vector<PassSpec> v;
    if (L <= (uint32_t)TT) {
        v.push_back({0, L, 0, L});
        return v;
    }
    v.push_back({0, (uint32_t)TT, 0, (uint32_t)TT});
    uint32_t lo = TT;
    const uint32_t max_g = (uint32_t)std::min(TT - 4, std::max(4, tunable(TUNE_FFT_MAX_STRIDED)));
    while (lo < L) {
        uint32_t rem = L - lo;
        uint32_t chunks = (rem + max_g - 1) / max_g;
        uint32_t g = (rem + chunks - 1) / chunks;
        v.push_back({lo, lo + g, TT - g, (uint32_t)TT});
        lo += g;
    }
    return v;
}

// The integer ceiling of every FFT pass: the rate of the passes' own forward butterfly
// (butterfly<false>: an m31_mul2 product, a sum and a difference) with operands in
// registers only. Each thread keeps 16 independent pairs and feeds every butterfly's
// outputs into its next one; the XOR of the final values goes to sink so that nothing
// is optimised away.
constexpr int PROBE_PAIRS = 16;
constexpr int PROBE_THREADS = 256;

__global__ void __launch_bounds__(PROBE_THREADS) butterfly_probe_kernel(uint32_t iters, uint32_t *sink) {
    const uint32_t tid = blockIdx.x * PROBE_THREADS + threadIdx.x;
    uint32_t a[PROBE_PAIRS], b[PROBE_PAIRS], t2[PROBE_PAIRS];
#pragma unroll
    for (int k = 0; k < PROBE_PAIRS; k++) {
        a[k] = (tid * 2654435761u + (uint32_t)k) & 0x3fffffffu;
        b[k] = (tid * 40503u + 7919u * (uint32_t)k) & 0x3fffffffu;
        t2[k] = ((tid ^ (0x9e3779b9u * (uint32_t)(k + 1))) & 0x3fffffffu) << 1;
    }
    for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < PROBE_PAIRS; k++) butterfly<false>(a[k], b[k], t2[k]);
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < PROBE_PAIRS; k++) x ^= a[k] ^ b[k];
    sink[tid] = x;
}

}  // namespace

int butterfly_probe_async(uint32_t iters, uint32_t *sink, uint64_t sink_words, uint64_t *butterflies,
                          cudaStream_t st) {
    STWO_REQUIRE(butterflies && sink, STWO_ERR_INVALID_ARGUMENT, "null argument");
    const uint64_t blocks = (uint64_t)device_sm_count() * (2048 / PROBE_THREADS);
    const uint64_t threads = blocks * PROBE_THREADS;
    STWO_REQUIRE(sink_words >= threads, STWO_ERR_INVALID_ARGUMENT, "the probe needs a sink of %llu words",
                 (unsigned long long)threads);
    butterfly_probe_kernel<<<(unsigned)blocks, PROBE_THREADS, 0, st>>>(iters, sink);
    STWO_LAUNCH_CHECK("butterfly_probe_kernel");
    *butterflies = threads * PROBE_PAIRS * (uint64_t)iters;
    return STWO_OK;
}

// (x, y) of the first point of the half coset of a 2^N-point circle domain, N <= 2,
// as twiddles (inv = false) or inverse twiddles (inv = true). The tree does not
// store y for these sizes (CpuBackend reads it from the domain itself), so it is
// derived from the first line layer of the 8-point domain, which holds the pair
// [x8, y8] of that domain's first point P8 (the [x, y] pairing the circle
// twiddles rely on, poly/utils.cu:3-14): P4 = P8^2 = (2 x8^2 - 1, 2 x8 y8) and
// P2 = P4^2. `suffix_end` points one past the 2^N domain's suffix of the tree;
// the 8-point domain's first line layer is the two entries 4 before it.
int small_circle_point(const uint32_t *suffix_end, uint64_t avail, uint32_t N, bool inv, uint32_t *tx,
                       uint32_t *ty, cudaStream_t st) {
    STWO_REQUIRE(avail >= 4, STWO_ERR_UNSUPPORTED_SIZE,
                 "a 2^%u-point circle domain needs a twiddle tree that also covers the 8-point domain", N);
    uint32_t l8[2];
    void *stage = nullptr;
    int wrc = host_stage(sizeof(l8), &stage);
    if (wrc) return wrc;
    STWO_CUDA_TRY(cudaMemcpyAsync(stage, suffix_end - 4, sizeof(l8), cudaMemcpyDeviceToHost, st));
    wrc = wait_stream(st);
    if (wrc) return wrc;
    memcpy(l8, stage, sizeof(l8));
    uint32_t x8 = inv ? m31_inv(l8[0]) : l8[0];
    uint32_t y8 = inv ? m31_inv(l8[1]) : l8[1];
    uint32_t x = m31_sub(m31_add(m31_sqr(x8), m31_sqr(x8)), 1), y = m31_mul(m31_add(x8, x8), y8);
    if (N == 1) {
        uint32_t nx = m31_sub(m31_add(m31_sqr(x), m31_sqr(x)), 1), ny = m31_mul(m31_add(x, x), y);
        x = nx;
        y = ny;
    }
    *tx = inv ? m31_inv(x) : x;
    *ty = inv ? m31_inv(y) : y;
    return STWO_OK;
}

// Runs a transform over n_cols columns of one size. src[i] may equal dst[i]
// (in place); for an extension read (L < N) src holds 2^L coefficients.
// dev_table, when given, holds the same (srcs[i], dsts[i]) pairs in device memory; it
// serves launches of more than 64 columns (the prover's tables travel in its uploaded
// image, so its launch sequence stays capturable). Without it such launches stage a
// table through the library's pool.
int fft_columns_tab(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                    const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st, const void *dev_table) {
    if (n_cols == 0) return STWO_OK;
    STWO_REQUIRE(N >= 1 && N <= 30 && L <= N, STWO_ERR_UNSUPPORTED_SIZE, "fft log size %u unsupported", N);
    STWO_REQUIRE(tree != nullptr, STWO_ERR_INVALID_ARGUMENT, "null twiddle tree");
    if (N <= 2) {
        STWO_REQUIRE(L == N, STWO_ERR_UNSUPPORTED_SIZE, "extension to a 2^%u domain unsupported", N);
        TinyLaunch t{};
        t.N = N;
        int rc = small_circle_point(tree + tree_size, tree_size, N, inv, &t.t_x, &t.t_y, st);
        if (rc) return rc;
        t.scale = m31_inv_pow2(N);
        for (uint32_t base = 0; base < n_cols; base += MAX_COLS_PER_LAUNCH) {
            uint32_t cnt = std::min<uint32_t>(MAX_COLS_PER_LAUNCH, n_cols - base);
            for (uint32_t i = 0; i < MAX_COLS_PER_LAUNCH; i++)
                t.cols[i] = i < cnt ? FftColumn{srcs[base + i], dsts[base + i]} : FftColumn{nullptr, nullptr};
            if (inv) fft_tiny_kernel<true><<<1, cnt, 0, st>>>(t);
            else fft_tiny_kernel<false><<<1, cnt, 0, st>>>(t);
            STWO_LAUNCH_CHECK("fft_tiny_kernel");
        }
        return STWO_OK;
    }
    STWO_REQUIRE(tree_size >= (1ull << (N - 1)), STWO_ERR_INVALID_ARGUMENT,
                 "twiddle tree of %llu entries is smaller than the 2^%u domain's half coset",
                 (unsigned long long)tree_size, N);
    STWO_REQUIRE(L >= 2, STWO_ERR_UNSUPPORTED_SIZE, "extension from fewer than 4 coefficients unsupported");
    for (uint32_t i = 0; i < n_cols; i++) {
        STWO_REQUIRE(srcs[i] && dsts[i], STWO_ERR_INVALID_ARGUMENT, "null column pointer");
        STWO_REQUIRE(((uintptr_t)srcs[i] & 15) == 0 && ((uintptr_t)dsts[i] & 15) == 0, STWO_ERR_INVALID_ARGUMENT,
                     "column pointers must be 16-byte aligned");
    }
    FftLaunch p{};
    p.tw = tree + (tree_size - (1ull << (N - 1)));
    p.N = N;
    // More than 64 columns: every pass is one launch over a device table.
    const FftColumn *table = nullptr;
    void *staged = nullptr;
    if (n_cols > (uint32_t)MAX_COLS_PER_LAUNCH) {
        if (dev_table) {
            table = static_cast<const FftColumn *>(dev_table);
        } else {
            std::vector<FftColumn> h(n_cols);
            for (uint32_t i = 0; i < n_cols; i++) h[i] = FftColumn{srcs[i], dsts[i]};
            int arc = pool_alloc(&staged, sizeof(FftColumn) * n_cols, st);
            if (arc) return arc;
            // from pageable memory: the copy has read h when it returns
            STWO_CUDA_TRY(cudaMemcpyAsync(staged, h.data(), sizeof(FftColumn) * n_cols, cudaMemcpyHostToDevice, st));
            table = static_cast<const FftColumn *>(staged);
        }
    }
    struct FreeStaged {
        void *p;
        cudaStream_t st;
        ~FreeStaged() {
            if (p) cudaFreeAsync(p, st);
        }
    } free_staged{staged, st};
    std::vector<PassSpec> passes = plan_passes(L);
    if (!inv) std::reverse(passes.begin(), passes.end());
    for (size_t pi = 0; pi < passes.size(); pi++) {
        const PassSpec &ps = passes[pi];
        p.lo = ps.lo;
        p.hi = ps.hi;
        p.c = ps.c;
        p.tile_log = ps.tile_log;
        bool first = pi == 0, last = pi + 1 == passes.size();
        p.src_mask = (first && L < N) ? ((1u << L) - 1u) : 0xffffffffu;
        p.scale2 = (inv && last) ? (m31_inv_pow2(N) << 1) : 0u;
        const uint32_t per_launch = table ? n_cols : (uint32_t)MAX_COLS_PER_LAUNCH;
        p.table = table;
        p.src_from_dst = first ? 0u : 1u;
        for (uint32_t base = 0; base < n_cols; base += per_launch) {
            uint32_t cnt = std::min<uint32_t>(per_launch, n_cols - base);
            if (!table)
                for (uint32_t i = 0; i < cnt; i++)
                    p.cols[i] = FftColumn{first ? srcs[base + i] : dsts[base + i], dsts[base + i]};
            const uint32_t G = ps.hi - ps.lo;
            // Specialised 2^15 tiles: strided passes, or contiguous passes of >= 11 layers whose
            // tiles pack evenly into CTAs.
            // (vector twiddle loads need the tree suffix 16-byte aligned)
            const bool spec = ((uintptr_t)p.tw & 15) == 0 &&
                              ((ps.c > 0 && ps.tile_log == (uint32_t)TT) ||
                               (ps.c == 0 && G >= 11 && G <= (uint32_t)TT &&
                                ((uint64_t)cnt << (N - G)) % (1ull << (TT - G)) == 0));
            int rc = spec ? (inv ? launchT<true>(p, cnt, G, ps.c, st) : launchT<false>(p, cnt, G, ps.c, st))
                          : launch_pass(p, cnt, inv, st);
            if (rc) return rc;
        }
    }
    return STWO_OK;
}

int fft_columns(const uint32_t *const *srcs, uint32_t *const *dsts, uint32_t n_cols, uint32_t N, uint32_t L,
                const uint32_t *tree, uint64_t tree_size, bool inv, cudaStream_t st) {
    return fft_columns_tab(srcs, dsts, n_cols, N, L, tree, tree_size, inv, st, nullptr);
}

}  // namespace stwo
