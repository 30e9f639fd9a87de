/*
 * SIMD CPU restatement of the prover's heavy functions — BASELINE ONLY.
 *
 * A stand-in for stwo's SimdBackend (stwo-prover @ ce5b975, Rust, absent from this
 * image): the functions the oracle prover (stwo_oracle_prover.c) spends its time in,
 * rewritten with vector lanes (16 x u32 with AVX-512, 8 with AVX2) and OpenMP
 * threads. Every function returns exactly the scalar oracle's values
 * (stwo_oracle.c; tests/test_simd_baseline.py compares them), so the prover built
 * on them (libstwo_simd_*.so: the oracle prover's protocol code with these
 * functions in place of the scalar ones, oracle/simd_remap.h) writes the same proof
 * bytes. The benchmark times it as the reference CPU path; nothing on the product
 * path loads it.
 *
 * Methods (each a standard CPU technique, not the GPU kernels):
 *  - M31 products on lanes: 32x32->64-bit even/odd multiplies (vpmuludq), folded
 *    by x = (x & p) + (x >> 31) and one conditional subtraction;
 *  - circle FFT: the bottom 12 layers on 4096-element blocks held in L1, the upper
 *    layers one at a time across the column; layers whose butterfly pairs are at
 *    least a vector apart run on lanes (one twiddle a vector), the lowest ones in
 *    scalar code; whole columns per thread when a batch has enough of them;
 *  - Blake2s Merkle layers: one node per lane, 16 (or 8) nodes a compression;
 *  - DEEP quotients and the composition: 64-bit dot products on lanes over rows,
 *    the per-row denominators in scalar code;
 *  - OODS evaluation: 16-coefficient partial sums on lanes, then the fold;
 *  - twiddle trees by running point products and a Montgomery batch inverse.
 */
#include <immintrin.h>
#include <omp.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "stwo_oracle.h"

namespace {

constexpr uint32_t P = 0x7fffffffu;

#if defined(__AVX512F__)
constexpr int W = 16;
typedef uint32_t V __attribute__((vector_size(64)));
typedef uint64_t V64 __attribute__((vector_size(64)));
inline V64 mul_even(V64 a, V64 b) { return (V64)_mm512_mul_epu32((__m512i)a, (__m512i)b); }
#else
constexpr int W = 8;
typedef uint32_t V __attribute__((vector_size(32)));
typedef uint64_t V64 __attribute__((vector_size(32)));
inline V64 mul_even(V64 a, V64 b) { return (V64)_mm256_mul_epu32((__m256i)a, (__m256i)b); }
#endif
constexpr int LOGW = W == 16 ? 4 : 3;

inline V splat(uint32_t x) { return V{} + x; }
inline V64 splat64(uint64_t x) { return V64{} + x; }
inline V vload(const uint32_t *p) { V v; memcpy(&v, p, sizeof(V)); return v; }
inline void vstore(uint32_t *p, V v) { memcpy(p, &v, sizeof(V)); }
inline V vmin(V a, V b) { return a < b ? a : b; }
inline V vadd(V a, V b) { V s = a + b; return vmin(s, s - P); }
inline V vsub(V a, V b) { V d = a - b; return vmin(d, d + P); }
// Fold of 64-bit lanes below 2^62 to 32 bits: (x & p) + (x >> 31) < 2^32.
inline V64 fold(V64 x) { return (x & (uint64_t)P) + (x >> 31); }
inline V vmul(V a, V b) {
    const V64 pe = mul_even((V64)a, (V64)b), po = mul_even((V64)a >> 32, (V64)b >> 32);
    const V r = (V)(fold(pe) | (fold(po) << 32));
    return vmin(r, r - P);
}

// ---------------------------------------------------------------- scalar field
inline uint32_t m_add(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P ? s - P : s; }
inline uint32_t m_sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }
inline uint32_t m_neg(uint32_t a) { return a ? P - a : 0; }
inline uint32_t m_red64(uint64_t v) {
    uint64_t s = (v & P) + (v >> 31);
    s = (s & P) + (s >> 31);
    return s >= P ? (uint32_t)(s - P) : (uint32_t)s;
}
inline uint32_t m_mul(uint32_t a, uint32_t b) { return m_red64((uint64_t)a * b); }
uint32_t m_pow(uint32_t a, uint64_t e) {
    uint32_t r = 1;
    while (e) {
        if (e & 1) r = m_mul(r, a);
        a = m_mul(a, a);
        e >>= 1;
    }
    return r;
}
inline uint32_t m_inv(uint32_t a) { return m_pow(a, P - 2); }

inline cm31_t c_add(cm31_t x, cm31_t y) { return {m_add(x.a, y.a), m_add(x.b, y.b)}; }
inline cm31_t c_sub(cm31_t x, cm31_t y) { return {m_sub(x.a, y.a), m_sub(x.b, y.b)}; }
inline cm31_t c_mul(cm31_t x, cm31_t y) {
    return {m_sub(m_mul(x.a, y.a), m_mul(x.b, y.b)), m_add(m_mul(x.a, y.b), m_mul(x.b, y.a))};
}
inline qm31_t q_add(qm31_t x, qm31_t y) { return {c_add(x.a, y.a), c_add(x.b, y.b)}; }
inline qm31_t q_sub(qm31_t x, qm31_t y) { return {c_sub(x.a, y.a), c_sub(x.b, y.b)}; }
inline qm31_t q_mul(qm31_t x, qm31_t y) {
    const cm31_t ac = c_mul(x.a, y.a), bd = c_mul(x.b, y.b), ad = c_mul(x.a, y.b), bc = c_mul(x.b, y.a);
    const cm31_t rbd = {m_sub(m_add(bd.a, bd.a), bd.b), m_add(m_add(bd.b, bd.b), bd.a)};  // (2 + i) bd
    return {c_add(ac, rbd), c_add(ad, bc)};
}
inline qm31_t q_scale(qm31_t x, uint32_t s) {
    return {{m_mul(x.a.a, s), m_mul(x.a.b, s)}, {m_mul(x.b.a, s), m_mul(x.b.b, s)}};
}
inline qm31_t q_mul_cm31(qm31_t x, cm31_t s) { return {c_mul(x.a, s), c_mul(x.b, s)}; }
inline qm31_t q_zero() { return {{0, 0}, {0, 0}}; }

inline uint32_t bitrev(uint32_t i, uint32_t log) {
    uint32_t r = i;
    r = ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
    r = ((r >> 2) & 0x33333333u) | ((r & 0x33333333u) << 2);
    r = ((r >> 4) & 0x0f0f0f0fu) | ((r & 0x0f0f0f0fu) << 4);
    r = __builtin_bswap32(r);
    return log == 0 ? i : r >> (32 - log);
}

// G^idx for a 31-bit circle-group index as a product of three table entries:
// G^(idx mod 2^11), G^(2^11 (idx >> 11 mod 2^11)), G^(2^22 (idx >> 22)).
struct PointTables {
    std::vector<cpoint_t> t0, t1, t2;
    PointTables() : t0(2048), t1(2048), t2(512) {
        fill(t0, or_index_to_point(1));
        fill(t1, or_index_to_point(1u << 11));
        fill(t2, or_index_to_point(1u << 22));
    }
    static void fill(std::vector<cpoint_t> &t, cpoint_t step) {
        cpoint_t r = {1, 0};
        for (auto &e : t) {
            e = r;
            r = {m_sub(m_mul(r.x, step.x), m_mul(r.y, step.y)), m_add(m_mul(r.x, step.y), m_mul(r.y, step.x))};
        }
    }
    cpoint_t at(uint32_t idx) const;
};

inline cpoint_t pt_mul(cpoint_t p, cpoint_t q) {
    return {m_sub(m_mul(p.x, q.x), m_mul(p.y, q.y)), m_add(m_mul(p.x, q.y), m_mul(p.y, q.x))};
}
cpoint_t PointTables::at(uint32_t idx) const {
    idx &= P;
    return pt_mul(pt_mul(t0[idx & 2047u], t1[(idx >> 11) & 2047u]), t2[idx >> 22]);
}
// CircleDomain::at(i) of the domain with half coset hc: the half coset, then its
// conjugates (negated indices).
inline cpoint_t domain_point(const PointTables &pt, coset_t hc, uint64_t i) {
    const uint64_t half = 1ull << hc.log_size;
    if (i < half) return pt.at((uint32_t)(hc.initial_index + (uint64_t)hc.step_size * i));
    const uint32_t idx = (uint32_t)((hc.initial_index + (uint64_t)hc.step_size * (i - half)) & P);
    return pt.at((0x80000000u - idx) & P);
}
// ---------------------------------------------------------------- circle FFT
constexpr uint32_t BLOCK_LOG = 12;

// Line-layer twiddles of a size-2^L domain: sl[k] (k = 1..L-1), 2^(L-1-k) entries.
void twiddle_slices(const uint32_t *tree, size_t tree_size, uint32_t L, const uint32_t **sl) {
    const uint32_t *suffix = tree + (tree_size - ((size_t)1 << (L - 1)));
    size_t off = 0;
    for (uint32_t k = 1; k < L; k++) {
        sl[k] = suffix + off;
        off += (size_t)1 << (L - 1 - k);
    }
}
// Circle-layer twiddle of pair h: [y, -y, -x, x] of the first line layer's pair h / 4.
inline uint32_t circle_tw(const uint32_t *lt0, size_t h) {
    const size_t k = h >> 2;
    switch (h & 3) {
    case 0: return lt0[2 * k + 1];
    case 1: return m_neg(lt0[2 * k + 1]);
    case 2: return m_neg(lt0[2 * k]);
    default: return lt0[2 * k];
    }
}
inline uint32_t layer_tw(const uint32_t *const *sl, uint32_t k, size_t h) { return k == 0 ? circle_tw(sl[1], h) : sl[k][h]; }

// One layer k on elements [j0, j1) of v (j0, j1 multiples of 2^(k+1)).
template <bool INV>
void fft_layer_range(uint32_t *v, const uint32_t *const *sl, uint32_t k, size_t j0, size_t j1) {
    const size_t half = (size_t)1 << k;
    if (half >= (size_t)W) {
        for (size_t i0 = j0; i0 < j1; i0 += 2 * half) {
            const V t = splat(layer_tw(sl, k, i0 >> (k + 1)));
            uint32_t *a = v + i0, *b = v + i0 + half;
            for (size_t l = 0; l < half; l += W) {
                const V x = vload(a + l), y = vload(b + l);
                if (INV) {
                    vstore(a + l, vadd(x, y));
                    vstore(b + l, vmul(vsub(x, y), t));
                } else {
                    const V ty = vmul(y, t);
                    vstore(a + l, vadd(x, ty));
                    vstore(b + l, vsub(x, ty));
                }
            }
        }
    } else {
        for (size_t i0 = j0; i0 < j1; i0 += 2 * half) {
            const uint32_t t = layer_tw(sl, k, i0 >> (k + 1));
            for (size_t l = 0; l < half; l++) {
                const uint32_t x = v[i0 + l], y = v[i0 + l + half];
                if (INV) {
                    v[i0 + l] = m_add(x, y);
                    v[i0 + l + half] = m_mul(m_sub(x, y), t);
                } else {
                    const uint32_t ty = m_mul(y, t);
                    v[i0 + l] = m_add(x, ty);
                    v[i0 + l + half] = m_sub(x, ty);
                }
            }
        }
    }
}

// A whole transform of one column of 2^L (L >= 3) elements; `parallel`: split each
// step across the threads of the enclosing parallel region (every thread calls it).
template <bool INV>
void fft_column(uint32_t *v, uint32_t L, const uint32_t *tree, size_t tree_size, bool parallel) {
    const uint32_t *sl[32] = {};
    twiddle_slices(tree, tree_size, L, sl);
    const size_t n = (size_t)1 << L;
    const uint32_t kb = L < BLOCK_LOG ? L : BLOCK_LOG;
    const size_t blk = (size_t)1 << kb;
    auto bottom = [&]() {
        auto block = [&](size_t b0) {
            if (INV)
                for (uint32_t k = 0; k < kb; k++) fft_layer_range<INV>(v, sl, k, b0, b0 + blk);
            else
                for (int k = (int)kb - 1; k >= 0; k--) fft_layer_range<INV>(v, sl, (uint32_t)k, b0, b0 + blk);
        };
        if (parallel) {
#pragma omp for schedule(static)
            for (size_t b0 = 0; b0 < n; b0 += blk) block(b0);
        } else {
            for (size_t b0 = 0; b0 < n; b0 += blk) block(b0);
        }
    };
    auto top = [&](uint32_t k) {
        // chunks of 2^(k+1) elements (one twiddle group each), at least 8192 elements
        const size_t span = (size_t)2 << k, chunk = span < 8192 ? 8192 : span;
        if (parallel) {
#pragma omp for schedule(static)
            for (size_t j0 = 0; j0 < n; j0 += chunk) fft_layer_range<INV>(v, sl, k, j0, j0 + chunk);
        } else {
            fft_layer_range<INV>(v, sl, k, 0, n);
        }
    };
    if (INV) {
        bottom();
        for (uint32_t k = kb; k < L; k++) top(k);
        const uint32_t scale = m_inv(m_pow(2, L));
        const V s = splat(scale);
        if (n < (size_t)W) {  // shorter than a vector
            for (size_t i = 0; i < n; i++) v[i] = m_mul(v[i], scale);
        } else if (parallel) {
#pragma omp for schedule(static)
            for (size_t i = 0; i < n; i += W) vstore(v + i, vmul(vload(v + i), s));
        } else {
            for (size_t i = 0; i < n; i += W) vstore(v + i, vmul(vload(v + i), s));
        }
    } else {
        for (int k = (int)L - 1; k >= (int)kb; k--) top((uint32_t)k);
        bottom();
    }
}

}  // namespace

extern "C" {

int simd_interpolate(coset_t hc, m31_t *v, const m31_t *itw, size_t tree_size) {
    const uint32_t L = hc.log_size + 1;
    if (L < 3 || L - 1 > 30) return or_interpolate(hc, v, itw, tree_size);  // 2- and 4-point special cases
    if (tree_size < ((size_t)1 << (L - 1))) return -1;
    if (L >= 16) {
#pragma omp parallel
        fft_column<true>(v, L, itw, tree_size, true);
    } else {
        fft_column<true>(v, L, itw, tree_size, false);
    }
    return 0;
}

int simd_evaluate(coset_t hc, m31_t *v, const m31_t *tw, size_t tree_size) {
    const uint32_t L = hc.log_size + 1;
    if (L < 3 || L - 1 > 30) return or_evaluate(hc, v, tw, tree_size);
    if (tree_size < ((size_t)1 << (L - 1))) return -1;
    if (L >= 16) {
#pragma omp parallel
        fft_column<false>(v, L, tw, tree_size, true);
    } else {
        fft_column<false>(v, L, tw, tree_size, false);
    }
    return 0;
}

// Batches: whole columns per thread when there are at least as many columns as
// threads, else each column split across the threads.
void simd_interpolate_many(coset_t hc, m31_t *const *cols, size_t n_cols, const m31_t *itw, size_t tree_size) {
    const uint32_t L = hc.log_size + 1;
    if (L < 3) {
        for (size_t c = 0; c < n_cols; c++) or_interpolate(hc, cols[c], itw, tree_size);
        return;
    }
    if (n_cols >= (size_t)omp_get_max_threads()) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t c = 0; c < n_cols; c++) fft_column<true>(cols[c], L, itw, tree_size, false);
    } else {
        for (size_t c = 0; c < n_cols; c++) simd_interpolate(hc, cols[c], itw, tree_size);
    }
}

void simd_evaluate_many(coset_t hc, const m31_t *const *coeffs, size_t coeff_len, m31_t *const *out, size_t n_cols,
                        const m31_t *tw, size_t tree_size) {
    const uint32_t L = hc.log_size + 1;
    const size_t n = (size_t)1 << L;
    auto prep = [&](size_t c) {
        memcpy(out[c], coeffs[c], coeff_len * 4);
        memset(out[c] + coeff_len, 0, (n - coeff_len) * 4);
    };
    if (L < 3) {
        for (size_t c = 0; c < n_cols; c++) {
            prep(c);
            or_evaluate(hc, out[c], tw, tree_size);
        }
        return;
    }
    if (n_cols >= (size_t)omp_get_max_threads()) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t c = 0; c < n_cols; c++) {
            prep(c);
            fft_column<false>(out[c], L, tw, tree_size, false);
        }
    } else {
        for (size_t c = 0; c < n_cols; c++) {
            prep(c);
            simd_evaluate(hc, out[c], tw, tree_size);
        }
    }
}

// ---------------------------------------------------------------- twiddle trees
// Layer j of the tree: x of the j-th doubling of the root coset at bit-reversed
// positions, by running products of the coset's step from each chunk's first point.
void simd_precompute_twiddles(coset_t root, m31_t *tw, m31_t *itw) {
    const size_t size = (size_t)1 << root.log_size;
    size_t off = 0;
    coset_t c = root;
    for (uint32_t layer = 0; layer < root.log_size; layer++) {
        const size_t half = ((size_t)1 << c.log_size) / 2;
        const uint32_t hl = c.log_size - 1;
        const cpoint_t step = or_index_to_point(c.step_size);
        const size_t chunk = 4096;
#pragma omp parallel for schedule(static)
        for (size_t h0 = 0; h0 < half; h0 += chunk) {
            cpoint_t p = or_coset_at(c, h0);
            const size_t h1 = h0 + chunk < half ? h0 + chunk : half;
            for (size_t h = h0; h < h1; h++) {
                tw[off + bitrev((uint32_t)h, hl)] = p.x;
                p = pt_mul(p, step);
            }
        }
        off += half;
        c.initial_index = (c.initial_index * 2) & P;
        c.step_size = (c.step_size * 2) & P;
        c.log_size--;
    }
    tw[size - 1] = 1;
    if (!itw) return;
    // Montgomery's batch inverse per chunk. The FFT divides by these twiddles, so a
    // tree that can serve as one has no zero entry (and the pad is 1).
    const size_t chunk = 4096;
#pragma omp parallel for schedule(static)
    for (size_t i0 = 0; i0 < size; i0 += chunk) {
        const size_t i1 = i0 + chunk < size ? i0 + chunk : size;
        uint32_t acc = 1;
        for (size_t i = i0; i < i1; i++) {
            itw[i] = acc;
            acc = m_mul(acc, tw[i]);
        }
        uint32_t inv = m_inv(acc);
        for (size_t i = i1; i-- > i0;) {
            const uint32_t t = m_mul(inv, itw[i]);
            inv = m_mul(inv, tw[i]);
            itw[i] = t;
        }
    }
}

// ---------------------------------------------------------------- Blake2s Merkle
}  // extern "C"

namespace {

inline V rotr(V x, int c) { return (x >> c) | (x << (32 - c)); }

const uint8_t SIGMA[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0},
};
const uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                        0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

#define SG(a, b, c, d, x, y)     \
    a = a + b + (x);             \
    d = rotr(d ^ a, 16);         \
    c = c + d;                   \
    b = rotr(b ^ c, 12);         \
    a = a + b + (y);             \
    d = rotr(d ^ a, 8);          \
    c = c + d;                   \
    b = rotr(b ^ c, 7);

// The Merkle hasher's compression (zero counter and flags) on W nodes at once.
inline void compress_lanes(V h[8], const V m[16]) {
    V v[16];
    for (int i = 0; i < 8; i++) {
        v[i] = h[i];
        v[i + 8] = splat(IV[i]);
    }
    for (int r = 0; r < 10; r++) {
        const uint8_t *s = SIGMA[r];
        SG(v[0], v[4], v[8], v[12], m[s[0]], m[s[1]])
        SG(v[1], v[5], v[9], v[13], m[s[2]], m[s[3]])
        SG(v[2], v[6], v[10], v[14], m[s[4]], m[s[5]])
        SG(v[3], v[7], v[11], v[15], m[s[6]], m[s[7]])
        SG(v[0], v[5], v[10], v[15], m[s[8]], m[s[9]])
        SG(v[1], v[6], v[11], v[12], m[s[10]], m[s[11]])
        SG(v[2], v[7], v[8], v[13], m[s[12]], m[s[13]])
        SG(v[3], v[4], v[9], v[14], m[s[14]], m[s[15]])
    }
    for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}
#undef SG

}  // namespace

extern "C" {

void simd_merkle_commit_on_layer(uint32_t log_size, const uint32_t *prev, const uint32_t *const *cols, size_t ncols,
                                 uint32_t *out) {
    const size_t n = (size_t)1 << log_size;
    if (n < (size_t)W) {
        or_merkle_commit_on_layer(log_size, prev, cols, ncols, out);
        return;
    }
#pragma omp parallel for schedule(static) if (n >= 1024)
    for (size_t i = 0; i < n; i += W) {
        V h[8], m[16];
        for (int k = 0; k < 8; k++) h[k] = V{};
        if (prev) {
            // lane l: the children of node i + l, prev[16 (i + l) .. +16)
            alignas(64) uint32_t t[16][W];
            for (int l = 0; l < W; l++)
                for (int w = 0; w < 16; w++) t[w][l] = prev[16 * (i + l) + w];
            for (int w = 0; w < 16; w++) m[w] = vload(t[w]);
            compress_lanes(h, m);
        }
        for (size_t c0 = 0; c0 < ncols; c0 += 16) {
            for (int w = 0; w < 16; w++) m[w] = c0 + w < ncols ? vload(cols[c0 + w] + i) : V{};
            compress_lanes(h, m);
        }
        alignas(64) uint32_t o[8][W];
        for (int k = 0; k < 8; k++) vstore(o[k], h[k]);
        for (int l = 0; l < W; l++)
            for (int k = 0; k < 8; k++) out[8 * (i + l) + k] = o[k][l];
    }
}

// ---------------------------------------------------------------- eval_at_point
// p(P) = sum_i c_i prod_{bit b of i} f_b (f_0 = y, f_1 = x, f_b = pi^(b-1)(x)): the
// 16 products of the factors of bits 0..3 weight each group of 16 coefficients
// (lanes), then the group partials fold with the factors of the remaining bits.
}  // extern "C"

namespace {
inline qm31_t double_x(qm31_t x) {
    const qm31_t s = q_mul(x, x);
    qm31_t r = q_add(s, s);
    r.a.a = m_sub(r.a.a, 1);
    return r;
}
qm31_t fold_q(const qm31_t *vals, size_t n, const qm31_t *f) {  // f[0] multiplies the upper half
    if (n == 1) return vals[0];
    const qm31_t lo = fold_q(vals, n / 2, f + 1), hi = fold_q(vals + n / 2, n / 2, f + 1);
    return q_add(lo, q_mul(hi, f[0]));
}
qm31_t eval_at_point_one(const m31_t *c, uint32_t L, spoint_t p) {
    if (L < 6) return or_eval_at_point(c, L, p);
    qm31_t f[32];  // f[b]: factor of coefficient-index bit b
    f[0] = p.y;
    qm31_t x = p.x;
    for (uint32_t b = 1; b < L; b++) {
        f[b] = x;
        x = double_x(x);
    }
    // weights of the low 4 bits, per coordinate, as lanes (16 lanes; 2 vectors with AVX2)
    alignas(64) uint32_t wt[4][16];
    for (int j = 0; j < 16; j++) {
        qm31_t w = {{1, 0}, {0, 0}};
        for (int b = 0; b < 4; b++)
            if ((j >> b) & 1) w = q_mul(w, f[b]);
        wt[0][j] = w.a.a;
        wt[1][j] = w.a.b;
        wt[2][j] = w.b.a;
        wt[3][j] = w.b.b;
    }
    const size_t groups = (size_t)1 << (L - 4);
    std::vector<qm31_t> part(groups);
    for (size_t g = 0; g < groups; g++) {
        uint64_t s[4] = {0, 0, 0, 0};
        for (int h = 0; h < 16; h += W) {
            const V cv = vload(c + 16 * g + h);
            for (int t = 0; t < 4; t++) {
                const V w = vload(wt[t] + h);
                const V64 pe = mul_even((V64)cv, (V64)w), po = mul_even((V64)cv >> 32, (V64)w >> 32);
                const V64 r = fold(pe) + fold(po);  // below 2^33 a lane
                alignas(64) uint64_t lanes[W / 2];
                memcpy(lanes, &r, sizeof(r));
                for (int l = 0; l < W / 2; l++) s[t] += lanes[l];
            }
        }
        part[g] = {{m_red64(s[0]), m_red64(s[1])}, {m_red64(s[2]), m_red64(s[3])}};
    }
    // factors of the group index bits, highest first (fold_q's order)
    qm31_t fh[32];
    for (uint32_t b = 0; b + 4 < L; b++) fh[b] = f[L - 1 - b];
    return fold_q(part.data(), groups, fh);
}
}  // namespace

extern "C" {

qm31_t simd_eval_at_point(const m31_t *coeffs, uint32_t L, spoint_t p) { return eval_at_point_one(coeffs, L, p); }

void simd_eval_at_point_many(const m31_t *const *coeffs, const uint32_t *log_sizes, size_t n, spoint_t p,
                             qm31_t *out) {
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t i = 0; i < n; i++) out[i] = eval_at_point_one(coeffs[i], log_sizes[i], p);
}

// ---------------------------------------------------------------- quotients
// Per row: the batches' column sums sum_j c_j col_j[row] as 64-bit lane dot
// products over W consecutive rows; the line terms, denominators (inverted through
// the CM31 norm) and the Horner accumulation over batches per row.
void simd_accumulate_quotients(coset_t hc, const m31_t *const *cols, size_t ncols, qm31_t rc, size_t nb,
                               const spoint_t *pts, const uint32_t *bsz, const uint32_t *cidx, const qm31_t *vals,
                               m31_t *const out[4]) {
    (void)ncols;
    const uint32_t L = hc.log_size + 1;
    const size_t n = (size_t)1 << L;
    if (n < (size_t)W) {
        or_accumulate_quotients(hc, cols, ncols, rc, nb, pts, bsz, cidx, vals, out);
        return;
    }
    size_t total = 0;
    for (size_t b = 0; b < nb; b++) total += bsz[b];
    std::vector<qm31_t> ka(total), kb(total), kc(total), bcoef(nb);
    std::vector<qm31_t> asum(nb), bsum(nb);
    size_t off = 0;
    for (size_t b = 0; b < nb; b++) {
        bcoef[b] = or_qm31_pow(rc, bsz[b]);
        qm31_t alpha = {{1, 0}, {0, 0}};
        const qm31_t py = pts[b].y, cpy = {py.a, {m_neg(py.b.a), m_neg(py.b.b)}};
        asum[b] = bsum[b] = q_zero();
        for (uint32_t j = 0; j < bsz[b]; j++) {
            alpha = q_mul(alpha, rc);
            const qm31_t v = vals[off + j], cv = {v.a, {m_neg(v.b.a), m_neg(v.b.b)}};
            const qm31_t a = q_sub(cv, v), c = q_sub(cpy, py);
            const qm31_t bb = q_sub(q_mul(v, c), q_mul(a, py));
            asum[b] = q_add(asum[b], q_mul(alpha, a));
            bsum[b] = q_add(bsum[b], q_mul(alpha, bb));
            kc[off + j] = q_mul(alpha, c);
        }
        off += bsz[b];
    }
    const PointTables tabs;
    const size_t rows_per_task = W * 64;
#pragma omp parallel for schedule(static)
    for (size_t r0 = 0; r0 < n; r0 += rows_per_task) {
        const size_t r1 = r0 + rows_per_task < n ? r0 + rows_per_task : n;
        alignas(64) uint32_t sums[4][W];
        for (size_t r = r0; r < r1; r += W) {
            qm31_t acc[W];
            cpoint_t dps[W];
            for (int l = 0; l < W; l++) {
                acc[l] = q_zero();
                dps[l] = domain_point(tabs, hc, bitrev((uint32_t)(r + l), L));
            }
            size_t o = 0;
            for (size_t b = 0; b < nb; b++) {
                // lane dot products, even and odd lanes, folded every 3 terms
                V64 se[4] = {}, so[4] = {};
                for (uint32_t j = 0; j < bsz[b]; j++) {
                    const V x = vload(cols[cidx[o + j]] + r);
                    const qm31_t c = kc[o + j];
                    const uint32_t cc[4] = {c.a.a, c.a.b, c.b.a, c.b.b};
                    for (int t = 0; t < 4; t++) {
                        se[t] += mul_even((V64)x, splat64(cc[t]));
                        so[t] += mul_even((V64)x >> 32, splat64(cc[t]));
                    }
                    if (j % 3 == 2)
                        for (int t = 0; t < 4; t++) {
                            se[t] = fold(se[t]);
                            so[t] = fold(so[t]);
                        }
                }
                for (int t = 0; t < 4; t++) {
                    const V64 e = fold(fold(se[t])), od = fold(fold(so[t]));  // below 2^32
                    V s = (V)(e | (od << 32));
                    s = vmin(s, s - P);
                    s = vmin(s, s - P);
                    vstore(sums[t], s);
                }
                const cm31_t prx = pts[b].x.a, pry = pts[b].y.a, pix = pts[b].x.b, piy = pts[b].y.b;
                for (int l = 0; l < W; l++) {
                    const cpoint_t dp = dps[l];
                    const cm31_t d = c_sub(c_mul({m_sub(prx.a, dp.x), prx.b}, piy), c_mul({m_sub(pry.a, dp.y), pry.b}, pix));
                    const uint32_t ni = m_inv(m_add(m_mul(d.a, d.a), m_mul(d.b, d.b)));
                    const cm31_t dinv = {m_mul(d.a, ni), m_mul(m_neg(d.b), ni)};
                    qm31_t num = {{sums[0][l], sums[1][l]}, {sums[2][l], sums[3][l]}};
                    num = q_sub(num, q_add(q_scale(asum[b], dp.y), bsum[b]));
                    acc[l] = b == 0 ? q_mul_cm31(num, dinv) : q_add(q_mul(acc[l], bcoef[b]), q_mul_cm31(num, dinv));
                }
                o += bsz[b];
            }
            for (int l = 0; l < W; l++) {
                out[0][r + l] = acc[l].a.a;
                out[1][r + l] = acc[l].a.b;
                out[2][r + l] = acc[l].b.a;
                out[3][r + l] = acc[l].b.b;
            }
        }
    }
}

// ---------------------------------------------------------------- composition
void simd_wide_fib_composition(const m31_t *const *tr, size_t nc, size_t ext, const qm31_t *pw, const m31_t *den_inv,
                               m31_t *const out[4]) {
    if (ext < (size_t)W || nc < 3) {
        or_wide_fib_composition(tr, nc, ext, pw, den_inv, out);
        return;
    }
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < ext; r += W) {
        V64 se[4] = {}, so[4] = {};
        V a = vload(tr[0] + r), b = vload(tr[1] + r);
        V aa = vmul(a, a), bb = vmul(b, b);
        for (size_t i = 0; i + 2 < nc; i++) {
            const V c = vload(tr[i + 2] + r);
            const V cons = vsub(vadd(aa, bb), c);
            const qm31_t w = pw[nc - 3 - i];
            const uint32_t ww[4] = {w.a.a, w.a.b, w.b.a, w.b.b};
            for (int t = 0; t < 4; t++) {
                se[t] += mul_even((V64)cons, splat64(ww[t]));
                so[t] += mul_even((V64)cons >> 32, splat64(ww[t]));
            }
            if (i % 3 == 2)
                for (int t = 0; t < 4; t++) {
                    se[t] = fold(se[t]);
                    so[t] = fold(so[t]);
                }
            aa = bb;
            bb = vmul(c, c);
        }
        const V d = vload(den_inv + r);
        for (int t = 0; t < 4; t++) {
            const V64 e = fold(fold(se[t])), od = fold(fold(so[t]));
            V s = (V)(e | (od << 32));
            s = vmin(s, s - P);
            s = vmin(s, s - P);
            vstore(out[t] + r, vmul(s, d));
        }
    }
}

// ---------------------------------------------------------------- trace, vanishing
void simd_wide_fib_trace(const m31_t *a0, const m31_t *a1, size_t n_rows, size_t n_columns, m31_t *const *cols) {
    if (n_rows < (size_t)W || n_columns < 2) {
        or_wide_fib_trace(a0, a1, n_rows, n_columns, cols);
        return;
    }
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < n_rows; r += W) {
        V x = vload(a0 + r), y = vload(a1 + r);
        vstore(cols[0] + r, x);
        vstore(cols[1] + r, y);
        for (size_t c = 2; c < n_columns; c++) {
            const V z = vadd(vmul(x, x), vmul(y, y));
            vstore(cols[c] + r, z);
            x = y;
            y = z;
        }
    }
}

// The vanishing polynomial of CanonicCoset(L) takes one value on each half of
// CanonicCoset(L + 1) in bit-reversed order (both halves are cosets of the
// 2^L-point subgroup the polynomial vanishes on, shifted by a point and its
// conjugate): two inversions fill the column.
void simd_vanishing_inverses(uint32_t L, m31_t *den_inv) {
    const uint32_t E = L + 1;
    const size_t ne = (size_t)1 << E;
    const coset_t hc = or_canonic_half_coset(E), vc = or_canonic_coset(L);
    const uint32_t v0 = m_inv(or_coset_vanishing_m31(vc, or_circle_domain_at(hc, bitrev(0, E))));
    const uint32_t v1 = m_inv(or_coset_vanishing_m31(vc, or_circle_domain_at(hc, bitrev((uint32_t)(ne / 2), E))));
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < ne; i++) den_inv[i] = i < ne / 2 ? v0 : v1;
}

// ---------------------------------------------------------------- FRI folds
void simd_fold_line(const m31_t *const src[4], size_t n, coset_t dom, qm31_t alpha, m31_t *const dst[4]) {
    const uint32_t lg = (uint32_t)__builtin_ctzll(n);
    // x of the domain points, inverted in chunks (Montgomery)
#pragma omp parallel for schedule(static) if (n >= 65536)
    for (size_t i0 = 0; i0 < n / 2; i0 += 1024) {
        const size_t i1 = i0 + 1024 < n / 2 ? i0 + 1024 : n / 2;
        uint32_t xs[1024], pre[1024];
        uint32_t acc = 1;
        for (size_t i = i0; i < i1; i++) {
            xs[i - i0] = or_coset_at(dom, bitrev((uint32_t)(i << 1), lg)).x;
            pre[i - i0] = acc;
            acc = m_mul(acc, xs[i - i0]);
        }
        uint32_t inv = m_inv(acc);
        for (size_t i = i1; i-- > i0;) {
            const uint32_t xi = m_mul(inv, pre[i - i0]);
            inv = m_mul(inv, xs[i - i0]);
            const qm31_t fx = {{src[0][2 * i], src[1][2 * i]}, {src[2][2 * i], src[3][2 * i]}};
            const qm31_t fnx = {{src[0][2 * i + 1], src[1][2 * i + 1]}, {src[2][2 * i + 1], src[3][2 * i + 1]}};
            const qm31_t f0 = q_add(fx, fnx), f1 = q_scale(q_sub(fx, fnx), xi);
            const qm31_t r = q_add(f0, q_mul(alpha, f1));
            dst[0][i] = r.a.a;
            dst[1][i] = r.a.b;
            dst[2][i] = r.b.a;
            dst[3][i] = r.b.b;
        }
    }
}

void simd_fold_circle_into_line(const m31_t *const src[4], size_t n, coset_t hc, qm31_t alpha, m31_t *const dst[4]) {
    const uint32_t lg = (uint32_t)__builtin_ctzll(n);
    const qm31_t a2 = q_mul(alpha, alpha);
#pragma omp parallel for schedule(static) if (n >= 65536)
    for (size_t i0 = 0; i0 < n / 2; i0 += 1024) {
        const size_t i1 = i0 + 1024 < n / 2 ? i0 + 1024 : n / 2;
        uint32_t ys[1024], pre[1024];
        uint32_t acc = 1;
        for (size_t i = i0; i < i1; i++) {
            ys[i - i0] = or_circle_domain_at(hc, bitrev((uint32_t)(i << 1), lg)).y;
            pre[i - i0] = acc;
            acc = m_mul(acc, ys[i - i0]);
        }
        uint32_t inv = m_inv(acc);
        for (size_t i = i1; i-- > i0;) {
            const uint32_t yi = m_mul(inv, pre[i - i0]);
            inv = m_mul(inv, ys[i - i0]);
            const qm31_t fp = {{src[0][2 * i], src[1][2 * i]}, {src[2][2 * i], src[3][2 * i]}};
            const qm31_t fnp = {{src[0][2 * i + 1], src[1][2 * i + 1]}, {src[2][2 * i + 1], src[3][2 * i + 1]}};
            const qm31_t f0 = q_add(fp, fnp), f1 = q_scale(q_sub(fp, fnp), yi);
            const qm31_t d = {{dst[0][i], dst[1][i]}, {dst[2][i], dst[3][i]}};
            const qm31_t r = q_add(q_mul(d, a2), q_add(q_mul(alpha, f1), f0));
            dst[0][i] = r.a.a;
            dst[1][i] = r.a.b;
            dst[2][i] = r.b.a;
            dst[3][i] = r.b.b;
        }
    }
}

// Montgomery's batch inverse per chunk, on the threads.
void simd_batch_inverse_m31(const m31_t *src, m31_t *dst, size_t n) {
#pragma omp parallel for schedule(static) if (n >= 65536)
    for (size_t i0 = 0; i0 < n; i0 += 4096) {
        const size_t i1 = i0 + 4096 < n ? i0 + 4096 : n;
        uint32_t acc = 1;
        for (size_t i = i0; i < i1; i++) {
            dst[i] = acc;
            acc = m_mul(acc, src[i]);
        }
        uint32_t inv = m_inv(acc);
        for (size_t i = i1; i-- > i0;) {
            const uint32_t t = m_mul(inv, dst[i]);
            inv = m_mul(inv, src[i]);
            dst[i] = t;
        }
    }
}

void simd_set_threads(int n) { omp_set_num_threads(n < 1 ? 1 : n); }
int simd_lane_count(void) { return W; }

}  // extern "C"
