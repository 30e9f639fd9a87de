/*
 * CPU oracle for the Stwo circle-STARK hot path — TEST INFRASTRUCTURE ONLY.
 *
 * Restates stwo CpuBackend (stwo-prover @ ce5b975, a git dependency of the
 * reference, stwo_gpu_backend/Cargo.toml:8, absent from the reference tree) for
 * every trait method on the hot path. Each function cites the reference file:line
 * whose behaviour it follows; the reference's own tests assert those CUDA kernels
 * equal CpuBackend element for element (the #[cfg(test)] modules of stwo_gpu_backend/src).
 * Where the reference CUDA code and CpuBackend disagree (non-canonical neg(0) = p,
 * the n = 4 circle twiddle, mixed-size quotient batches) this file follows the
 * CpuBackend semantics that the reference tests encode.
 *
 * The oracle is the checker: only tests, the smoke check and the CPU-baseline leg
 * of the benchmark load it. It is deliberately written from the mathematical
 * definitions (domain points, Montgomery-free inverses, scalar loops) rather than
 * the GPU algorithms it checks.
 */
#include "stwo_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define P 2147483647u

static int g_threads = 1;

void or_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }
int or_get_threads(void) { return g_threads; }

/* Range-parallel loop over [0, n) on g_threads POSIX threads (the timed CPU
 * baseline uses every host core; tests run single-threaded). */
typedef void (*range_fn)(void *ctx, size_t lo, size_t hi);
typedef struct { range_fn f; void *ctx; size_t lo, hi; } range_job;
static void *range_tramp(void *p) { range_job *j = (range_job *)p; j->f(j->ctx, j->lo, j->hi); return NULL; }
static void par_range(size_t n, range_fn f, void *ctx) {
    int t = g_threads;
    if (t <= 1 || n < 4096) { f(ctx, 0, n); return; }
    pthread_t th[256];
    range_job jobs[256];
    jobs[0] = (range_job){f, ctx, 0, 0};
    size_t chunk = (n + t - 1) / t;
    int started = 0;
    for (int i = 0; i < t; i++) {
        size_t lo = (size_t)i * chunk, hi = lo + chunk > n ? n : lo + chunk;
        if (lo >= hi) break;
        jobs[i] = (range_job){f, ctx, lo, hi};
        if (i == 0) continue;
        if (pthread_create(&th[i], NULL, range_tramp, &jobs[i]) != 0) { f(ctx, lo, hi); jobs[i].f = NULL; }
        started = i;
    }
    f(ctx, jobs[0].lo, jobs[0].hi);
    for (int i = 1; i <= started; i++) if (jobs[i].f) pthread_join(th[i], NULL);
}

/* ======================================================================
 * M31 / CM31 / QM31   (cuda/include/fields.cuh:5-19, cuda/src/fields.cu:3-160)
 * p = 2^31 - 1; CM31 = M31[i]/(i^2+1); QM31 = CM31[u]/(u^2 - (2+i)).
 * ====================================================================== */
static inline m31_t m_add(m31_t a, m31_t b) { uint32_t s = a + b; return s >= P ? s - P : s; }
static inline m31_t m_sub(m31_t a, m31_t b) { return a >= b ? a - b : a + P - b; }
static inline m31_t m_neg(m31_t a) { return a ? P - a : 0; }
static inline m31_t m_mul(m31_t a, m31_t b) {
    uint64_t v = (uint64_t)a * b;
    uint64_t s = (v & P) + (v >> 31);
    s = (s & P) + (s >> 31);
    return s >= P ? (m31_t)(s - P) : (m31_t)s;
}
static m31_t m_pow(m31_t a, uint64_t e) {
    m31_t r = 1;
    while (e) { if (e & 1) r = m_mul(r, a); a = m_mul(a, a); e >>= 1; }
    return r;
}
/* fields.cu:32-40 computes x^(p-2) by an addition chain; Fermat gives the same value. */
static m31_t m_inv(m31_t a) { return m_pow(a, P - 2); }

m31_t or_m31_mul(m31_t a, m31_t b) { return m_mul(a, b); }
m31_t or_m31_inv(m31_t a) { return m_inv(a); }

static inline cm31_t c_add(cm31_t x, cm31_t y) { return (cm31_t){m_add(x.a, y.a), m_add(x.b, y.b)}; }
static inline cm31_t c_sub(cm31_t x, cm31_t y) { return (cm31_t){m_sub(x.a, y.a), m_sub(x.b, y.b)}; }
static inline cm31_t c_neg(cm31_t x) { return (cm31_t){m_neg(x.a), m_neg(x.b)}; }
static inline cm31_t c_mul(cm31_t x, cm31_t y) {
    return (cm31_t){m_sub(m_mul(x.a, y.a), m_mul(x.b, y.b)), m_add(m_mul(x.a, y.b), m_mul(x.b, y.a))};
}
static inline cm31_t c_scale(cm31_t x, m31_t s) { return (cm31_t){m_mul(x.a, s), m_mul(x.b, s)}; }
/* fields.cu:81-84: (a+bi)^-1 = (a-bi)/(a^2+b^2) */
static cm31_t c_inv(cm31_t x) {
    m31_t f = m_inv(m_add(m_mul(x.a, x.a), m_mul(x.b, x.b)));
    return (cm31_t){m_mul(x.a, f), m_mul(m_neg(x.b), f)};
}

static const cm31_t R_NONRESIDUE = {2, 1};

static inline qm31_t q_add(qm31_t x, qm31_t y) { return (qm31_t){c_add(x.a, y.a), c_add(x.b, y.b)}; }
static inline qm31_t q_sub(qm31_t x, qm31_t y) { return (qm31_t){c_sub(x.a, y.a), c_sub(x.b, y.b)}; }
static inline qm31_t q_neg(qm31_t x) { return (qm31_t){c_neg(x.a), c_neg(x.b)}; }
/* fields.cu:92-101: (a + bu)(c + du) = (ac + R bd) + (ad + bc) u */
static inline qm31_t q_mul(qm31_t x, qm31_t y) {
    cm31_t ac = c_mul(x.a, y.a), bd = c_mul(x.b, y.b);
    cm31_t ad = c_mul(x.a, y.b), bc = c_mul(x.b, y.a);
    return (qm31_t){c_add(ac, c_mul(R_NONRESIDUE, bd)), c_add(ad, bc)};
}
static inline qm31_t q_scale(qm31_t x, m31_t s) { return (qm31_t){c_scale(x.a, s), c_scale(x.b, s)}; }
static inline qm31_t q_mul_cm31(qm31_t x, cm31_t s) { return (qm31_t){c_mul(x.a, s), c_mul(x.b, s)}; }
static inline qm31_t q_from_m31(m31_t v) { return (qm31_t){{v, 0}, {0, 0}}; }
static inline qm31_t q_add_m31(qm31_t x, m31_t v) { x.a.a = m_add(x.a.a, v); return x; }
/* fields.cu:138-144: (a + bu)^-1 = (a - bu) / (a^2 - R b^2) */
static qm31_t q_inv(qm31_t x) {
    cm31_t b2 = c_mul(x.b, x.b);
    cm31_t denom = c_sub(c_mul(x.a, x.a), c_mul(R_NONRESIDUE, b2));
    cm31_t di = c_inv(denom);
    return (qm31_t){c_mul(x.a, di), c_neg(c_mul(x.b, di))};
}
static qm31_t q_pow(qm31_t x, uint64_t e) {
    qm31_t r = q_from_m31(1);
    while (e) { if (e & 1) r = q_mul(r, x); x = q_mul(x, x); e >>= 1; }
    return r;
}
/* complex conjugate over CM31[u]: a + bu -> a - bu (quotients.cu:50-51) */
static inline qm31_t q_conj(qm31_t x) { return (qm31_t){x.a, c_neg(x.b)}; }

qm31_t or_qm31_mul(qm31_t a, qm31_t b) { return q_mul(a, b); }
qm31_t or_qm31_inv(qm31_t a) { return q_inv(a); }
qm31_t or_qm31_pow(qm31_t a, uint64_t e) { return q_pow(a, e); }

/* ======================================================================
 * Circle group   (cuda/include/point.cuh:7-65)
 * Generator of the order-2^31 group: (2, 1268011823) (point.cuh:17).
 * ====================================================================== */
static const cpoint_t GEN = {2, 1268011823u};

static inline cpoint_t pt_mul(cpoint_t p, cpoint_t q) {
    return (cpoint_t){m_sub(m_mul(p.x, q.x), m_mul(p.y, q.y)), m_add(m_mul(p.x, q.y), m_mul(p.y, q.x))};
}
static inline cpoint_t pt_conj(cpoint_t p) { return (cpoint_t){p.x, m_neg(p.y)}; }

/* CirclePointIndex -> point: GEN^(index mod 2^31) by square-and-multiply (point.cuh:36-46). */
cpoint_t or_index_to_point(uint32_t index) {
    index &= 0x7fffffffu;
    cpoint_t r = {1, 0}, b = GEN;
    while (index) { if (index & 1) r = pt_mul(r, b); b = pt_mul(b, b); index >>= 1; }
    return r;
}

uint32_t or_bit_reverse_index(uint32_t i, uint32_t log_size) {
    if (log_size == 0) return i;
    uint32_t r = 0;
    for (uint32_t k = 0; k < log_size; k++) r |= ((i >> k) & 1u) << (log_size - 1 - k);
    return r;
}

/* Coset::index_at(i) = initial_index + step_size * i (mod 2^31) (quotients.cu:17-29). */
static inline uint32_t coset_index_at(coset_t c, uint64_t i) {
    return (uint32_t)(((uint64_t)c.initial_index + (uint64_t)c.step_size * i) & 0x7fffffffu);
}
cpoint_t or_coset_at(coset_t c, uint64_t i) { return or_index_to_point(coset_index_at(c, i)); }

/* CircleDomain::at: first half = half coset, second half = its conjugates
 * (negated indices) (quotients.cu:20-28). */
cpoint_t or_circle_domain_at(coset_t hc, uint64_t i) {
    uint64_t half = 1ull << hc.log_size;
    if (i < half) return or_index_to_point(coset_index_at(hc, i));
    uint32_t idx = coset_index_at(hc, i - half);
    return or_index_to_point((0x80000000u - idx) & 0x7fffffffu);
}

/* CanonicCoset(L).circle_domain().half_coset = Coset::half_odds(L-1):
 * initial index 2^(30-L), step 2^(32-L), log size L-1. Literal check:
 * poly.rs:583-595 (root coset 8388608 / 33554432 / 6 for L = 7). */
coset_t or_canonic_half_coset(uint32_t L) {
    coset_t c;
    c.log_size = L - 1;
    c.initial_index = 1u << (30 - L);
    c.step_size = (uint32_t)((1ull << (32 - L)) & 0x7fffffffu);
    return c;
}
/* CanonicCoset(L).coset = Coset::odds(L): initial 2^(30-L), step 2^(31-L). */
coset_t or_canonic_coset(uint32_t L) {
    coset_t c;
    c.log_size = L;
    c.initial_index = 1u << (30 - L);
    c.step_size = 1u << (31 - L);
    return c;
}

static coset_t coset_double(coset_t c) {
    c.initial_index = (c.initial_index * 2u) & 0x7fffffffu;
    c.step_size = (c.step_size * 2u) & 0x7fffffffu;
    c.log_size -= 1;
    return c;
}

/* ======================================================================
 * ColumnOps::bit_reverse_column (cuda/src/bit_reverse.cu:6-33, column.rs:10-34)
 * ====================================================================== */
static uint32_t log2_exact(size_t n) { uint32_t l = 0; while (((size_t)1 << l) < n) l++; return l; }

void or_bit_reverse_u32(uint32_t *v, size_t n) {
    uint32_t lg = log2_exact(n);
    for (size_t i = 0; i < n; i++) {
        size_t j = or_bit_reverse_index((uint32_t)i, lg);
        if (j > i) { uint32_t t = v[i]; v[i] = v[j]; v[j] = t; }
    }
}
void or_bit_reverse_qm31(qm31_t *v, size_t n) {
    uint32_t lg = log2_exact(n);
    for (size_t i = 0; i < n; i++) {
        size_t j = or_bit_reverse_index((uint32_t)i, lg);
        if (j > i) { qm31_t t = v[i]; v[i] = v[j]; v[j] = t; }
    }
}

/* ======================================================================
 * FieldOps::batch_inverse (cuda/src/batch_inverse.cu:25-177, field.rs:8-30).
 * The result is the element-wise inverse whatever the grouping.
 * ====================================================================== */
typedef struct { const void *src; void *dst; } inv_ctx;
static void inv_m31_range(void *c, size_t lo, size_t hi) {
    inv_ctx *x = (inv_ctx *)c;
    for (size_t i = lo; i < hi; i++) ((m31_t *)x->dst)[i] = m_inv(((const m31_t *)x->src)[i]);
}
static void inv_qm31_range(void *c, size_t lo, size_t hi) {
    inv_ctx *x = (inv_ctx *)c;
    for (size_t i = lo; i < hi; i++) ((qm31_t *)x->dst)[i] = q_inv(((const qm31_t *)x->src)[i]);
}
void or_batch_inverse_m31(const m31_t *src, m31_t *dst, size_t n) {
    inv_ctx c = {src, dst};
    par_range(n, inv_m31_range, &c);
}
void or_batch_inverse_qm31(const qm31_t *src, qm31_t *dst, size_t n) {
    inv_ctx c = {src, dst};
    par_range(n, inv_qm31_range, &c);
}

/* ======================================================================
 * PolyOps::precompute_twiddles (cuda/src/poly/twiddles.cu:29-73, poly.rs:170-192):
 * for each doubling of the root coset, the x coordinates of its first half in
 * bit-reversed order, concatenated; then a single 1. itwiddles = inverses.
 * ====================================================================== */
typedef struct { m31_t *tw; const m31_t *src; coset_t c; size_t off; } tw_ctx;
static void tw_layer_range(void *cv, size_t lo, size_t hi) {
    tw_ctx *x = (tw_ctx *)cv;
    uint32_t hl = x->c.log_size - 1;
    for (size_t h = lo; h < hi; h++)
        x->tw[x->off + or_bit_reverse_index((uint32_t)h, hl)] = or_coset_at(x->c, h).x;
}
static void tw_inv_range(void *cv, size_t lo, size_t hi) {
    tw_ctx *x = (tw_ctx *)cv;
    for (size_t i = lo; i < hi; i++) x->tw[i] = m_inv(x->src[i]);
}
void or_precompute_twiddles(coset_t root, m31_t *tw, m31_t *itw) {
    size_t size = (size_t)1 << root.log_size;
    size_t off = 0;
    coset_t c = root;
    for (uint32_t layer = 0; layer < root.log_size; layer++) {
        size_t half = ((size_t)1 << c.log_size) / 2;
        tw_ctx x = {tw, NULL, c, off};
        par_range(half, tw_layer_range, &x);
        off += half;
        c = coset_double(c);
    }
    tw[size - 1] = 1;
    if (itw) {
        tw_ctx x = {itw, tw, c, 0};
        par_range(size, tw_inv_range, &x);
    }
}

/* PolyOps::new_canonical_ordered (twiddles.cu:4-27): even positions, then odd
 * positions read backwards, then bit reversal. */
void or_new_canonical_ordered(uint32_t L, const m31_t *src, m31_t *dst) {
    size_t n = (size_t)1 << L, half = n / 2;
    for (size_t i = 0; i < half; i++) dst[i] = src[i << 1];
    for (size_t i = 0; i < half; i++) dst[half + i] = src[n - 1 - (i << 1)];
    or_bit_reverse_u32(dst, n);
}

/* ======================================================================
 * Circle FFT (cuda/src/poly/rfft.cu:5-64, ifft.cu:3-65, poly/utils.cu:3-14).
 * Line twiddles of a domain are the suffix of the tree of length n/2; layer k >= 1
 * uses the slice of length n/2^(k+1); the circle layer derives its twiddles from
 * the first line layer as [y, -y, -x, x] per pair (poly/utils.cu:3-14).
 * ====================================================================== */
static inline m31_t circle_twiddle(const m31_t *lt0, size_t h) {
    size_t k = h >> 2;
    switch (h & 3) {
    case 0: return lt0[2 * k + 1];
    case 1: return m_neg(lt0[2 * k + 1]);
    case 2: return m_neg(lt0[2 * k]);
    default: return lt0[2 * k];
    }
}

static void layer_twiddle_slices(const m31_t *tree, size_t tree_size, uint32_t L, const m31_t **slices) {
    /* slices[k] for k = 1..L-1: line layer k twiddles, length 2^(L-1-k). */
    const m31_t *suffix = tree + (tree_size - ((size_t)1 << (L - 1)));
    size_t off = 0;
    for (uint32_t k = 1; k < L; k++) {
        slices[k] = suffix + off;
        off += (size_t)1 << (L - 1 - k);
    }
}

/* One butterfly layer over pair indices [lo, hi): pair b belongs to twiddle
 * group h = b >> k (fft_layer_loop in CpuBackend). */
typedef struct { m31_t *v; const m31_t **sl; uint32_t k; uint32_t pad; m31_t scale; } fft_ctx;
static void ifft_layer_range(void *cv, size_t lo, size_t hi) {
    fft_ctx *c = (fft_ctx *)cv;
    uint32_t k = c->k;
    size_t half = (size_t)1 << k;
    for (size_t b = lo; b < hi; b++) {
        size_t h = b >> k, l = b & (half - 1);
        size_t i0 = (h << (k + 1)) + l, i1 = i0 + half;
        m31_t t = k == 0 ? circle_twiddle(c->sl[1], h) : c->sl[k][h];
        m31_t a = c->v[i0], d = c->v[i1];
        c->v[i0] = m_add(a, d);
        c->v[i1] = m_mul(m_sub(a, d), t);
    }
}
static void rfft_layer_range(void *cv, size_t lo, size_t hi) {
    fft_ctx *c = (fft_ctx *)cv;
    uint32_t k = c->k;
    size_t half = (size_t)1 << k;
    for (size_t b = lo; b < hi; b++) {
        size_t h = b >> k, l = b & (half - 1);
        size_t i0 = (h << (k + 1)) + l, i1 = i0 + half;
        m31_t t = k == 0 ? circle_twiddle(c->sl[1], h) : c->sl[k][h];
        m31_t a = c->v[i0], d = m_mul(c->v[i1], t);
        c->v[i0] = m_add(a, d);
        c->v[i1] = m_sub(a, d);
    }
}
static void scale_range(void *cv, size_t lo, size_t hi) {
    fft_ctx *c = (fft_ctx *)cv;
    for (size_t i = lo; i < hi; i++) c->v[i] = m_mul(c->v[i], c->scale);
}

/* CpuBackend::interpolate; returns 0 on success, -1 on a bad size. */
int or_interpolate(coset_t hc, m31_t *v, const m31_t *itw, size_t tree_size) {
    uint32_t L = hc.log_size + 1;
    size_t n = (size_t)1 << L;
    if (L == 0 || hc.log_size > 30) return -1;
    if (L == 1) {
        /* CpuBackend special case: ibutterfly with 1/y of the half coset's point. */
        cpoint_t p = or_coset_at(hc, 0);
        m31_t yi = m_inv(p.y), ni = m_inv(2);
        m31_t a = v[0], b = v[1];
        v[0] = m_mul(m_add(a, b), ni);
        v[1] = m_mul(m_mul(m_sub(a, b), yi), ni);
        return 0;
    }
    if (L == 2) {
        cpoint_t p = or_coset_at(hc, 0);
        m31_t xi = m_inv(p.x), yi = m_inv(p.y), ni = m_inv(4);
        m31_t v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3], t;
        t = v0; v0 = m_add(t, v1); v1 = m_mul(m_sub(t, v1), yi);
        t = v2; v2 = m_add(t, v3); v3 = m_mul(m_sub(t, v3), m_neg(yi));
        t = v0; v0 = m_add(t, v2); v2 = m_mul(m_sub(t, v2), xi);
        t = v1; v1 = m_add(t, v3); v3 = m_mul(m_sub(t, v3), xi);
        v[0] = m_mul(v0, ni); v[1] = m_mul(v1, ni); v[2] = m_mul(v2, ni); v[3] = m_mul(v3, ni);
        return 0;
    }
    if (tree_size < n / 2) return -1;
    const m31_t *sl[32];
    layer_twiddle_slices(itw, tree_size, L, sl);
    for (uint32_t k = 0; k < L; k++) {
        fft_ctx c = {v, sl, k, 0, 0};
        par_range(n / 2, ifft_layer_range, &c);
    }
    /* rescale by 2^-L (ifft.cu:60-64) */
    fft_ctx c = {v, sl, 0, 0, m_inv((m31_t)(1u << L) % P)};
    par_range(n, scale_range, &c);
    return 0;
}

/* CpuBackend::evaluate on an already-extended coefficient buffer. */
int or_evaluate(coset_t hc, m31_t *v, const m31_t *tw, size_t tree_size) {
    uint32_t L = hc.log_size + 1;
    size_t n = (size_t)1 << L;
    if (hc.log_size > 30) return -1;
    if (L == 1) {
        cpoint_t p = or_coset_at(hc, 0);
        m31_t a = v[0], t = m_mul(v[1], p.y);
        v[0] = m_add(a, t); v[1] = m_sub(a, t);
        return 0;
    }
    if (L == 2) {
        cpoint_t p = or_coset_at(hc, 0);
        m31_t v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3], t;
        t = m_mul(v2, p.x); v2 = m_sub(v0, t); v0 = m_add(v0, t);
        t = m_mul(v3, p.x); v3 = m_sub(v1, t); v1 = m_add(v1, t);
        t = m_mul(v1, p.y); v1 = m_sub(v0, t); v0 = m_add(v0, t);
        t = m_mul(v3, m_neg(p.y)); v3 = m_sub(v2, t); v2 = m_add(v2, t);
        v[0] = v0; v[1] = v1; v[2] = v2; v[3] = v3;
        return 0;
    }
    if (tree_size < n / 2) return -1;
    const m31_t *sl[32];
    layer_twiddle_slices(tw, tree_size, L, sl);
    for (int k = (int)L - 1; k >= 0; k--) {
        fft_ctx c = {v, sl, (uint32_t)k, 0, 0};
        par_range(n / 2, rfft_layer_range, &c);
    }
    return 0;
}

/* Column batches, as the prover drives them: every column interpolated in place;
 * every column's coeff_len coefficients evaluated on the domain of half coset hc
 * into out (zero-extended). */
void or_interpolate_many(coset_t hc, m31_t *const *cols, size_t n_cols, const m31_t *itw, size_t tree_size) {
    for (size_t c = 0; c < n_cols; c++) or_interpolate(hc, cols[c], itw, tree_size);
}
void or_evaluate_many(coset_t hc, const m31_t *const *coeffs, size_t coeff_len, m31_t *const *out, size_t n_cols,
                      const m31_t *tw, size_t tree_size) {
    const size_t n = (size_t)2 << hc.log_size;
    for (size_t c = 0; c < n_cols; c++) {
        memcpy(out[c], coeffs[c], coeff_len * 4);
        memset(out[c] + coeff_len, 0, (n - coeff_len) * 4);
        or_evaluate(hc, out[c], tw, tree_size);
    }
}

/* Generic fold (CpuBackend poly/utils.rs `fold`): values split in halves, the
 * first factor multiplies the upper half. */
static qm31_t fold_m31(const m31_t *vals, size_t n, const qm31_t *factors) {
    if (n == 1) return q_from_m31(vals[0]);
    qm31_t lo = fold_m31(vals, n / 2, factors + 1);
    qm31_t hi = fold_m31(vals + n / 2, n / 2, factors + 1);
    return q_add(lo, q_mul(hi, factors[0]));
}
static qm31_t fold_q(const qm31_t *vals, size_t n, const qm31_t *factors) {
    if (n == 1) return vals[0];
    qm31_t lo = fold_q(vals, n / 2, factors + 1);
    qm31_t hi = fold_q(vals + n / 2, n / 2, factors + 1);
    return q_add(lo, q_mul(hi, factors[0]));
}

static qm31_t double_x_q(qm31_t x) {
    /* x -> 2x^2 - 1 (CirclePoint::double_x) */
    qm31_t s = q_mul(x, x);
    return q_sub(q_add(s, s), q_from_m31(1));
}

/* PolyOps::eval_at_point (cuda/src/poly/eval_at_point.cu:99-109): factors, from
 * the highest coefficient bit down: [pi^(L-2)(x), ..., pi(x), x, y]. */
qm31_t or_eval_at_point(const m31_t *coeffs, uint32_t L, spoint_t p) {
    if (L == 0) return q_from_m31(coeffs[0]);
    qm31_t f[32];
    f[L - 1] = p.y;
    qm31_t x = p.x;
    for (uint32_t i = 1; i < L; i++) {
        f[L - 1 - i] = x;
        x = double_x_q(x);
    }
    return fold_m31(coeffs, (size_t)1 << L, f);
}

void or_eval_at_point_many(const m31_t *const *coeffs, const uint32_t *log_sizes, size_t n, spoint_t p, qm31_t *out) {
    for (size_t i = 0; i < n; i++) out[i] = or_eval_at_point(coeffs[i], log_sizes[i], p);
}

/* LinePoly::eval_at_point (bit-reversed coefficient storage): factors
 * [x, pi(x), pi^2(x), ...] from the highest bit down (the identity checked by
 * stwo_gpu_backend/src/fri.rs:142-192). */
qm31_t or_line_eval_at_point(const qm31_t *coeffs, uint32_t L, qm31_t x) {
    if (L == 0) return coeffs[0];
    qm31_t f[32];
    for (uint32_t i = 0; i < L; i++) { f[i] = x; x = double_x_q(x); }
    return fold_q(coeffs, (size_t)1 << L, f);
}

/* Definition-level evaluation: out[pos] = poly(domain point at bit_reverse(pos)).
 * O(n * 2^coeffs_log); used to pin the FFT on small domains. */
void or_evaluate_direct(coset_t hc, const m31_t *coeffs, uint32_t coeffs_log, m31_t *out) {
    uint32_t L = hc.log_size + 1;
    size_t n = (size_t)1 << L;
    for (size_t pos = 0; pos < n; pos++) {
        cpoint_t p = or_circle_domain_at(hc, or_bit_reverse_index((uint32_t)pos, L));
        spoint_t sp = {q_from_m31(p.x), q_from_m31(p.y)};
        qm31_t r = or_eval_at_point(coeffs, coeffs_log, sp);
        out[pos] = r.a.a;
    }
}

/* ======================================================================
 * FriOps (cuda/src/fri/fold_line.cu:5-53, fold_circle_into_line.cu:7-69,
 * stwo_gpu_backend/src/fri.rs:16-66). QM31 columns are 4 M31 coordinate arrays.
 * ====================================================================== */
static inline qm31_t load_q(const m31_t *const c[4], size_t i) {
    return (qm31_t){{c[0][i], c[1][i]}, {c[2][i], c[3][i]}};
}
static inline void store_q(m31_t *const c[4], size_t i, qm31_t v) {
    c[0][i] = v.a.a; c[1][i] = v.a.b; c[2][i] = v.b.a; c[3][i] = v.b.b;
}

typedef struct { const m31_t *const *src; m31_t *const *dst; coset_t dom; qm31_t alpha, a2; uint32_t lg; } fold_ctx;
static void fold_line_range(void *cv, size_t lo, size_t hi) {
    fold_ctx *c = (fold_ctx *)cv;
    for (size_t i = lo; i < hi; i++) {
        m31_t x = or_coset_at(c->dom, or_bit_reverse_index((uint32_t)(i << 1), c->lg)).x;
        qm31_t fx = load_q(c->src, 2 * i), fnx = load_q(c->src, 2 * i + 1);
        qm31_t f0 = q_add(fx, fnx), f1 = q_scale(q_sub(fx, fnx), m_inv(x));
        store_q(c->dst, i, q_add(f0, q_mul(c->alpha, f1)));
    }
}
void or_fold_line(const m31_t *const src[4], size_t n, coset_t dom, qm31_t alpha, m31_t *const dst[4]) {
    fold_ctx c = {src, dst, dom, alpha, alpha, log2_exact(n)};
    par_range(n / 2, fold_line_range, &c);
}

static void fold_circle_range(void *cv, size_t lo, size_t hi) {
    fold_ctx *c = (fold_ctx *)cv;
    for (size_t i = lo; i < hi; i++) {
        cpoint_t p = or_circle_domain_at(c->dom, or_bit_reverse_index((uint32_t)(i << 1), c->lg));
        qm31_t fp = load_q(c->src, 2 * i), fnp = load_q(c->src, 2 * i + 1);
        qm31_t f0 = q_add(fp, fnp), f1 = q_scale(q_sub(fp, fnp), m_inv(p.y));
        qm31_t fprime = q_add(q_mul(c->alpha, f1), f0);
        store_q(c->dst, i, q_add(q_mul(load_q((const m31_t *const *)c->dst, i), c->a2), fprime));
    }
}
void or_fold_circle_into_line(const m31_t *const src[4], size_t n, coset_t hc, qm31_t alpha,
                              m31_t *const dst[4]) {
    fold_ctx c = {src, dst, hc, alpha, q_mul(alpha, alpha), log2_exact(n)};
    par_range(n / 2, fold_circle_range, &c);
}

/* ======================================================================
 * Blake2s (cuda/src/blake2s.cu:5-95) and the Merkle layer hash
 * (blake2s.cu:97-151, stwo_gpu_backend/src/blake2s.rs:19-97).
 * The Merkle hasher uses the bare compression function: chaining state starts
 * at zero, the IV fills v[8..15], counter and finalisation flags are zero, and
 * column words are absorbed in zero-padded 16-word chunks.
 * ====================================================================== */
static const uint32_t B2_IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                  0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
static const uint8_t B2_SIGMA[10][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15},
    {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4},
    {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13},
    {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11},
    {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5},
    {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0},
};
static inline uint32_t rotr32(uint32_t x, int c) { return (x >> c) | (x << (32 - c)); }
#define B2G(a, b, c, d, x, y)        \
    do {                             \
        a = a + b + (x);             \
        d = rotr32(d ^ a, 16);       \
        c = c + d;                   \
        b = rotr32(b ^ c, 12);       \
        a = a + b + (y);             \
        d = rotr32(d ^ a, 8);        \
        c = c + d;                   \
        b = rotr32(b ^ c, 7);        \
    } while (0)

void or_blake2s_compress(uint32_t h[8], const uint32_t m[16], uint32_t t0, uint32_t t1,
                         uint32_t f0, uint32_t f1) {
    uint32_t v[16];
    for (int i = 0; i < 8; i++) { v[i] = h[i]; v[i + 8] = B2_IV[i]; }
    v[12] ^= t0; v[13] ^= t1; v[14] ^= f0; v[15] ^= f1;
    for (int r = 0; r < 10; r++) {
        const uint8_t *s = B2_SIGMA[r];
        B2G(v[0], v[4], v[8], v[12], m[s[0]], m[s[1]]);
        B2G(v[1], v[5], v[9], v[13], m[s[2]], m[s[3]]);
        B2G(v[2], v[6], v[10], v[14], m[s[4]], m[s[5]]);
        B2G(v[3], v[7], v[11], v[15], m[s[6]], m[s[7]]);
        B2G(v[0], v[5], v[10], v[15], m[s[8]], m[s[9]]);
        B2G(v[1], v[6], v[11], v[12], m[s[10]], m[s[11]]);
        B2G(v[2], v[7], v[8], v[13], m[s[12]], m[s[13]]);
        B2G(v[3], v[4], v[9], v[14], m[s[14]], m[s[15]]);
    }
    for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}

/* Standard BLAKE2s-256 (RFC 7693), used only to pin the compression function
 * against an independent implementation. */
void or_blake2s_std(const uint8_t *msg, size_t len, uint8_t out[32]) {
    uint32_t h[8];
    for (int i = 0; i < 8; i++) h[i] = B2_IV[i];
    h[0] ^= 0x01010000u ^ 32u;
    uint64_t t = 0;
    size_t off = 0;
    uint32_t m[16];
    while (len - off > 64) {
        memcpy(m, msg + off, 64);
        t += 64; off += 64;
        or_blake2s_compress(h, m, (uint32_t)t, (uint32_t)(t >> 32), 0, 0);
    }
    memset(m, 0, 64);
    memcpy(m, msg + off, len - off);
    t += len - off;
    or_blake2s_compress(h, m, (uint32_t)t, (uint32_t)(t >> 32), 0xffffffffu, 0);
    memcpy(out, h, 32);
}

typedef struct { const uint32_t *prev; const uint32_t *const *cols; size_t ncols; uint32_t *out; } merkle_ctx;
static void merkle_range(void *cv, size_t lo, size_t hi) {
    merkle_ctx *c = (merkle_ctx *)cv;
    const uint32_t *prev = c->prev;
    const uint32_t *const *cols = c->cols;
    size_t ncols = c->ncols;
    uint32_t *out = c->out;
    for (size_t i = lo; i < hi; i++) {
        uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        uint32_t m[16];
        if (prev) {
            memcpy(m, prev + 16 * i, 64); /* left child hash, then right child hash */
            or_blake2s_compress(h, m, 0, 0, 0, 0);
        }
        for (size_t c = 0; c < ncols; c += 16) {
            for (int j = 0; j < 16; j++) m[j] = (c + j < ncols) ? cols[c + j][i] : 0;
            or_blake2s_compress(h, m, 0, 0, 0, 0);
        }
        memcpy(out + 8 * i, h, 32);
    }
}
void or_merkle_commit_on_layer(uint32_t log_size, const uint32_t *prev,
                               const uint32_t *const *cols, size_t ncols, uint32_t *out) {
    merkle_ctx c = {prev, cols, ncols, out};
    par_range((size_t)1 << log_size, merkle_range, &c);
}

/* ======================================================================
 * QuotientOps::accumulate_quotients (cuda/src/quotients.cu:49-178,
 * stwo_gpu_backend/src/quotient.rs:17-115). Line coefficients are indexed by the
 * cumulative batch offset (the CpuBackend semantics), batch coefficient
 * = random_coeff^|batch|, denominator in CM31.
 * ====================================================================== */
typedef struct {
    coset_t hc; const m31_t *const *cols; size_t nb; const spoint_t *pts; const uint32_t *bsz, *cidx;
    const qm31_t *abc, *bcoef; m31_t *const *out; uint32_t L;
} quot_ctx;
static void quot_range(void *cv, size_t lo, size_t hi);

void or_accumulate_quotients(coset_t hc, const m31_t *const *cols, size_t ncols, qm31_t rc,
                             size_t nb, const spoint_t *pts, const uint32_t *bsz,
                             const uint32_t *cidx, const qm31_t *vals, m31_t *const out[4]) {
    (void)ncols;
    uint32_t L = hc.log_size + 1;
    size_t n = (size_t)1 << L;
    size_t total = 0;
    for (size_t b = 0; b < nb; b++) total += bsz[b];
    qm31_t *abc = (qm31_t *)malloc(sizeof(qm31_t) * 3 * (total ? total : 1));
    qm31_t *bcoef = (qm31_t *)malloc(sizeof(qm31_t) * (nb ? nb : 1));
    size_t off = 0;
    for (size_t b = 0; b < nb; b++) {
        bcoef[b] = q_pow(rc, bsz[b]);
        qm31_t alpha = q_from_m31(1);
        for (uint32_t j = 0; j < bsz[b]; j++) {
            alpha = q_mul(alpha, rc);
            qm31_t v = vals[off + j], py = pts[b].y;
            qm31_t a = q_sub(q_conj(v), v);
            qm31_t c = q_sub(q_conj(py), py);
            qm31_t bb = q_sub(q_mul(v, c), q_mul(a, py));
            abc[3 * (off + j) + 0] = q_mul(alpha, a);
            abc[3 * (off + j) + 1] = q_mul(alpha, bb);
            abc[3 * (off + j) + 2] = q_mul(alpha, c);
        }
        off += bsz[b];
    }
    quot_ctx qc = {hc, cols, nb, pts, bsz, cidx, abc, bcoef, out, L};
    par_range(n, quot_range, &qc);
    free(abc);
    free(bcoef);
}

static void quot_range(void *cv, size_t lo, size_t hi) {
    quot_ctx *q = (quot_ctx *)cv;
    coset_t hc = q->hc;
    const m31_t *const *cols = q->cols;
    size_t nb = q->nb;
    const spoint_t *pts = q->pts;
    const uint32_t *bsz = q->bsz, *cidx = q->cidx;
    const qm31_t *abc = q->abc, *bcoef = q->bcoef;
    m31_t *const *out = q->out;
    uint32_t L = q->L;
    for (size_t row = lo; row < hi; row++) {
        cpoint_t dp = or_circle_domain_at(hc, or_bit_reverse_index((uint32_t)row, L));
        qm31_t acc = q_from_m31(0);
        size_t o = 0;
        for (size_t b = 0; b < nb; b++) {
            cm31_t prx = pts[b].x.a, pry = pts[b].y.a, pix = pts[b].x.b, piy = pts[b].y.b;
            cm31_t d = c_sub(c_mul((cm31_t){m_sub(prx.a, dp.x), prx.b}, piy),
                             c_mul((cm31_t){m_sub(pry.a, dp.y), pry.b}, pix));
            cm31_t dinv = c_inv(d);
            qm31_t num = q_from_m31(0);
            for (uint32_t j = 0; j < bsz[b]; j++) {
                const qm31_t *k = abc + 3 * (o + j);
                qm31_t value = q_scale(k[2], cols[cidx[o + j]][row]);
                qm31_t lin = q_add(q_scale(k[0], dp.y), k[1]);
                num = q_add(num, q_sub(value, lin));
            }
            acc = q_add(q_mul(acc, bcoef[b]), q_mul_cm31(num, dinv));
            o += bsz[b];
        }
        store_q(out, row, acc);
    }
}

/* AccumulationOps::accumulate (cuda/src/accumulate.cu:4-26). */
void or_accumulate(m31_t *const l[4], const m31_t *const r[4], size_t n) {
    for (int c = 0; c < 4; c++)
        for (size_t i = 0; i < n; i++) l[c][i] = m_add(l[c][i], r[c][i]);
}

/* ======================================================================
 * Wide-Fibonacci AIR (stwo_gpu_backend/src/examples/wide_fibonacci.rs:90-203,
 * cuda/src/examples/wide_fibonacci.cu:3-38).
 * ====================================================================== */

/* constraints::coset_vanishing: shift p by -initial + step/2, take x, double
 * log_size - 1 times. */
m31_t or_coset_vanishing_m31(coset_t c, cpoint_t p) {
    cpoint_t init = or_index_to_point(c.initial_index);
    cpoint_t half_step = or_index_to_point(c.step_size >> 1);
    p = pt_mul(pt_mul(p, pt_conj(init)), half_step);
    m31_t x = p.x;
    for (uint32_t i = 1; i < c.log_size; i++) x = m_sub(m_add(m_mul(x, x), m_mul(x, x)), 1);
    return x;
}

void or_wide_fib_trace_row(m31_t a, m31_t b, size_t n, m31_t *row) {
    row[0] = a;
    if (n > 1) row[1] = b;
    for (size_t i = 2; i < n; i++) row[i] = m_add(m_mul(row[i - 1], row[i - 1]), m_mul(row[i - 2], row[i - 2]));
}

/* The trace's columns: row r of write_trace_row (wide_fibonacci.rs:177-191) in
 * cols[c][r]. */
void or_wide_fib_trace(const m31_t *a0, const m31_t *a1, size_t n_rows, size_t n_columns, m31_t *const *cols) {
    m31_t *row = (m31_t *)malloc(sizeof(m31_t) * (n_columns ? n_columns : 1));
    for (size_t r = 0; r < n_rows; r++) {
        or_wide_fib_trace_row(a0[r], a1[r], n_columns, row);
        for (size_t c = 0; c < n_columns; c++) cols[c][r] = row[c];
    }
    free(row);
}

/* Inverses of the vanishing polynomial of CanonicCoset(L) over CanonicCoset(L + 1)
 * in bit-reversed order (wide_fibonacci.rs:101-104): 2^(L+1) values. */
void or_vanishing_inverses(uint32_t L, m31_t *den_inv) {
    const uint32_t E = L + 1;
    const size_t ne = (size_t)1 << E;
    coset_t hc = or_canonic_half_coset(E), vc = or_canonic_coset(L);
    m31_t *den = (m31_t *)malloc(sizeof(m31_t) * ne);
    for (size_t pos = 0; pos < ne; pos++)
        den[pos] = or_coset_vanishing_m31(vc, or_circle_domain_at(hc, or_bit_reverse_index((uint32_t)pos, E)));
    or_batch_inverse_m31(den, den_inv, ne);
    free(den);
}

typedef struct { const m31_t *const *tr; size_t nc; const qm31_t *pw; const m31_t *den_inv; m31_t *const *out; } wf_ctx;
static void wf_range(void *cv, size_t lo, size_t hi) {
    wf_ctx *c = (wf_ctx *)cv;
    const m31_t *const *tr = c->tr;
    size_t nc = c->nc;
    const qm31_t *pw = c->pw;
    for (size_t r = lo; r < hi; r++) {
        qm31_t num = q_from_m31(0);
        for (size_t i = 0; i + 2 < nc; i++) {
            m31_t a = tr[i][r], b = tr[i + 1][r], c = tr[i + 2][r];
            m31_t cons = m_sub(m_add(m_mul(a, a), m_mul(b, b)), c);
            num = q_add(num, q_scale(pw[nc - 3 - i], cons));
        }
        store_q(c->out, r, q_scale(num, c->den_inv[r]));
    }
}
void or_wide_fib_composition(const m31_t *const *tr, size_t nc, size_t ext, const qm31_t *pw,
                             const m31_t *den_inv, m31_t *const out[4]) {
    wf_ctx c = {tr, nc, pw, den_inv, out};
    par_range(ext, wf_range, &c);
}
