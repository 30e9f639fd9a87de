/*
 * CPU oracle of the wide-Fibonacci STARK prover — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of stwo's prove() (stwo-prover @ ce5b975, not vendored) as
 * the reference drives it for the wide-Fibonacci AIR
 * (stwo_gpu_backend/src/examples/wide_fibonacci.rs:205-250), built on this oracle's
 * CpuBackend restatements (stwo_oracle.c). Its proof bytes are the checker for the
 * GPU prover: both must be identical for the same job and inputs.
 *
 * Protocol pieces restated here (from stwo's published sources, recalled; no copy of
 * stwo is present to pin them):
 *   core/channel/blake2s.rs   Blake2sChannel: digest, n_sent; mix_felts, mix_nonce
 *                             (one compression of the digest with [lo, hi, 0..]),
 *                             draw_random_bytes, draw_felt (retry while any u32 >= 2P)
 *   core/vcs/blake2_merkle.rs mix_root = H(digest || root)
 *   core/vcs/prover.rs        MerkleProver::commit / decommit
 *   core/pcs/prover.rs        CommitmentSchemeProver::commit / prove_values
 *   core/pcs/quotients.rs     compute_fri_quotients (groups by size, largest first)
 *   core/fri.rs               FriProver::commit / decommit, Queries
 *   core/prover/mod.rs        prove(): composition, OODS point, sanity check
 *   core/circle.rs            CirclePoint::get_random_point
 *   core/constraints.rs       coset_vanishing
 *   core/backend/cpu/grind    least nonce with pow_bits trailing zeros
 *
 * Proof bytes: CommitmentSchemeProof's fields in declaration order, little endian,
 * u64 vector lengths, 32-byte hashes, u32 field words.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "stwo_oracle.h"

#define P_M31 0x7fffffffu

/* ---------------------------------------------------------------- field helpers */
static m31_t fa(m31_t a, m31_t b) { uint32_t s = a + b; return s >= P_M31 ? s - P_M31 : s; }
static m31_t fs(m31_t a, m31_t b) { return a >= b ? a - b : a + P_M31 - b; }
static qm31_t qa(qm31_t x, qm31_t y) {
    qm31_t r = {{fa(x.a.a, y.a.a), fa(x.a.b, y.a.b)}, {fa(x.b.a, y.b.a), fa(x.b.b, y.b.b)}};
    return r;
}
static qm31_t qs(qm31_t x, qm31_t y) {
    qm31_t r = {{fs(x.a.a, y.a.a), fs(x.a.b, y.a.b)}, {fs(x.b.a, y.b.a), fs(x.b.b, y.b.b)}};
    return r;
}
static qm31_t qsc(qm31_t x, m31_t s) {
    qm31_t r = {{or_m31_mul(x.a.a, s), or_m31_mul(x.a.b, s)}, {or_m31_mul(x.b.a, s), or_m31_mul(x.b.b, s)}};
    return r;
}
static qm31_t qone(void) { qm31_t r = {{1, 0}, {0, 0}}; return r; }
static qm31_t qzero(void) { qm31_t r = {{0, 0}, {0, 0}}; return r; }
static int qeq(qm31_t x, qm31_t y) {
    return x.a.a == y.a.a && x.a.b == y.a.b && x.b.a == y.b.a && x.b.b == y.b.b;
}

/* ---------------------------------------------------------------- byte buffer */
typedef struct { uint8_t *p; size_t n, cap; } buf_t;
static void put(buf_t *b, const void *src, size_t n) {
    if (b->n + n > b->cap) {
        size_t c = b->cap ? b->cap : 4096;
        while (c < b->n + n) c *= 2;
        b->p = (uint8_t *)realloc(b->p, c);
        b->cap = c;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
}
static void put_u32(buf_t *b, uint32_t v) { put(b, &v, 4); }
static void put_u64(buf_t *b, uint64_t v) { put(b, &v, 8); }
static void put_q(buf_t *b, qm31_t v) { put_u32(b, v.a.a); put_u32(b, v.a.b); put_u32(b, v.b.a); put_u32(b, v.b.b); }

/* ---------------------------------------------------------------- Blake2sChannel */
typedef struct { uint8_t digest[32]; uint64_t n_sent; } channel_t;

static void ch_update(channel_t *c, const uint8_t d[32]) { memcpy(c->digest, d, 32); c->n_sent = 0; }
static void ch_mix_root(channel_t *c, const uint8_t root[32]) {
    uint8_t m[64], out[32];
    memcpy(m, c->digest, 32);
    memcpy(m + 32, root, 32);
    or_blake2s_std(m, 64, out);
    ch_update(c, out);
}
static void ch_mix_felts(channel_t *c, const qm31_t *f, size_t n) {
    uint8_t *m = (uint8_t *)malloc(32 + 16 * n), out[32];
    memcpy(m, c->digest, 32);
    for (size_t i = 0; i < n; i++) {
        uint32_t w[4] = {f[i].a.a, f[i].a.b, f[i].b.a, f[i].b.b};
        memcpy(m + 32 + 16 * i, w, 16);
    }
    or_blake2s_std(m, 32 + 16 * n, out);
    free(m);
    ch_update(c, out);
}
static void nonce_digest(const uint8_t digest[32], uint64_t nonce, uint8_t out[32]) {
    uint32_t h[8], m[16];
    memset(m, 0, sizeof(m));
    memcpy(h, digest, 32);
    m[0] = (uint32_t)nonce;
    m[1] = (uint32_t)(nonce >> 32);
    or_blake2s_compress(h, m, 0, 0, 0, 0);
    memcpy(out, h, 32);
}
static void ch_mix_nonce(channel_t *c, uint64_t nonce) {
    uint8_t out[32];
    nonce_digest(c->digest, nonce, out);
    ch_update(c, out);
}
static void ch_draw_bytes(channel_t *c, uint8_t out[32]) {
    uint8_t m[64];
    memset(m, 0, sizeof(m));
    memcpy(m, c->digest, 32);
    memcpy(m + 32, &c->n_sent, 8);
    c->n_sent++;
    or_blake2s_std(m, 64, out);
}
static qm31_t ch_draw_felt(channel_t *c) {
    for (;;) {
        uint8_t b[32];
        uint32_t u[8];
        int ok = 1;
        ch_draw_bytes(c, b);
        memcpy(u, b, 32);
        for (int i = 0; i < 8; i++) ok = ok && u[i] < 2 * P_M31;
        if (!ok) continue;
        for (int i = 0; i < 4; i++) u[i] = u[i] >= P_M31 ? u[i] - P_M31 : u[i];
        qm31_t r = {{u[0], u[1]}, {u[2], u[3]}};
        return r;
    }
}
static uint32_t digest_trailing_zeros(const uint8_t d[32]) {
    for (int i = 0; i < 16; i++)
        if (d[i]) return 8 * i + (uint32_t)__builtin_ctz(d[i]);
    return 128;
}

/* ---------------------------------------------------------------- Merkle tree */
typedef struct {
    uint32_t max_log;
    size_t n_cols;
    const m31_t **cols;    /* sorted by decreasing size (stable) */
    uint32_t *col_logs;
    uint32_t **layers;     /* layers[l]: 2^l nodes of 8 words */
} tree_t;

static void tree_commit(tree_t *t, const m31_t *const *cols, const uint32_t *logs, size_t n) {
    t->n_cols = n;
    t->cols = (const m31_t **)malloc(sizeof(*t->cols) * n);
    t->col_logs = (uint32_t *)malloc(sizeof(uint32_t) * n);
    size_t k = 0;
    uint32_t max_log = 0;
    for (size_t i = 0; i < n; i++) max_log = logs[i] > max_log ? logs[i] : max_log;
    for (int l = (int)max_log; l >= 0; l--)  /* stable sort by decreasing size */
        for (size_t i = 0; i < n; i++)
            if (logs[i] == (uint32_t)l) { t->cols[k] = cols[i]; t->col_logs[k] = logs[i]; k++; }
    t->max_log = max_log;
    t->layers = (uint32_t **)calloc(max_log + 1, sizeof(uint32_t *));
    for (int l = (int)max_log; l >= 0; l--) {
        const m31_t *lc[4096];
        size_t nl = 0;
        for (size_t i = 0; i < n; i++)
            if (t->col_logs[i] == (uint32_t)l) lc[nl++] = t->cols[i];
        t->layers[l] = (uint32_t *)malloc(sizeof(uint32_t) * 8 << l);
        or_merkle_commit_on_layer((uint32_t)l, l < (int)max_log ? t->layers[l + 1] : NULL, lc, nl, t->layers[l]);
    }
}
static void tree_root(const tree_t *t, uint8_t root[32]) { memcpy(root, t->layers[0], 32); }
static void tree_free(tree_t *t) {
    for (uint32_t l = 0; l <= t->max_log; l++) free(t->layers[l]);
    free(t->layers);
    free(t->cols);
    free(t->col_logs);
}

/* Sorted, deduplicated position lists. */
typedef struct { uint64_t *v; size_t n; } pos_t;
static pos_t pos_fold(pos_t q, uint32_t k) {
    pos_t r = {(uint64_t *)malloc(sizeof(uint64_t) * (q.n ? q.n : 1)), 0};
    for (size_t i = 0; i < q.n; i++) {
        uint64_t f = q.v[i] >> k;
        if (r.n == 0 || r.v[r.n - 1] != f) r.v[r.n++] = f;
    }
    return r;
}

/* MerkleProver::decommit. queries[l] (may be empty) are the queried positions of the
 * columns of size 2^l. Writes the MerkleDecommitment (hash witness, column witness) to
 * `dec` and, when `qv` is given, the queried values per column (tree order, u64
 * column count first) to `qv`. */
static void tree_decommit(const tree_t *t, const pos_t *queries, buf_t *dec, buf_t *qv) {
    buf_t hw = {0}, cw = {0};
    buf_t *colv = (buf_t *)calloc(t->n_cols ? t->n_cols : 1, sizeof(buf_t));
    size_t *colc = (size_t *)calloc(t->n_cols ? t->n_cols : 1, sizeof(size_t));
    uint64_t n_hw = 0, n_cw = 0;
    pos_t prev = {NULL, 0};
    for (int l = (int)t->max_log; l >= 0; l--) {
        pos_t cq = queries[l];
        pos_t cur = {(uint64_t *)malloc(sizeof(uint64_t) * (prev.n + cq.n + 1)), 0};
        size_t pi = 0, ci = 0;
        for (;;) {
            /* next node: the least of the next parent and the next column query */
            int have_p = pi < prev.n, have_c = ci < cq.n;
            if (!have_p && !have_c) break;
            uint64_t node;
            if (have_p && (!have_c || (prev.v[pi] >> 1) <= cq.v[ci])) node = prev.v[pi] >> 1;
            else node = cq.v[ci];
            if (l < (int)t->max_log) {
                for (uint64_t child = 2 * node; child <= 2 * node + 1; child++) {
                    if (pi < prev.n && prev.v[pi] == child) { pi++; continue; }
                    put(&hw, t->layers[l + 1] + 8 * child, 32);
                    n_hw++;
                }
            }
            int queried = ci < cq.n && cq.v[ci] == node;
            if (queried) ci++;
            for (size_t c = 0; c < t->n_cols; c++) {
                if (t->col_logs[c] != (uint32_t)l) continue;
                if (queried) { put_u32(&colv[c], t->cols[c][node]); colc[c]++; }
                else { put_u32(&cw, t->cols[c][node]); n_cw++; }
            }
            cur.v[cur.n++] = node;
        }
        free(prev.v);
        prev = cur;
    }
    free(prev.v);
    put_u64(dec, n_hw);
    if (hw.n) put(dec, hw.p, hw.n);
    put_u64(dec, n_cw);
    if (cw.n) put(dec, cw.p, cw.n);
    if (qv) {
        put_u64(qv, t->n_cols);
        for (size_t c = 0; c < t->n_cols; c++) {
            put_u64(qv, colc[c]);
            if (colv[c].n) put(qv, colv[c].p, colv[c].n);
        }
    }
    for (size_t c = 0; c < t->n_cols; c++) free(colv[c].p);
    free(colv);
    free(colc);
    free(hw.p);
    free(cw.p);
}

/* compute_decommitment_positions_and_witness_evals (fold step 1): the folding pair of
 * every query; the partner that is not a query is a witness (4 coordinates). */
static pos_t fri_layer_positions(pos_t q, const m31_t *const col[4], buf_t *witness, uint64_t *n_witness) {
    pos_t r = {(uint64_t *)malloc(sizeof(uint64_t) * (2 * q.n + 1)), 0};
    size_t i = 0;
    while (i < q.n) {
        size_t j = i;
        while (j < q.n && (q.v[j] >> 1) == (q.v[i] >> 1)) j++;
        for (uint64_t p = q.v[i] & ~1ull; p <= (q.v[i] | 1ull); p++) {
            int is_q = 0;
            r.v[r.n++] = p;
            for (size_t k = i; k < j; k++) is_q = is_q || q.v[k] == p;
            if (!is_q) {
                for (int c = 0; c < 4; c++) put_u32(witness, col[c][p]);
                (*n_witness)++;
            }
        }
        i = j;
    }
    return r;
}

static m31_t *col_alloc(size_t n) { return (m31_t *)calloc(n ? n : 1, sizeof(m31_t)); }

/* ---------------------------------------------------------------- the prover */
int or_wide_fib_prove(const or_wide_fib_job *job, const uint32_t *a0, const uint32_t *a1, uint8_t **proof_out,
                      size_t *proof_len) {
    const uint32_t L = job->log_n_rows, N = job->n_columns, B = job->log_blowup, E = L + 1;
    if (N < 3 || N > 1024 || B < 1 || B > 4 || L < 2 || L + 1 + B > 24) return -1;
    const size_t n = (size_t)1 << L, ne = n << 1, nb = n << B, neb = ne << B;
    channel_t ch;
    memset(&ch, 0, sizeof(ch));

    /* twiddles of CanonicCoset(L + 1 + B).half_coset */
    coset_t root = or_canonic_half_coset(L + 1 + B);
    const size_t tsz = (size_t)1 << root.log_size;
    m31_t *tw = col_alloc(tsz), *itw = col_alloc(tsz);
    or_precompute_twiddles(root, tw, itw);

    /* 1. trace: rows, interpolation, evaluation, commitment */
    m31_t **poly = (m31_t **)malloc(sizeof(m31_t *) * N), **tev = (m31_t **)malloc(sizeof(m31_t *) * N);
    for (uint32_t c = 0; c < N; c++) { poly[c] = col_alloc(n); tev[c] = col_alloc(nb); }
    or_wide_fib_trace(a0, a1, n, N, poly);
    or_interpolate_many(or_canonic_half_coset(L), poly, N, itw, tsz);
    or_evaluate_many(or_canonic_half_coset(L + B), (const m31_t *const *)poly, n, tev, N, tw, tsz);
    tree_t t_trace;
    {
        uint32_t *logs = (uint32_t *)malloc(4 * N);
        for (uint32_t c = 0; c < N; c++) logs[c] = L + B;
        tree_commit(&t_trace, (const m31_t *const *)tev, logs, N);
        free(logs);
    }
    uint8_t root_trace[32];
    tree_root(&t_trace, root_trace);
    ch_mix_root(&ch, root_trace);

    /* 2. composition on CanonicCoset(L + 1) */
    const qm31_t rc = ch_draw_felt(&ch);
    m31_t **text = (m31_t **)malloc(sizeof(m31_t *) * N);
    for (uint32_t c = 0; c < N; c++) text[c] = col_alloc(ne);
    or_evaluate_many(or_canonic_half_coset(E), (const m31_t *const *)poly, n, text, N, tw, tsz);
    m31_t *den_inv = col_alloc(ne);
    or_vanishing_inverses(L, den_inv);
    qm31_t *powers = (qm31_t *)malloc(sizeof(qm31_t) * N);
    powers[0] = qone();
    for (uint32_t k = 1; k + 2 < N; k++) powers[k] = or_qm31_mul(powers[k - 1], rc);
    m31_t *comp[4], *cev[4];
    for (int k = 0; k < 4; k++) { comp[k] = col_alloc(ne); cev[k] = col_alloc(neb); }
    or_wide_fib_composition((const m31_t *const *)text, N, ne, powers, den_inv, comp);
    or_interpolate_many(or_canonic_half_coset(E), comp, 4, itw, tsz);
    or_evaluate_many(or_canonic_half_coset(E + B), (const m31_t *const *)comp, ne, cev, 4, tw, tsz);
    tree_t t_comp;
    {
        uint32_t logs[4] = {E + B, E + B, E + B, E + B};
        tree_commit(&t_comp, (const m31_t *const *)cev, logs, 4);
    }
    uint8_t root_comp[32];
    tree_root(&t_comp, root_comp);
    ch_mix_root(&ch, root_comp);

    /* 3. OODS point, sampled values, sanity check */
    spoint_t oods;
    {
        qm31_t t = ch_draw_felt(&ch), t2 = or_qm31_mul(t, t);
        qm31_t inv = or_qm31_inv(qa(t2, qone()));
        oods.x = or_qm31_mul(qs(qone(), t2), inv);
        oods.y = or_qm31_mul(qa(t, t), inv);
    }
    qm31_t *sampled = (qm31_t *)malloc(sizeof(qm31_t) * (N + 4));
    {
        const m31_t **polys = (const m31_t **)malloc(sizeof(m31_t *) * (N + 4));
        uint32_t *logs = (uint32_t *)malloc(sizeof(uint32_t) * (N + 4));
        for (uint32_t c = 0; c < N; c++) { polys[c] = poly[c]; logs[c] = L; }
        for (int k = 0; k < 4; k++) { polys[N + k] = comp[k]; logs[N + k] = E; }
        or_eval_at_point_many(polys, logs, N + 4, oods, sampled);
        free(polys);
        free(logs);
    }
    ch_mix_felts(&ch, sampled, N + 4);
    int rc_status = 0;
    {
        const qm31_t basis[4] = {{{1, 0}, {0, 0}}, {{0, 1}, {0, 0}}, {{0, 0}, {1, 0}}, {{0, 0}, {0, 1}}};
        qm31_t cv = qzero(), acc = qzero();
        for (int k = 0; k < 4; k++) cv = qa(cv, or_qm31_mul(sampled[N + k], basis[k]));
        /* coset_vanishing(CanonicCoset(L).coset, oods): shift by -initial + step/2, double x L-1 times */
        coset_t vc = or_canonic_coset(L);
        cpoint_t init = or_index_to_point(vc.initial_index), hs = or_index_to_point(vc.step_size >> 1);
        cpoint_t ninit = {init.x, init.y ? P_M31 - init.y : 0};
        cpoint_t sh = {fs(or_m31_mul(ninit.x, hs.x), or_m31_mul(ninit.y, hs.y)),
                       fa(or_m31_mul(ninit.x, hs.y), or_m31_mul(ninit.y, hs.x))};
        qm31_t x = qs(qsc(oods.x, sh.x), qsc(oods.y, sh.y));
        for (uint32_t d = 1; d < L; d++) {
            qm31_t s = or_qm31_mul(x, x);
            x = qs(qa(s, s), qone());
        }
        for (uint32_t i = 0; i + 2 < N; i++) {
            qm31_t cons = qs(qa(or_qm31_mul(sampled[i], sampled[i]), or_qm31_mul(sampled[i + 1], sampled[i + 1])),
                             sampled[i + 2]);
            acc = qa(or_qm31_mul(acc, rc), cons);
        }
        acc = or_qm31_mul(acc, or_qm31_inv(x));
        if (!qeq(acc, cv)) rc_status = -2;
    }

    /* 4. quotients: composition group (log E + B) first, then the trace group */
    const qm31_t qrc = ch_draw_felt(&ch);
    m31_t *qc[4], *qt[4];
    for (int k = 0; k < 4; k++) { qc[k] = col_alloc(neb); qt[k] = col_alloc(nb); }
    {
        uint32_t idx[1024], sz;
        qm31_t vals[1024];
        for (int k = 0; k < 4; k++) { idx[k] = (uint32_t)k; vals[k] = sampled[N + k]; }
        sz = 4;
        or_accumulate_quotients(or_canonic_half_coset(E + B), (const m31_t *const *)cev, 4, qrc, 1, &oods, &sz, idx,
                                vals, qc);
        for (uint32_t c = 0; c < N; c++) { idx[c] = c; vals[c] = sampled[c]; }
        sz = N;
        or_accumulate_quotients(or_canonic_half_coset(L + B), (const m31_t *const *)tev, N, qrc, 1, &oods, &sz, idx,
                                vals, qt);
    }
    /* FRI first layer: one tree over the 8 coordinate columns */
    tree_t t_fri0;
    {
        const m31_t *cols[8] = {qc[0], qc[1], qc[2], qc[3], qt[0], qt[1], qt[2], qt[3]};
        uint32_t logs[8] = {E + B, E + B, E + B, E + B, L + B, L + B, L + B, L + B};
        tree_commit(&t_fri0, cols, logs, 8);
    }
    uint8_t root_fri0[32];
    tree_root(&t_fri0, root_fri0);
    ch_mix_root(&ch, root_fri0);
    /* inner layers */
    const uint32_t n_layers = E - 1;  /* line domains of log E+B-1 down to B+1 */
    m31_t *lv[32][4];
    tree_t lt[32];
    uint8_t lroot[32][32];
    coset_t ldom;  /* LineDomain(Coset::half_odds(E + B - 1)): initial 2^(29-log), step 2^(31-log) */
    ldom.log_size = E + B - 1;
    ldom.initial_index = 1u << (29 - ldom.log_size);
    ldom.step_size = 1u << (31 - ldom.log_size);
    m31_t *cur[4];
    for (int k = 0; k < 4; k++) cur[k] = col_alloc((size_t)1 << ldom.log_size);
    qm31_t alpha = ch_draw_felt(&ch);
    or_fold_circle_into_line((const m31_t *const *)qc, neb, or_canonic_half_coset(E + B), alpha, cur);
    uint32_t cur_log = E + B - 1;
    int trace_folded = 0;
    for (uint32_t li = 0; cur_log > B; li++) {
        if (!trace_folded && cur_log == L + B - 1) {
            or_fold_circle_into_line((const m31_t *const *)qt, nb, or_canonic_half_coset(L + B), alpha, cur);
            trace_folded = 1;
        }
        for (int k = 0; k < 4; k++) lv[li][k] = cur[k];
        {
            uint32_t logs[4] = {cur_log, cur_log, cur_log, cur_log};
            tree_commit(&lt[li], (const m31_t *const *)cur, logs, 4);
        }
        tree_root(&lt[li], lroot[li]);
        ch_mix_root(&ch, lroot[li]);
        alpha = ch_draw_felt(&ch);
        m31_t *nxt[4];
        for (int k = 0; k < 4; k++) nxt[k] = col_alloc((size_t)1 << (cur_log - 1));
        or_fold_line((const m31_t *const *)cur, (size_t)1 << cur_log, ldom, alpha, nxt);
        for (int k = 0; k < 4; k++) cur[k] = nxt[k];
        ldom.initial_index = (ldom.initial_index * 2) & P_M31;
        ldom.step_size = (ldom.step_size * 2) & P_M31;
        ldom.log_size--;
        cur_log--;
    }
    /* last layer: 2^B values -> constant (degree bound 1) */
    qm31_t last;
    {
        size_t m = (size_t)1 << B;
        qm31_t v0 = {{cur[0][0], cur[1][0]}, {cur[2][0], cur[3][0]}};
        qm31_t sum = qzero();
        for (size_t i = 0; i < m; i++) {
            qm31_t v = {{cur[0][i], cur[1][i]}, {cur[2][i], cur[3][i]}};
            if (!qeq(v, v0)) rc_status = rc_status ? rc_status : -3;
            sum = qa(sum, v);
        }
        last = qsc(sum, or_m31_inv((m31_t)m));
        ch_mix_felts(&ch, &last, 1);
    }

    /* 5. proof of work, queries, decommitments */
    uint64_t nonce = 0;
    for (;; nonce++) {
        uint8_t d[32];
        nonce_digest(ch.digest, nonce, d);
        if (digest_trailing_zeros(d) >= job->pow_bits) break;
    }
    ch_mix_nonce(&ch, nonce);
    pos_t queries = {(uint64_t *)malloc(sizeof(uint64_t) * job->n_queries), 0};
    {
        uint32_t cnt = 0, mask = (uint32_t)(((uint64_t)1 << (E + B)) - 1);
        while (cnt < job->n_queries) {
            uint8_t b[32];
            ch_draw_bytes(&ch, b);
            for (int i = 0; i < 8 && cnt < job->n_queries; i++, cnt++) {
                uint32_t u;
                memcpy(&u, b + 4 * i, 4);
                uint64_t q = u & mask;
                /* insert into the sorted set */
                size_t k = 0;
                while (k < queries.n && queries.v[k] < q) k++;
                if (k < queries.n && queries.v[k] == q) continue;
                memmove(queries.v + k + 1, queries.v + k, sizeof(uint64_t) * (queries.n - k));
                queries.v[k] = q;
                queries.n++;
            }
        }
    }
    pos_t *tq = (pos_t *)calloc(E + B + 1, sizeof(pos_t));
    tq[E + B] = queries;
    tq[L + B] = pos_fold(queries, 1);

    buf_t out = {0};
    /* commitments */
    put_u64(&out, 2);
    put(&out, root_trace, 32);
    put(&out, root_comp, 32);
    /* sampled_values */
    put_u64(&out, 2);
    put_u64(&out, N);
    for (uint32_t c = 0; c < N; c++) { put_u64(&out, 1); put_q(&out, sampled[c]); }
    put_u64(&out, 4);
    for (int k = 0; k < 4; k++) { put_u64(&out, 1); put_q(&out, sampled[N + k]); }
    /* decommitments and queried_values */
    buf_t qv = {0};
    put_u64(&out, 2);
    tree_decommit(&t_trace, tq, &out, &qv);
    tree_decommit(&t_comp, tq, &out, &qv);
    put_u64(&out, 2);
    put(&out, qv.p, qv.n);
    free(qv.p);
    put_u64(&out, nonce);
    /* fri_proof.first_layer */
    {
        buf_t wit = {0};
        uint64_t n_wit = 0;
        pos_t *fq = (pos_t *)calloc(E + B + 1, sizeof(pos_t));
        fq[E + B] = fri_layer_positions(queries, (const m31_t *const *)qc, &wit, &n_wit);
        pos_t tq1 = pos_fold(queries, 1);
        fq[L + B] = fri_layer_positions(tq1, (const m31_t *const *)qt, &wit, &n_wit);
        free(tq1.v);
        put_u64(&out, n_wit);
        if (wit.n) put(&out, wit.p, wit.n);
        tree_decommit(&t_fri0, fq, &out, NULL);
        put(&out, root_fri0, 32);
        free(fq[E + B].v);
        free(fq[L + B].v);
        free(fq);
        free(wit.p);
    }
    /* fri_proof.inner_layers */
    put_u64(&out, n_layers);
    {
        pos_t lq = pos_fold(queries, 1);
        for (uint32_t li = 0; li < n_layers; li++) {
            buf_t wit = {0};
            uint64_t n_wit = 0;
            uint32_t lg = E + B - 1 - li;
            pos_t *fq = (pos_t *)calloc(lg + 1, sizeof(pos_t));
            fq[lg] = fri_layer_positions(lq, (const m31_t *const *)lv[li], &wit, &n_wit);
            put_u64(&out, n_wit);
            if (wit.n) put(&out, wit.p, wit.n);
            tree_decommit(&lt[li], fq, &out, NULL);
            put(&out, lroot[li], 32);
            free(fq[lg].v);
            free(fq);
            free(wit.p);
            pos_t nq = pos_fold(lq, 1);
            free(lq.v);
            lq = nq;
        }
        free(lq.v);
    }
    /* fri_proof.last_layer_poly */
    put_u64(&out, 1);
    put_q(&out, last);
    put_u32(&out, 0);

    *proof_out = out.p;
    *proof_len = out.n;

    /* cleanup */
    for (uint32_t li = 0; li < n_layers; li++) {
        tree_free(&lt[li]);
        for (int k = 0; k < 4; k++) free(lv[li][k]);
    }
    for (int k = 0; k < 4; k++) { free(cur[k]); free(qc[k]); free(qt[k]); free(comp[k]); free(cev[k]); }
    tree_free(&t_trace);
    tree_free(&t_comp);
    tree_free(&t_fri0);
    for (uint32_t c = 0; c < N; c++) { free(poly[c]); free(tev[c]); free(text[c]); }
    free(poly); free(tev); free(text);
    free(den_inv); free(powers); free(sampled);
    free(tq[L + B].v);
    free(tq);
    free(queries.v);
    free(tw); free(itw);
    return rc_status;
}

void or_free(void *p) { free(p); }
