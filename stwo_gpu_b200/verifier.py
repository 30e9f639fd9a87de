"""Verifier for wide-Fibonacci proofs (stwo's verify(), restated in Python).

The prover (`stwo_wide_fib_prove`, csrc/prover.cu) emits the CommitmentSchemeProof of
stwo-prover @ ce5b975 for the wide-Fibonacci AIR of the reference's e2e test
(stwo_gpu_backend/src/examples/wide_fibonacci.rs:205-250). This module checks such a
proof the way stwo's CommitmentSchemeVerifier / FriVerifier do: it replays the
Blake2s channel, checks the composition polynomial against the constraints at the
out-of-domain point, recomputes every Merkle root from the decommitments, recomputes
the DEEP quotients at the queried positions, folds them through every FRI layer and
compares with the last layer, and checks the proof of work.

It is plain Python (integers mod 2^31 - 1) and independent of the CUDA library, so
it can check proofs anywhere. `verify` raises VerificationError on the first failure.
"""
import hashlib
import struct

P = (1 << 31) - 1
GEN = (2, 1268011823)


class VerificationError(Exception):
    pass


# ---------------------------------------------------------------- field
def cm_mul(x, y):
    return ((x[0] * y[0] - x[1] * y[1]) % P, (x[0] * y[1] + x[1] * y[0]) % P)


def cm_inv(x):
    n = pow((x[0] * x[0] + x[1] * x[1]) % P, P - 2, P)
    return (x[0] * n % P, (P - x[1]) * n % P)


def q_add(x, y):
    return tuple((a + b) % P for a, b in zip(x, y))


def q_sub(x, y):
    return tuple((a - b) % P for a, b in zip(x, y))


def q_scale(x, s):
    return tuple(a * s % P for a in x)


def q_mul(x, y):
    a, b = (x[0], x[1]), (x[2], x[3])
    c, d = (y[0], y[1]), (y[2], y[3])
    ac, bd = cm_mul(a, c), cm_mul(b, d)
    bd_r = cm_mul(bd, (2, 1))  # u^2 = 2 + i
    ad, bc = cm_mul(a, d), cm_mul(b, c)
    return ((ac[0] + bd_r[0]) % P, (ac[1] + bd_r[1]) % P, (ad[0] + bc[0]) % P, (ad[1] + bc[1]) % P)


def q_inv(x):
    a, b = (x[0], x[1]), (x[2], x[3])
    b2 = cm_mul(cm_mul(b, b), (2, 1))
    den = cm_inv(((cm_mul(a, a)[0] - b2[0]) % P, (cm_mul(a, a)[1] - b2[1]) % P))
    ra = cm_mul(a, den)
    rb = cm_mul(((P - b[0]) % P, (P - b[1]) % P), den)
    return (ra[0], ra[1], rb[0], rb[1])


def q_conj(x):  # QM31::complex_conjugate: a + b*u -> a - b*u
    return (x[0], x[1], (P - x[2]) % P, (P - x[3]) % P)


ONE = (1, 0, 0, 0)
ZERO = (0, 0, 0, 0)


# ---------------------------------------------------------------- circle
def pt_mul(p, q):
    return ((p[0] * q[0] - p[1] * q[1]) % P, (p[0] * q[1] + p[1] * q[0]) % P)


def index_to_point(k):
    k &= (1 << 31) - 1
    r, g = (1, 0), GEN
    while k:
        if k & 1:
            r = pt_mul(r, g)
        g = pt_mul(g, g)
        k >>= 1
    return r


def bit_reverse(i, log):
    return int(format(i, f"0{log}b")[::-1], 2) if log else 0


def circle_domain_point(log, pos):
    """Point at bit-reversed position pos of CanonicCoset(log).circle_domain()."""
    i = bit_reverse(pos, log)
    half = 1 << (log - 1)
    init, step = 1 << (30 - log), (1 << (32 - log)) & ((1 << 31) - 1)
    if i < half:
        return index_to_point(init + step * i)
    return index_to_point(-(init + step * (i - half)))


def line_domain_x(log, pos):
    """x of the point at bit-reversed position pos of LineDomain(Coset::half_odds(log))."""
    i = bit_reverse(pos, log)
    return index_to_point((1 << (29 - log)) + (1 << (31 - log)) * i)[0]


def deep_quotient(log, pos, values, samples, point, random_coeff):
    """One row of QuotientOps::accumulate_quotients for one sample batch: the columns'
    values at bit-reversed position pos of CanonicCoset(log), sampled at `point` with
    `samples`, combined with the powers of random_coeff."""
    ox, oy = point
    px, py = circle_domain_point(log, pos)
    num = ZERO
    alpha = ONE
    c0 = q_sub(q_conj(oy), oy)
    for v, s in zip(values, samples):
        alpha = q_mul(alpha, random_coeff)
        a = q_sub(q_conj(s), s)
        b = q_sub(q_mul(s, c0), q_mul(a, oy))
        a, b, c = q_mul(alpha, a), q_mul(alpha, b), q_mul(alpha, c0)
        num = q_add(num, q_sub(q_scale(c, v), q_add(q_scale(a, py), b)))
    den = cm_mul(((ox[0] - px) % P, ox[1]), (oy[2], oy[3]))
    den2 = cm_mul(((oy[0] - py) % P, oy[1]), (ox[2], ox[3]))
    dinv = cm_inv(((den[0] - den2[0]) % P, (den[1] - den2[1]) % P))
    return cm_mul((num[0], num[1]), dinv) + cm_mul((num[2], num[3]), dinv)


# ---------------------------------------------------------------- BLAKE2s
_IV = [0x6A09E667, 0xBB67AE85, 0x3C6EF372, 0xA54FF53A, 0x510E527F, 0x9B05688C, 0x1F83D9AB, 0x5BE0CD19]
_SIGMA = [
    [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15], [14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3],
    [11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4], [7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8],
    [9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13], [2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9],
    [12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11], [13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10],
    [6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5], [10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0],
]
M32 = 0xFFFFFFFF


def _rotr(x, c):
    return ((x >> c) | (x << (32 - c))) & M32


def compress(h, m):
    """BLAKE2s compression with zero counter and flags (RFC 7693, t = 0, f = 0)."""
    v = list(h) + list(_IV)

    def g(a, b, c, d, x, y):
        v[a] = (v[a] + v[b] + x) & M32
        v[d] = _rotr(v[d] ^ v[a], 16)
        v[c] = (v[c] + v[d]) & M32
        v[b] = _rotr(v[b] ^ v[c], 12)
        v[a] = (v[a] + v[b] + y) & M32
        v[d] = _rotr(v[d] ^ v[a], 8)
        v[c] = (v[c] + v[d]) & M32
        v[b] = _rotr(v[b] ^ v[c], 7)

    for s in _SIGMA:
        g(0, 4, 8, 12, m[s[0]], m[s[1]])
        g(1, 5, 9, 13, m[s[2]], m[s[3]])
        g(2, 6, 10, 14, m[s[4]], m[s[5]])
        g(3, 7, 11, 15, m[s[6]], m[s[7]])
        g(0, 5, 10, 15, m[s[8]], m[s[9]])
        g(1, 6, 11, 12, m[s[10]], m[s[11]])
        g(2, 7, 8, 13, m[s[12]], m[s[13]])
        g(3, 4, 9, 14, m[s[14]], m[s[15]])
    return [h[i] ^ v[i] ^ v[i + 8] for i in range(8)]


def hash_node(children, values):
    """Blake2sMerkleHasher::hash_node: zero state; children (64 bytes) then the column
    values in zero-padded 16-word chunks; digest as 8 little-endian words."""
    h = [0] * 8
    if children is not None:
        h = compress(h, list(struct.unpack("<16I", children[0] + children[1])))
    vals = list(values)
    if vals:
        vals += [0] * ((-len(vals)) % 16)
        for k in range(0, len(vals), 16):
            h = compress(h, vals[k:k + 16])
    return struct.pack("<8I", *h)


def blake2s(data):
    return hashlib.blake2s(data, digest_size=32).digest()


# ---------------------------------------------------------------- channel
class Channel:
    """Blake2sChannel with the Blake2sMerkleChannel root mixing."""

    def __init__(self):
        self.digest = bytes(32)
        self.n_sent = 0

    def _update(self, d):
        self.digest = d
        self.n_sent = 0

    def mix_root(self, root):
        self._update(blake2s(self.digest + root))

    def mix_felts(self, felts):
        self._update(blake2s(self.digest + b"".join(struct.pack("<4I", *f) for f in felts)))

    def mix_nonce(self, nonce):
        self._update(self.nonce_digest(nonce))

    def nonce_digest(self, nonce):
        h = list(struct.unpack("<8I", self.digest))
        m = [nonce & M32, nonce >> 32] + [0] * 14
        return struct.pack("<8I", *compress(h, m))

    def draw_random_bytes(self):
        out = blake2s(self.digest + struct.pack("<Q", self.n_sent) + bytes(24))
        self.n_sent += 1
        return out

    def draw_felt(self):
        while True:
            u = struct.unpack("<8I", self.draw_random_bytes())
            if all(x < 2 * P for x in u):
                return tuple(x % P for x in u[:4])


def trailing_zeros(digest):
    v = int.from_bytes(digest[:16], "little")
    return 128 if v == 0 else (v & -v).bit_length() - 1


# ---------------------------------------------------------------- proof parsing
class _Reader:
    def __init__(self, b):
        self.b, self.o = b, 0

    def take(self, n):
        if self.o + n > len(self.b):
            raise VerificationError("proof truncated")
        r = self.b[self.o:self.o + n]
        self.o += n
        return r

    def u32(self):
        return struct.unpack("<I", self.take(4))[0]

    def u64(self):
        return struct.unpack("<Q", self.take(8))[0]

    def vec_len(self, limit=1 << 24):
        n = self.u64()
        if n > limit:
            raise VerificationError("vector length out of range")
        return n

    def felt(self):
        v = struct.unpack("<I", self.take(4))[0]
        if v >= P:
            raise VerificationError("non-canonical field element")
        return v

    def qm31(self):
        return tuple(self.felt() for _ in range(4))

    def hash(self):
        return self.take(32)

    def decommitment(self):
        hw = [self.hash() for _ in range(self.vec_len())]
        cw = [self.felt() for _ in range(self.vec_len())]
        return hw, cw


def parse_proof(b):
    r = _Reader(b)
    proof = {}
    n = r.vec_len()
    proof["commitments"] = [r.hash() for _ in range(n)]
    proof["sampled_values"] = [[[r.qm31() for _ in range(r.vec_len())] for _ in range(r.vec_len())]
                               for _ in range(r.vec_len())]
    proof["decommitments"] = [r.decommitment() for _ in range(r.vec_len())]
    proof["queried_values"] = [[[r.felt() for _ in range(r.vec_len())] for _ in range(r.vec_len())]
                               for _ in range(r.vec_len())]
    proof["proof_of_work"] = r.u64()

    def layer():
        wit = [r.qm31() for _ in range(r.vec_len())]
        dec = r.decommitment()
        return {"fri_witness": wit, "decommitment": dec, "commitment": r.hash()}

    proof["fri_first"] = layer()
    proof["fri_inner"] = [layer() for _ in range(r.vec_len())]
    proof["last_layer"] = [r.qm31() for _ in range(r.vec_len())]
    proof["last_layer_log_size"] = r.u32()
    if r.o != len(b):
        raise VerificationError("trailing bytes after the proof")
    return proof


# ---------------------------------------------------------------- Merkle verification
def merkle_root(col_logs, queries, queried, decommitment):
    """MerkleVerifier::verify: the root implied by the queried values (per column, at
    the sorted queries of its size) and the decommitment. col_logs: per column (in
    tree order, decreasing). queries: {log: sorted positions}."""
    hw, cw = list(decommitment[0]), list(decommitment[1])
    hw.reverse()
    cw.reverse()
    max_log = max(col_logs)
    col_iters = [list(reversed(q)) for q in queried]
    prev = {}  # opened node -> hash of the layer below
    for layer in range(max_log, -1, -1):
        cols = [c for c, lg in enumerate(col_logs) if lg == layer]
        colq = sorted(queries.get(layer, []))
        nodes = sorted(set(colq) | {k >> 1 for k in prev})
        cur = {}
        for node in nodes:
            children = None
            if layer < max_log:
                kids = []
                for child in (2 * node, 2 * node + 1):
                    if child in prev:
                        kids.append(prev[child])
                    else:
                        if not hw:
                            raise VerificationError("hash witness too short")
                        kids.append(hw.pop())
                children = tuple(kids)
            if node in colq:
                vals = []
                for c in cols:
                    if not col_iters[c]:
                        raise VerificationError("queried values too short")
                    vals.append(col_iters[c].pop())
            else:
                if len(cw) < len(cols):
                    raise VerificationError("column witness too short")
                vals = [cw.pop() for _ in cols]
            cur[node] = hash_node(children, vals)
        prev = cur
    if hw or cw or any(col_iters):
        raise VerificationError("decommitment has unused entries")
    if list(prev) != [0]:
        raise VerificationError("merkle tree did not reduce to one root")
    return prev[0]


def fold_positions(q, n):
    out = []
    for v in q:
        f = v >> n
        if not out or out[-1] != f:
            out.append(f)
    return out


def pairs_with_witness(queries, values, witness_iter):
    """Positions of the folding pairs of `queries` and their values: queried positions
    take `values` (aligned with queries), partners take the next witness."""
    pos, vals = [], []
    qv = dict(zip(queries, values))
    seen = set()
    for q in queries:
        start = q & ~1
        if start in seen:
            continue
        seen.add(start)
        for p in (start, start + 1):
            pos.append(p)
            if p in qv:
                vals.append(qv[p])
            else:
                try:
                    vals.append(next(witness_iter))
                except StopIteration:
                    raise VerificationError("FRI witness too short") from None
    return pos, vals


# ---------------------------------------------------------------- verify
def verify(proof_bytes, log_n_rows, n_columns, log_blowup=1, n_queries=3, pow_bits=5):
    """Checks a wide-Fibonacci proof; raises VerificationError if it does not hold."""
    L, N, B = log_n_rows, n_columns, log_blowup
    E = L + 1
    pr = parse_proof(proof_bytes)
    if len(pr["commitments"]) != 2:
        raise VerificationError("expected two tree commitments")
    sv = pr["sampled_values"]
    if len(sv) != 2 or len(sv[0]) != N or len(sv[1]) != 4 or any(len(c) != 1 for t in sv for c in t):
        raise VerificationError("sampled values have the wrong shape")
    ch = Channel()
    ch.mix_root(pr["commitments"][0])
    rc = ch.draw_felt()
    ch.mix_root(pr["commitments"][1])

    # out-of-domain point and the composition check
    t = ch.draw_felt()
    t2 = q_mul(t, t)
    inv = q_inv(q_add(t2, ONE))
    ox, oy = q_mul(q_sub(ONE, t2), inv), q_mul(q_add(t, t), inv)
    trace_s = [c[0] for c in sv[0]]
    comp_s = [c[0] for c in sv[1]]
    ch.mix_felts(trace_s + comp_s)
    comp_val = ZERO
    for k, basis in enumerate([(1, 0, 0, 0), (0, 1, 0, 0), (0, 0, 1, 0), (0, 0, 0, 1)]):
        comp_val = q_add(comp_val, q_mul(comp_s[k], basis))
    # coset_vanishing(CanonicCoset(L).coset, oods): -initial + step/2 is the identity
    # for an odds coset; then x doubled L-1 times.
    init = index_to_point(1 << (30 - L))
    half_step = index_to_point(1 << (30 - L))
    sh = pt_mul((init[0], (P - init[1]) % P), half_step)
    x = q_sub(q_scale(ox, sh[0]), q_scale(oy, sh[1]))
    for _ in range(L - 1):
        s = q_mul(x, x)
        x = q_sub(q_add(s, s), ONE)
    acc = ZERO
    for i in range(N - 2):
        cons = q_sub(q_add(q_mul(trace_s[i], trace_s[i]), q_mul(trace_s[i + 1], trace_s[i + 1])), trace_s[i + 2])
        acc = q_add(q_mul(acc, rc), cons)
    if q_mul(acc, q_inv(x)) != comp_val:
        raise VerificationError("composition polynomial disagrees with the constraints at the OODS point")

    # FRI commitments
    qrc = ch.draw_felt()
    ch.mix_root(pr["fri_first"]["commitment"])
    alphas = [ch.draw_felt()]
    n_inner = E + B - 1 - B
    if len(pr["fri_inner"]) != n_inner:
        raise VerificationError("wrong number of FRI layers")
    for lay in pr["fri_inner"]:
        ch.mix_root(lay["commitment"])
        alphas.append(ch.draw_felt())
    if len(pr["last_layer"]) != 1 or pr["last_layer_log_size"] != 0:
        raise VerificationError("last layer exceeds its degree bound")
    last = pr["last_layer"][0]
    ch.mix_felts([last])

    # proof of work
    nonce = pr["proof_of_work"]
    if trailing_zeros(ch.nonce_digest(nonce)) < pow_bits:
        raise VerificationError("proof of work does not meet pow_bits")
    ch.mix_nonce(nonce)

    # queries
    D = E + B
    qs = set()
    cnt = 0
    while cnt < n_queries:
        b = ch.draw_random_bytes()
        for i in range(8):
            if cnt == n_queries:
                break
            qs.add(struct.unpack("<I", b[4 * i:4 * i + 4])[0] & ((1 << D) - 1))
            cnt += 1
    queries = sorted(qs)
    tq = {D: queries, L + B: fold_positions(queries, 1)}

    # trace and composition trees
    qv = pr["queried_values"]
    if len(qv) != 2 or len(qv[0]) != N or len(qv[1]) != 4:
        raise VerificationError("queried values have the wrong shape")
    if merkle_root([L + B] * N, tq, qv[0], pr["decommitments"][0]) != pr["commitments"][0]:
        raise VerificationError("trace tree decommitment does not match its root")
    if merkle_root([D] * 4, tq, qv[1], pr["decommitments"][1]) != pr["commitments"][1]:
        raise VerificationError("composition tree decommitment does not match its root")

    # DEEP quotients at the queried positions (accumulate_row_quotients)
    def quotient(log, pos, values, samples):
        return deep_quotient(log, pos, values, samples, (ox, oy), qrc)

    comp_q = [quotient(D, p, [qv[1][k][i] for k in range(4)], comp_s) for i, p in enumerate(tq[D])]
    trace_q = [quotient(L + B, p, [qv[0][c][i] for c in range(N)], trace_s) for i, p in enumerate(tq[L + B])]

    # FRI first layer: the pairs of both quotient columns, one tree
    first = pr["fri_first"]
    wit = iter(first["fri_witness"])
    pos_c, val_c = pairs_with_witness(tq[D], comp_q, wit)
    pos_t, val_t = pairs_with_witness(tq[L + B], trace_q, wit)
    if next(wit, None) is not None:
        raise VerificationError("FRI first-layer witness too long")
    cols = [[v[k] for v in val_c] for k in range(4)] + [[v[k] for v in val_t] for k in range(4)]
    if merkle_root([D] * 4 + [L + B] * 4, {D: pos_c, L + B: pos_t}, cols, first["decommitment"]) != \
            first["commitment"]:
        raise VerificationError("FRI first layer decommitment does not match its root")

    def fold_circle(log, pos, vals, alpha):
        out = {}
        for k in range(0, len(pos), 2):
            p = circle_domain_point(log, pos[k])
            f0 = q_add(vals[k], vals[k + 1])
            f1 = q_scale(q_sub(vals[k], vals[k + 1]), pow(p[1], P - 2, P))
            out[pos[k] >> 1] = q_add(f0, q_mul(alpha, f1))
        return out

    layer_vals = fold_circle(D, pos_c, val_c, alphas[0])  # first inner layer, log D - 1
    layer_q = fold_positions(queries, 1)
    for li, lay in enumerate(pr["fri_inner"]):
        log = D - 1 - li
        if log == L + B - 1:
            # the trace quotient joins with the previous layer's alpha (accumulate_line)
            folded = fold_circle(L + B, pos_t, val_t, alphas[li])
            a2 = q_mul(alphas[li], alphas[li])
            layer_vals = {k: q_add(q_mul(layer_vals[k], a2), folded[k]) for k in layer_vals}
        w = iter(lay["fri_witness"])
        pos, vals = pairs_with_witness(layer_q, [layer_vals[k] for k in layer_q], w)
        if next(w, None) is not None:
            raise VerificationError("FRI layer witness too long")
        cols = [[v[k] for v in vals] for k in range(4)]
        if merkle_root([log] * 4, {log: pos}, cols, lay["decommitment"]) != lay["commitment"]:
            raise VerificationError(f"FRI layer {li} decommitment does not match its root")
        alpha = alphas[li + 1]
        nxt = {}
        for k in range(0, len(pos), 2):
            xinv = pow(line_domain_x(log, pos[k]), P - 2, P)
            f0 = q_add(vals[k], vals[k + 1])
            f1 = q_scale(q_sub(vals[k], vals[k + 1]), xinv)
            nxt[pos[k] >> 1] = q_add(f0, q_mul(alpha, f1))
        layer_vals = nxt
        layer_q = fold_positions(layer_q, 1)
    for k in layer_q:
        if layer_vals[k] != last:
            raise VerificationError("FRI last layer disagrees with the folded queries")
    return True
