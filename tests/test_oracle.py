"""The oracle pinned against the reference's literal vectors and independent definitions (CPU).

Golden vectors: tests/golden/reference_literals.json, extracted from the
reference's tests by tests/golden/make_golden.py.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from helpers import P, m31, q_add, q_mul, random_circle_point, rng

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_literals.json")))


def test_circle_points_match_reference_coset_literals(oracle):
    # Coset literals in poly.rs / fri.rs pin CirclePointIndex -> CirclePoint.
    for cp in GOLDEN["circle_points"]:
        assert oracle.index_to_point(cp["index"]) == tuple(cp["point"])


def test_twiddle_tree_matches_reference_literals(oracle):
    # poly.rs:451-595: twiddles and itwiddles of root coset {8388608, 33554432, log 6}.
    f = GOLDEN["interpolate_from_fib"]
    rc = f["root_coset"]
    tw, itw = oracle.precompute_twiddles(oracle.coset(rc["initial_index"], rc["step_size"], rc["log_size"]))
    assert tw.tolist() == f["twiddles"]
    assert itw.tolist() == f["itwiddles"]
    assert GOLDEN["fold_circle_into_line_fib"]["twiddles"] == f["twiddles"]


def test_canonic_cosets_match_literals(oracle):
    # The literal root coset is CanonicCoset(7).half_coset(); the fib domain CanonicCoset(5)'s.
    hc = oracle.canonic_half_coset(7)
    rc = GOLDEN["interpolate_from_fib"]["root_coset"]
    assert (hc.initial_index, hc.step_size, hc.log_size) == (rc["initial_index"], rc["step_size"], rc["log_size"])
    d = GOLDEN["interpolate_from_fib"]["domain_half_coset"]
    hc5 = oracle.canonic_half_coset(5)
    assert (hc5.initial_index, hc5.step_size, hc5.log_size) == (d["initial_index"], d["step_size"], d["log_size"])


@pytest.mark.parametrize("n", [0, 1, 3, 55, 63, 64, 65, 127, 128, 129, 1000, 4096])
def test_blake2s_compression_matches_hashlib(oracle, n):
    data = bytes(rng(n).integers(0, 256, n, dtype=np.uint8))
    assert oracle.blake2s_std(data) == hashlib.blake2s(data).digest()


@pytest.mark.parametrize("log_n", range(1, 11))
def test_fft_equals_definition(oracle, log_n):
    """evaluate (CpuBackend's butterfly network) == the circle polynomial
    evaluated at every domain point in bit-reversed order; interpolate inverts it."""
    r = rng(100 + log_n)
    hc = oracle.canonic_half_coset(log_n)
    tw, itw = oracle.precompute_twiddles(oracle.canonic_half_coset(log_n + 2))
    for coeff_log in sorted({max(0, log_n - 2), log_n}):
        c = m31(r, 1 << coeff_log)
        ev = oracle.evaluate(hc, c, tw)
        assert (ev == oracle.evaluate_direct(hc, c)).all()
        if coeff_log == log_n:
            assert (oracle.interpolate(hc, ev, itw) == c).all()


def test_interpolate_literal_inputs_roundtrip(oracle):
    # poly.rs:399-614 runs CpuBackend::interpolate on these literals with the literal tree.
    f = GOLDEN["interpolate_from_fib"]
    d = f["domain_half_coset"]
    hc = oracle.coset(d["initial_index"], d["step_size"], d["log_size"])
    vals = np.array(f["values"], np.uint32)
    coeffs = oracle.interpolate(hc, vals, np.array(f["itwiddles"], np.uint32))
    assert (oracle.evaluate(hc, coeffs, np.array(f["twiddles"], np.uint32)) == vals).all()
    assert (oracle.evaluate_direct(hc, coeffs) == vals).all()


def test_new_canonical_ordered_semantics(oracle):
    # Value i of a canonic-coset evaluation lands where the bit-reversed circle
    # domain holds the same point.
    L = 7
    vals = np.arange(1 << L, dtype=np.uint32)
    out = oracle.new_canonical_ordered(L, vals)
    cc = oracle.canonic_coset(L)
    hc = oracle.canonic_half_coset(L)
    lib = oracle.lib()
    for pos in range(1 << L):
        dom_pt = lib.or_circle_domain_at(hc, oracle.lib().or_bit_reverse_index(pos, L))
        can_pt = lib.or_coset_at(cc, int(out[pos]))
        assert (dom_pt.x, dom_pt.y) == (can_pt.x, can_pt.y)


def test_eval_at_point_matches_fft(oracle):
    L = 6
    r = rng(7)
    hc = oracle.canonic_half_coset(L)
    tw, _ = oracle.precompute_twiddles(hc)
    c = m31(r, 1 << L)
    ev = oracle.evaluate(hc, c, tw)
    lib = oracle.lib()
    for pos in [0, 1, 5, 33, 63]:
        p = lib.or_circle_domain_at(hc, lib.or_bit_reverse_index(pos, L))
        v = oracle.eval_at_point(c, (p.x, 0, 0, 0), (p.y, 0, 0, 0))
        assert v == (int(ev[pos]), 0, 0, 0)


def test_fold_line_identity(oracle):
    """fri.rs:142-192: folding the evaluation of f = f_e(pi(x)) + x f_o(pi(x)) gives
    2 (f_e + alpha f_o) on the doubled domain."""
    g = GOLDEN["fold_line_identity"]
    deg = g["degree"]
    even = [(v, 0, 0, 0) for v in g["even"]]
    odd = [(v, 0, 0, 0) for v in g["odd"]]
    alpha = (g["alpha"], 0, 0, 0)
    coeffs = np.array(even + odd, np.uint32)
    log_deg = deg.bit_length() - 1
    # LineDomain::new(Coset::half_odds(log deg)): initial 2^(31-(log+2)), step 2^(31-log)
    line = oracle.coset(1 << (31 - (log_deg + 2)), 1 << (31 - log_deg), log_deg)
    vals = [oracle.line_eval_at_point(coeffs, (oracle.lib().or_coset_at(line, i).x, 0, 0, 0)) for i in range(deg)]
    vals = oracle.bit_reverse(np.array(vals, np.uint32))
    folded = oracle.fold_line([vals[:, c] for c in range(4)], line, alpha)
    folded = oracle.bit_reverse(np.stack(folded, axis=1))
    dbl = oracle.coset_double(line)
    for i in range(deg // 2):
        x = (oracle.lib().or_coset_at(dbl, i).x, 0, 0, 0)
        fe = oracle.line_eval_at_point(np.array(even, np.uint32), x)
        fo = oracle.line_eval_at_point(np.array(odd, np.uint32), x)
        expect = q_add(fe, q_mul(alpha, fo))
        expect = q_add(expect, expect)
        assert tuple(int(v) for v in folded[i]) == expect


def test_accumulation_literals(oracle):
    n = 16
    for case in GOLDEN["accumulation"]:
        left = [np.full(n, v, np.uint32) for v in case["left"]]
        right = [np.full(n, v, np.uint32) for v in case["right"]]
        out = oracle.accumulate(left, right)
        assert [int(c[0]) for c in out] == case["expected"]
        assert all((c == c[0]).all() for c in out)


def _interp4(oracle, cols, hc, itw):
    return [oracle.interpolate(hc, c, itw) for c in cols]


def test_quotients_are_low_degree(oracle):
    """A DEEP quotient of columns sampled at their true values is a polynomial of
    degree below the trace size, so its top coefficients on the blown-up domain
    vanish (the property QuotientOps exists for)."""
    r = rng(11)
    trace_log, blow = 5, 1
    L = trace_log + blow
    hc = oracle.canonic_half_coset(L)
    tw, itw = oracle.precompute_twiddles(hc)
    polys = [m31(r, 1 << trace_log) for _ in range(3)]
    cols = [oracle.evaluate(hc, c, tw) for c in polys]
    batches = []
    for b in range(2):
        px, py = random_circle_point(r)
        batches.append((px, py, [(ci, oracle.eval_at_point(polys[ci], px, py)) for ci in range(3)]))
    rc = tuple(int(v) for v in m31(r, 4))
    out = oracle.accumulate_quotients(hc, cols, rc, batches)
    for coord in _interp4(oracle, out, hc, itw):
        assert (coord[(1 << trace_log):] == 0).all()
    # A wrong sampled value breaks the property.
    bad = [(batches[0][0], batches[0][1], [(0, q_add(batches[0][2][0][1], (1, 0, 0, 0)))])]
    out_bad = oracle.accumulate_quotients(hc, cols, rc, bad)
    assert any((c[(1 << trace_log):] != 0).any() for c in _interp4(oracle, out_bad, hc, itw))


def test_fri_folds_keep_low_degree(oracle):
    """Folding the evaluation of a low-degree circle polynomial (circle -> line) and
    then a line fold keeps the degree bound halving (FRI soundness property)."""
    r = rng(12)
    L, deg_log = 7, 4
    hc = oracle.canonic_half_coset(L)
    tw, itw = oracle.precompute_twiddles(hc)
    cols = []
    for _ in range(4):
        cols.append(oracle.evaluate(hc, m31(r, 1 << deg_log), tw))
    alpha = tuple(int(v) for v in m31(r, 4))
    line = [np.zeros(1 << (L - 1), np.uint32) for _ in range(4)]
    line = oracle.fold_circle_into_line(line, cols, hc, alpha)
    # the line evaluation over LineDomain(half coset) must come from a degree < 2^(deg_log-1) line poly
    line_dom = hc
    folded = oracle.fold_line(line, line_dom, alpha)
    folded2 = oracle.fold_line(folded, oracle.coset_double(line_dom), alpha)
    # after two line folds of a degree-2^3 line function: degree < 2^1 -> values on the
    # 2^(L-3)-point domain are affine in the bit-reversed basis: check by refolding to a constant.
    cur, dom = folded2, oracle.coset_double(oracle.coset_double(line_dom))
    while len(cur[0]) > 2:
        cur = oracle.fold_line(cur, dom, alpha)
        dom = oracle.coset_double(dom)
    f = oracle.fold_line(cur, dom, alpha)
    assert len(f[0]) == 1
    # a constant line function folds to 2*const: check degree through one more level
    # by verifying the pre-final layer is constant.
    assert all((c == c[0]).all() for c in cur)


def test_wide_fib_trace_and_composition(oracle):
    """A valid wide-Fibonacci trace makes every constraint vanish on the trace
    domain, so the composition is a low-degree polynomial on the extended domain."""
    r = rng(13)
    n_cols, log_rows = 8, 5
    a, b = m31(r, 1 << log_rows), m31(r, 1 << log_rows)
    trace = oracle.wide_fib_trace(n_cols, a, b)
    for i in range(2, n_cols):
        assert ((trace[i].astype(np.uint64) - ((trace[i - 1].astype(np.uint64) ** 2 + trace[i - 2].astype(np.uint64) ** 2) % P)) % P == 0).all()
    trace_hc, ext_hc = oracle.canonic_half_coset(log_rows), oracle.canonic_half_coset(log_rows + 1)
    tw, itw = oracle.precompute_twiddles(ext_hc)
    polys = [oracle.interpolate(trace_hc, c, itw) for c in trace]
    ext = [oracle.evaluate(ext_hc, p, tw) for p in polys]
    zero = oracle.canonic_coset(log_rows)
    lib = oracle.lib()
    den = np.array([oracle.coset_vanishing(zero, (lambda p: (p.x, p.y))(lib.or_circle_domain_at(ext_hc, i)))
                    for i in range(1 << (log_rows + 1))], np.uint32)
    den = oracle.bit_reverse(den)
    den_inv = oracle.batch_inverse_m31(den)
    powers = np.array([oracle.qm31_pow(tuple(int(v) for v in m31(r, 4)), 1)] * (n_cols - 2), np.uint32)
    comp = oracle.wide_fib_composition(ext, powers, den_inv)
    # numerator degree 2*2^log_rows over a vanishing polynomial of degree 2^log_rows:
    # nothing above basis index 2^log_rows survives.
    for coord in comp:
        co = oracle.interpolate(ext_hc, coord, itw)
        assert (co[(1 << log_rows) + 1:] == 0).all()
    # breaking one trace cell breaks it
    ext[3] = ext[3].copy()
    ext[3][5] ^= 1
    bad = oracle.wide_fib_composition(ext, powers, den_inv)
    assert any((oracle.interpolate(ext_hc, c, itw)[(1 << log_rows) + 1:] != 0).any() for c in bad)


def test_batch_inverse(oracle):
    r = rng(14)
    v = m31(r, 1000)
    v[v == 0] = 1
    inv = oracle.batch_inverse_m31(v)
    assert ((v.astype(np.uint64) * inv) % P == 1).all()
    q = m31(r, 400).reshape(100, 4)
    qi = oracle.batch_inverse_qm31(q)
    for x, y in zip(q, qi):
        assert q_mul(tuple(int(t) for t in x), tuple(int(t) for t in y)) == (1, 0, 0, 0)
