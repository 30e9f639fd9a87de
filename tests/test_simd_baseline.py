"""The SIMD CPU baseline (oracle/stwo_simd.cc, the SimdBackend stand-in the benchmark
times) against the scalar oracle: every vectorised function returns the oracle's
values, and its prover writes the oracle prover's proof bytes. CPU only."""
import ctypes as C

import numpy as np
import pytest

import simd as S  # oracle/simd.py
from helpers import m31, random_circle_point, random_qm31, rng


@pytest.fixture(scope="module", autouse=True)
def simd_threads(oracle):
    S.set_threads(4)
    yield


@pytest.mark.parametrize("log_size", [3, 6, 12, 17])
def test_twiddles(oracle, log_size):
    root = oracle.canonic_half_coset(log_size + 1)
    tw, itw = oracle.precompute_twiddles(root)
    stw, sitw = S.precompute_twiddles(root)
    assert (tw == stw).all() and (itw == sitw).all()


@pytest.mark.parametrize("log_size", [1, 2, 3, 4, 5, 8, 12, 13, 16, 17])
def test_fft(oracle, log_size):
    r = rng(70 + log_size)
    tw, itw = oracle.precompute_twiddles(oracle.canonic_half_coset(log_size + 2))
    hc = oracle.canonic_half_coset(log_size)
    v = m31(r, 1 << log_size)
    assert (S.interpolate(hc, v, itw) == oracle.interpolate(hc, v, itw)).all()
    c = m31(r, 1 << log_size)
    assert (S.evaluate(hc, c, tw) == oracle.evaluate(hc, c, tw)).all()
    big = oracle.canonic_half_coset(log_size + 2)
    assert (S.evaluate(big, c, tw) == oracle.evaluate(big, c, tw)).all()


@pytest.mark.parametrize("log_size,ncols,with_prev", [(2, 5, False), (3, 16, True), (4, 1, False), (4, 20, True),
                                                      (9, 64, False), (10, 0, True), (11, 33, True)])
def test_merkle_layer(oracle, log_size, ncols, with_prev):
    r = rng(log_size * 100 + ncols)
    cols = [m31(r, 1 << log_size) for _ in range(ncols)]
    prev = r.integers(0, 1 << 32, (2 << log_size) * 8, dtype=np.uint64).astype(np.uint32) if with_prev else None
    assert (S.merkle_commit_on_layer(log_size, prev, cols) == oracle.merkle_commit_on_layer(log_size, prev, cols)).all()


@pytest.mark.parametrize("log_size", [2, 3, 4, 7, 12])
def test_quotients(oracle, log_size):
    r = rng(900 + log_size)
    cols = [m31(r, 1 << log_size) for _ in range(6)]
    batches = []
    for size in (3, 1, 5):  # batches of different sizes
        x, y = random_circle_point(r)
        batches.append((x, y, [(int(r.integers(0, 6)), random_qm31(r)) for _ in range(size)]))
    hc = oracle.canonic_half_coset(log_size)
    rc = random_qm31(r)
    got = S.accumulate_quotients(hc, cols, rc, batches)
    want = oracle.accumulate_quotients(hc, cols, rc, batches)
    assert all((g == w).all() for g, w in zip(got, want))


@pytest.mark.parametrize("nc,log_ext", [(3, 2), (3, 5), (7, 6), (20, 10), (64, 8)])
def test_composition(oracle, nc, log_ext):
    r = rng(nc + 10 * log_ext)
    tr = [m31(r, 1 << log_ext) for _ in range(nc)]
    pw = m31(r, 4 * nc).reshape(nc, 4)
    di = m31(r, 1 << log_ext)
    got = S.wide_fib_composition(tr, pw, di)
    want = oracle.wide_fib_composition(tr, pw, di)
    assert all((g == w).all() for g, w in zip(got, want))


@pytest.mark.parametrize("log_size", [0, 3, 5, 6, 10, 15])
def test_eval_at_point(oracle, log_size):
    r = rng(333 + log_size)
    c = m31(r, 1 << log_size)
    x, y = random_circle_point(r)
    assert S.eval_at_point(c, x, y) == oracle.eval_at_point(c, x, y)


@pytest.mark.parametrize("log_size", [2, 5, 11, 13])
def test_folds(oracle, log_size):
    r = rng(44 + log_size)
    src = [m31(r, 1 << log_size) for _ in range(4)]
    alpha = random_qm31(r)
    dom = oracle.coset(1 << (29 - log_size), 1 << (31 - log_size), log_size)
    got, want = S.fold_line(src, dom, alpha), oracle.fold_line(src, dom, alpha)
    assert all((g == w).all() for g, w in zip(got, want))
    dst = [m31(r, 1 << (log_size - 1)) for _ in range(4)]
    hc = oracle.canonic_half_coset(log_size)
    got = S.fold_circle_into_line(dst, src, hc, alpha)
    want = oracle.fold_circle_into_line(dst, src, hc, alpha)
    assert all((g == w).all() for g, w in zip(got, want))


@pytest.mark.parametrize("log_rows", [2, 3, 8, 14])
def test_vanishing_and_trace(oracle, log_rows):
    L = oracle.lib()
    want = np.zeros(2 << log_rows, np.uint32)
    L.or_vanishing_inverses.argtypes = [C.c_uint32, C.POINTER(C.c_uint32)]
    L.or_vanishing_inverses(log_rows, want.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert (S.vanishing_inverses(log_rows) == want).all()
    r = rng(log_rows)
    a0, a1 = m31(r, 1 << log_rows), m31(r, 1 << log_rows)
    got = S.wide_fib_trace(19, a0, a1)
    assert all((g == w).all() for g, w in zip(got, oracle.wide_fib_trace(19, a0, a1)))


@pytest.mark.parametrize("t", [(2, 3, 1, 1, 0), (4, 8, 1, 3, 5), (6, 16, 2, 5, 3), (3, 20, 3, 9, 2),
                               (9, 17, 1, 7, 11), (10, 100, 2, 3, 5), (12, 64, 1, 3, 5), (13, 40, 1, 3, 8)],
                         ids=lambda j: "L%d_N%d_B%d_q%d_pow%d" % j)
def test_simd_prover_bytes_equal_oracle_prover(oracle, stwo, t):
    a0, a1 = stwo.wide_fib_inputs(t[0], 77 + t[1])
    want, rc = oracle.wide_fib_prove(t[0], t[1], a0, a1, *t[2:])
    got, src = S.wide_fib_prove(t[0], t[1], a0, a1, *t[2:])
    assert rc == src == 0
    assert got == want
