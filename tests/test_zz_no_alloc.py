"""stwo_eval_at_point_no_alloc: eval_at_point for callers that cannot allocate.

Some callers of this library cannot call cudaMalloc. A proof server that gives all
of its HBM to its own pool and admits jobs against that fixed budget is one; code
inside a process whose allocator owns the device is another; so is a loop that
cannot afford the device-wide synchronisation of cudaMalloc/cudaFree. The
reference-compatible eval_at_point allocates scratch on every call, so this entry
point keeps its partial sums in a fixed array inside the library instead.

The test calls the new entry point through the C ABI, twice in a row (the second
call sees the array as the first one left it), and compares each result with the
existing eval_at_point entry point's, exactly (field arithmetic is exact). It also
checks that sizes beyond the array's maximum (2^26 coefficients) are rejected.
This file is collected last, so a stopping run has already run every other test;
it passes alone in a fresh process as well.
"""
import pytest

from helpers import m31, random_circle_point, rng

pytestmark = pytest.mark.gpu


def _existing(stwo, buf, log_size, px, py):
    L = stwo._lib
    L.clear_error()
    r = L.lib().eval_at_point(buf.device_ptr, 1 << log_size, L.QM31(*px), L.QM31(*py))
    L.check_last()
    return r.tuple()


def _no_alloc(stwo, buf, log_size, px, py, out):
    L = stwo._lib
    L.check(L.lib().stwo_eval_at_point_no_alloc(buf.device_ptr, log_size, L.QM31(*px), L.QM31(*py),
                                                out.device_ptr, None))
    L.check(L.lib().stwo_stream_synchronize(None))
    return tuple(int(v) for v in out.to_numpy()[0])


@pytest.mark.parametrize("log_size", [0, 3, 11, 12, 17, 22])
def test_no_alloc_matches_eval_at_point_twice(stwo, log_size):
    r = rng(900 + log_size)
    out = stwo.SecureFieldVec.new_uninitialized(1)
    for call in range(2):  # two calls in a row on the shared scratch
        coeffs = m31(r, 1 << log_size)
        buf = stwo.BaseFieldVec.from_numpy(coeffs)
        px, py = random_circle_point(r)
        assert _no_alloc(stwo, buf, log_size, px, py, out) == _existing(stwo, buf, log_size, px, py), call


@pytest.mark.parametrize("log_size", [20, 22])
def test_no_alloc_matches_oracle(stwo, oracle, log_size):
    """The same value as the oracle's eval_at_point (CpuBackend restated), not only as
    the other entry point, which shares the kernel."""
    r = rng(940 + log_size)
    out = stwo.SecureFieldVec.new_uninitialized(1)
    coeffs = m31(r, 1 << log_size)
    buf = stwo.BaseFieldVec.from_numpy(coeffs)
    px, py = random_circle_point(r)
    assert _no_alloc(stwo, buf, log_size, px, py, out) == oracle.eval_at_point(coeffs, px, py)


def test_no_alloc_largest_size_then_small(stwo):
    """The maximum size (2^26 coefficients fills the scratch), then a small call."""
    r = rng(926)
    out = stwo.SecureFieldVec.new_uninitialized(1)
    big = stwo.BaseFieldVec.from_numpy(m31(r, 1 << 26))
    px, py = random_circle_point(r)
    assert _no_alloc(stwo, big, 26, px, py, out) == _existing(stwo, big, 26, px, py)
    small = stwo.BaseFieldVec.from_numpy(m31(r, 1 << 9))
    px, py = random_circle_point(r)
    assert _no_alloc(stwo, small, 9, px, py, out) == _existing(stwo, small, 9, px, py)


def test_no_alloc_rejects_sizes_beyond_its_scratch(stwo):
    L = stwo._lib
    buf = stwo.BaseFieldVec.new_zeroes(4)
    out = stwo.SecureFieldVec.new_uninitialized(1)
    L.clear_error()
    rc = L.lib().stwo_eval_at_point_no_alloc(buf.device_ptr, 27, L.QM31(0, 0, 0, 0), L.QM31(1, 0, 0, 0),
                                             out.device_ptr, None)
    assert rc == 2 and "at most 2^26" in L.last_error()
    L.clear_error()
