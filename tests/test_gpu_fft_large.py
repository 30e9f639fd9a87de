"""Circle FFT at the large sizes, element for element.

Above 2^14 points every transform runs a bottom pass of 14 layers and strided passes
over 2^14-element tiles; which strided template runs depends on the size
(plan_passes in csrc/fft.cu): 2^20 uses a 6-layer pass, 2^21..2^24 a 7..10-layer pass,
2^25 and 2^26 two passes. These tests compare interpolate, evaluate and the fused
extension (blowup 2 and 4, the 8 x 2^24 FFT step's shape) at every one of those sizes
with the oracle (CpuBackend restated in C, multi-threaded) and, for whole 8-column
steps, with the reference's own CUDA library built unmodified from its sources.
Bit-exact: all arithmetic is exact mod 2^31 - 1."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import m31, rng

pytestmark = pytest.mark.gpu

TOP = 26  # the largest domain: 2^24 coefficients at blowup 4


def _oc(o, c):
    return o.coset(c.initial_index, c.step_size, c.log_size)


@pytest.fixture(scope="module")
def big_tree(stwo, oracle):
    """The twiddle tree of the 2^26 domain (2^25 entries), checked whole against the
    oracle's tree before any transform uses it."""
    oracle.set_threads(os.cpu_count() or 1)
    try:
        root = stwo.CanonicCoset(TOP).half_coset()
        tree = stwo.CudaBackend.precompute_twiddles(root)
        tw, itw = oracle.precompute_twiddles(_oc(oracle, root))
        assert (tree.twiddles.to_numpy() == tw).all()
        assert (tree.itwiddles.to_numpy() == itw).all()
        yield tree, tw, itw
    finally:
        oracle.set_threads(1)


@pytest.fixture()
def threads(oracle):
    oracle.set_threads(os.cpu_count() or 1)
    yield
    oracle.set_threads(1)


@pytest.mark.parametrize("log_size", [20, 21, 22, 23, 24])
def test_large_fft_and_extension_match_oracle(stwo, oracle, big_tree, threads, log_size):
    """Two columns of 2^log_size: interpolate (interpolate_columns), evaluate on the same
    domain, and the fused extension to blowup 2 and 4 (evaluate_polynomials), each
    against the oracle."""
    B = stwo.CudaBackend
    tree, tw, itw = big_tree
    r = rng(2400 + log_size)
    vals = [m31(r, 1 << log_size) for _ in range(2)]
    dom = stwo.CanonicCoset(log_size).circle_domain()
    hc = _oc(oracle, stwo.CanonicCoset(log_size).half_coset())
    polys = B.interpolate_columns([stwo.CircleEvaluation(dom, stwo.BaseFieldVec.from_numpy(v)) for v in vals], tree)
    coeffs = []
    for v, p in zip(vals, polys):
        want = oracle.interpolate(hc, v, itw)
        got = p.coeffs.to_numpy()
        assert (got == want).all(), f"interpolate 2^{log_size}: first mismatch at {np.argmax(got != want)}"
        coeffs.append(want)
    # evaluate on the transform's own domain: a fresh polynomial, not the round trip
    c2 = m31(r, 1 << log_size)
    ev = B.evaluate(stwo.CirclePoly(stwo.BaseFieldVec.from_numpy(c2)), dom, tree).values.to_numpy()
    assert (ev == oracle.evaluate(hc, c2, tw)).all(), f"evaluate 2^{log_size}"
    for log_blowup in (1, 2):
        evals = B.evaluate_polynomials(polys, log_blowup, tree)
        ehc = _oc(oracle, stwo.CanonicCoset(log_size + log_blowup).half_coset())
        for c, e in zip(coeffs, evals):
            want = oracle.evaluate(ehc, c, tw)
            got = e.values.to_numpy()
            assert (got == want).all(), \
                f"extension 2^{log_size} -> 2^{log_size + log_blowup}: first mismatch at {np.argmax(got != want)}"


@pytest.mark.parametrize("log_size", [25, 26])
def test_two_strided_pass_sizes_match_oracle(stwo, oracle, big_tree, threads, log_size):
    """2^25 and 2^26 points take two strided passes above the bottom pass."""
    B = stwo.CudaBackend
    tree, tw, itw = big_tree
    r = rng(2500 + log_size)
    dom = stwo.CanonicCoset(log_size).circle_domain()
    hc = _oc(oracle, stwo.CanonicCoset(log_size).half_coset())
    v = m31(r, 1 << log_size)
    got = B.interpolate(stwo.CircleEvaluation(dom, stwo.BaseFieldVec.from_numpy(v)), tree).coeffs.to_numpy()
    assert (got == oracle.interpolate(hc, v, itw)).all()
    c = m31(r, 1 << log_size)
    got = B.evaluate(stwo.CirclePoly(stwo.BaseFieldVec.from_numpy(c)), dom, tree).values.to_numpy()
    assert (got == oracle.evaluate(hc, c, tw)).all()


@pytest.mark.parametrize("log_size", [20, 22, 24])
def test_fft_step_matches_reference_library(stwo, big_tree, log_size):
    """The whole FFT step of the bench (8 columns: interpolate, then extend to blowup 4
    and evaluate) against the reference's own CUDA library on the same device inputs:
    its interpolate_columns, then, as PolyOps::evaluate_polynomials does
    (poly.rs:128-168), every polynomial copied into a zeroed 2^(L+2) buffer and
    evaluate_columns."""
    import reflib
    if not reflib.available():
        pytest.skip("oracle/_ref/libgpubackend_ref.so not built (make -f oracle/ref.mk)")
    R = reflib.lib()
    L = stwo._lib
    lib = L.lib()
    tree, _, _ = big_tree
    ncols, lb = 8, 2
    N = log_size + lb
    r = rng(2600 + log_size)
    vals = [m31(r, 1 << log_size) for _ in range(ncols)]
    ours = [stwo.BaseFieldVec.from_numpy(v) for v in vals]
    refs = [stwo.BaseFieldVec.from_numpy(v) for v in vals]
    outs = [stwo.BaseFieldVec.new_uninitialized(1 << N) for _ in range(ncols)]
    tsz = len(tree.twiddles)
    logs = L.u32_array([log_size] * ncols)
    L.check(lib.stwo_interpolate_columns(L.ptr_array([b.device_ptr for b in ours]), logs, ncols,
                                         tree.itwiddles.device_ptr, tsz, None))
    L.check(lib.stwo_extend_evaluate_columns(L.ptr_array([b.device_ptr for b in ours]), logs,
                                             L.ptr_array([b.device_ptr for b in outs]), lb, ncols,
                                             tree.twiddles.device_ptr, tsz, None))
    L.check(lib.stwo_stream_synchronize(None))
    R.interpolate_columns(1 << (log_size - 1), (C.c_void_p * ncols)(*[b.device_ptr for b in refs]),
                          tree.itwiddles.device_ptr, tsz, ncols, 1 << log_size)
    ext = [stwo.BaseFieldVec.from_numpy(np.zeros(1 << N, np.uint32)) for _ in range(ncols)]
    for b, e in zip(refs, ext):
        R.copy_uint32_t_vec_from_device_to_device(b.device_ptr, e.device_ptr, 1 << log_size)
    R.evaluate_columns((C.c_int * ncols)(*([1 << (N - 1)] * ncols)),
                       (C.c_void_p * ncols)(*[e.device_ptr for e in ext]), tree.twiddles.device_ptr, tsz, ncols,
                       (C.c_int * ncols)(*([1 << N] * ncols)))
    for k in range(ncols):
        assert (ours[k].to_numpy() == refs[k].to_numpy()).all(), f"interpolate column {k}"
        assert (outs[k].to_numpy() == ext[k].to_numpy()).all(), f"blowup-4 evaluation column {k}"


@pytest.mark.parametrize("max_layers", [4, 5, 7])
def test_radix_split_setting_gives_the_same_transform(stwo, oracle, big_tree, threads, max_layers):
    """The FFT radix split (fft_max_strided_layers: at most this many layers a strided
    pass; fewer means more passes) changes the pass plan, not the values: 2^22 and
    2^24 transforms against the oracle under each setting."""
    L = stwo._lib
    lib = L.lib()
    B = stwo.CudaBackend
    tree, tw, itw = big_tree
    L.check(lib.stwo_set_tunable(b"fft_max_strided_layers", max_layers))
    try:
        for log_size in (22, 24):
            r = rng(2700 + log_size + max_layers)
            dom = stwo.CanonicCoset(log_size).circle_domain()
            hc = _oc(oracle, stwo.CanonicCoset(log_size).half_coset())
            v = m31(r, 1 << log_size)
            poly = B.interpolate(stwo.CircleEvaluation(dom, stwo.BaseFieldVec.from_numpy(v)), tree)
            coeffs = poly.coeffs.to_numpy()
            assert (coeffs == oracle.interpolate(hc, v, itw)).all(), log_size
            ev = B.evaluate_polynomials([poly], 2, tree)[0].values.to_numpy()
            ehc = _oc(oracle, stwo.CanonicCoset(log_size + 2).half_coset())
            assert (ev == oracle.evaluate(ehc, coeffs, tw)).all(), log_size
    finally:
        lib.stwo_set_tunable(b"fft_max_strided_layers", 10)
