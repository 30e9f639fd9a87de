"""PolyOps parity on the GPU against the oracle: twiddle trees, canonic ordering,
circle FFT (evaluate / interpolate / fused extension, mixed sizes), eval_at_point.
Bit-exact (integer field arithmetic)."""
import json
import os

import numpy as np
import pytest

from helpers import m31, random_circle_point, rng

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_literals.json")))


def _oc(o, c):
    return o.coset(c.initial_index, c.step_size, c.log_size)


@pytest.mark.parametrize("log_size", [1, 2, 3, 5, 8, 12, 16, 20])
def test_precompute_twiddles(stwo, oracle, log_size):
    B = stwo.CudaBackend
    coset = stwo.CanonicCoset(log_size + 1).half_coset()
    tree = B.precompute_twiddles(coset)
    tw, itw = oracle.precompute_twiddles(_oc(oracle, coset))
    assert (tree.twiddles.to_numpy() == tw).all()
    assert (tree.itwiddles.to_numpy() == itw).all()
    ref = B.precompute_twiddles_reference_abi(coset)
    assert (ref.twiddles.to_numpy() == tw).all()


def test_precompute_twiddles_golden(stwo):
    f = GOLDEN["interpolate_from_fib"]
    rc = f["root_coset"]
    tree = stwo.CudaBackend.precompute_twiddles(stwo.Coset(rc["initial_index"], rc["step_size"], rc["log_size"]))
    assert tree.twiddles.to_numpy().tolist() == f["twiddles"]
    assert tree.itwiddles.to_numpy().tolist() == f["itwiddles"]


@pytest.mark.parametrize("log_size", [1, 2, 5, 10, 11, 17])
def test_new_canonical_ordered(stwo, oracle, log_size):
    v = m31(rng(log_size), 1 << log_size)
    ev = stwo.CudaBackend.new_canonical_ordered(stwo.CanonicCoset(log_size), stwo.BaseFieldVec.from_numpy(v))
    assert (ev.values.to_numpy() == oracle.new_canonical_ordered(log_size, v)).all()


@pytest.mark.parametrize("log_size", list(range(1, 19)) + [20])
def test_interpolate_evaluate(stwo, oracle, log_size):
    """reference tests poly.rs:267 (interpolate) and :345 (evaluate) at every size."""
    B = stwo.CudaBackend
    r = rng(200 + log_size)
    coset = stwo.CanonicCoset(log_size)
    tree = B.precompute_twiddles(stwo.CanonicCoset(log_size + 2).half_coset())
    tw, itw = tree.twiddles.to_numpy(), tree.itwiddles.to_numpy()
    hc = _oc(oracle, coset.half_coset())
    vals = m31(r, 1 << log_size)
    poly = B.interpolate(stwo.CircleEvaluation(coset.circle_domain(), stwo.BaseFieldVec.from_numpy(vals)), tree)
    expect = oracle.interpolate(hc, vals, itw)
    assert (poly.coeffs.to_numpy() == expect).all()
    ev = B.evaluate(poly, coset.circle_domain(), tree)
    assert (ev.values.to_numpy() == vals).all()
    coeffs = m31(r, 1 << log_size)
    ev2 = B.evaluate(stwo.CirclePoly(stwo.BaseFieldVec.from_numpy(coeffs)), coset.circle_domain(), tree)
    assert (ev2.values.to_numpy() == oracle.evaluate(hc, coeffs, tw)).all()


def test_interpolate_golden_literal_tree(stwo, oracle):
    """poly.rs:399-614: the literal domain, values and twiddle tree."""
    f = GOLDEN["interpolate_from_fib"]
    d, rc = f["domain_half_coset"], f["root_coset"]
    tree = stwo.TwiddleTree(stwo.Coset(rc["initial_index"], rc["step_size"], rc["log_size"]),
                            stwo.BaseFieldVec.from_numpy(np.array(f["twiddles"], np.uint32)),
                            stwo.BaseFieldVec.from_numpy(np.array(f["itwiddles"], np.uint32)))
    dom = stwo.CircleDomain(stwo.Coset(d["initial_index"], d["step_size"], d["log_size"]))
    vals = np.array(f["values"], np.uint32)
    poly = stwo.CudaBackend.interpolate(stwo.CircleEvaluation(dom, stwo.BaseFieldVec.from_numpy(vals)), tree)
    expect = oracle.interpolate(oracle.coset(d["initial_index"], d["step_size"], d["log_size"]), vals,
                                np.array(f["itwiddles"], np.uint32))
    assert (poly.coeffs.to_numpy() == expect).all()
    # interpolate_2 (poly.rs:291-334) uses the same 32 values on CanonicCoset(5)
    assert f["values"] == GOLDEN["interpolate_2_values"]


@pytest.mark.parametrize("log_blowup", [1, 2])
@pytest.mark.parametrize("log_sizes", [[9] * 4, [2, 3, 4, 5, 6, 12, 15, 16, 17]])
def test_evaluate_polynomials_fused_extension(stwo, oracle, log_blowup, log_sizes):
    """evaluate_polynomials (poly.rs:128-168) with mixed column sizes; the extension
    is fused into the first FFT pass."""
    B = stwo.CudaBackend
    r = rng(7 + log_blowup)
    max_log = max(log_sizes) + log_blowup
    tree = B.precompute_twiddles(stwo.CanonicCoset(max_log).half_coset())
    tw = tree.twiddles.to_numpy()
    coeffs = [m31(r, 1 << lg) for lg in log_sizes]
    polys = [stwo.CirclePoly(stwo.BaseFieldVec.from_numpy(c)) for c in coeffs]
    evals = B.evaluate_polynomials(polys, log_blowup, tree)
    for c, lg, ev in zip(coeffs, log_sizes, evals):
        hc = _oc(oracle, stwo.CanonicCoset(lg + log_blowup).half_coset())
        assert (ev.values.to_numpy() == oracle.evaluate(hc, c, tw)).all(), lg


def test_interpolate_columns_mixed_sizes(stwo, oracle):
    B = stwo.CudaBackend
    r = rng(31)
    logs = [3, 7, 7, 11, 16, 16, 18]
    tree = B.precompute_twiddles(stwo.CanonicCoset(max(logs) + 1).half_coset())
    itw = tree.itwiddles.to_numpy()
    vals = [m31(r, 1 << lg) for lg in logs]
    cols = [stwo.CircleEvaluation(stwo.CanonicCoset(lg).circle_domain(), stwo.BaseFieldVec.from_numpy(v))
            for lg, v in zip(logs, vals)]
    polys = B.interpolate_columns(cols, tree)
    for lg, v, p in zip(logs, vals, polys):
        hc = _oc(oracle, stwo.CanonicCoset(lg).half_coset())
        assert (p.coeffs.to_numpy() == oracle.interpolate(hc, v, itw)).all()


def test_reference_abi_columns_entry_points(stwo, oracle):
    """interpolate_columns / evaluate_columns through the reference-compatible ABI
    (256 columns x 2^9, poly.rs:617-700 shapes)."""
    L = stwo._lib
    B = stwo.CudaBackend
    r = rng(5)
    log_size, ncols = 9, 256
    tree = B.precompute_twiddles(stwo.CanonicCoset(log_size + 2).half_coset())
    tw, itw = tree.twiddles.to_numpy(), tree.itwiddles.to_numpy()
    vals = [m31(r, 1 << log_size) for _ in range(ncols)]
    bufs = [stwo.BaseFieldVec.from_numpy(v) for v in vals]
    hc = _oc(oracle, stwo.CanonicCoset(log_size).half_coset())
    L.clear_error()
    L.lib().interpolate_columns(1 << (log_size - 1), L.ptr_array([b.device_ptr for b in bufs]),
                                tree.itwiddles.device_ptr, len(tree.itwiddles), ncols, 1 << log_size)
    L.check_last()
    for v, b in zip(vals[:8] + vals[-8:], bufs[:8] + bufs[-8:]):
        assert (b.to_numpy() == oracle.interpolate(hc, v, itw)).all()
    coeffs = [b.to_numpy() for b in bufs]
    sizes = L.u32_array([1 << log_size] * ncols)
    L.lib().evaluate_columns(L.u32_array([1 << (log_size - 1)] * ncols), L.ptr_array([b.device_ptr for b in bufs]),
                             tree.twiddles.device_ptr, len(tree.twiddles), ncols, sizes)
    L.check_last()
    for c, b in zip(coeffs[:8], bufs[:8]):
        assert (b.to_numpy() == oracle.evaluate(hc, c, tw)).all()


@pytest.mark.parametrize("log_size", [9, 12, 16])
def test_fft_columns_beyond_one_parameter_block(stwo, oracle, log_size):
    """More than 64 columns of one size run each pass as one launch over a device table
    of column pointers: 300 columns, interpolated in place and extended to blowup 4,
    compared with the oracle on columns around the 64-column boundaries."""
    L = stwo._lib
    lib = L.lib()
    B = stwo.CudaBackend
    r = rng(640 + log_size)
    ncols, lb = 300, 2
    tree = B.precompute_twiddles(stwo.CanonicCoset(log_size + lb).half_coset())
    tw, itw = tree.twiddles.to_numpy(), tree.itwiddles.to_numpy()
    vals = [m31(r, 1 << log_size) for _ in range(ncols)]
    bufs = [stwo.BaseFieldVec.from_numpy(v) for v in vals]
    outs = [stwo.BaseFieldVec.new_uninitialized(1 << (log_size + lb)) for _ in range(ncols)]
    logs = L.u32_array([log_size] * ncols)
    launches0 = lib.stwo_kernel_launches()
    L.check(lib.stwo_interpolate_columns(L.ptr_array([b.device_ptr for b in bufs]), logs, ncols,
                                         tree.itwiddles.device_ptr, len(tree.itwiddles), None))
    L.check(lib.stwo_extend_evaluate_columns(L.ptr_array([b.device_ptr for b in bufs]), logs,
                                             L.ptr_array([o.device_ptr for o in outs]), lb, ncols,
                                             tree.twiddles.device_ptr, len(tree.twiddles), None))
    L.check(lib.stwo_stream_synchronize(None))
    passes = 1 if log_size <= 14 else 2
    assert lib.stwo_kernel_launches() - launches0 == 2 * passes  # one launch per pass, not one per 64 columns
    hc = _oc(oracle, stwo.CanonicCoset(log_size).half_coset())
    ehc = _oc(oracle, stwo.CanonicCoset(log_size + lb).half_coset())
    for k in (0, 63, 64, 127, 128, 255, 299):
        coeffs = oracle.interpolate(hc, vals[k], itw)
        assert (bufs[k].to_numpy() == coeffs).all(), k
        assert (outs[k].to_numpy() == oracle.evaluate(ehc, coeffs, tw)).all(), k


def test_fft_log24_roundtrip_and_linearity(stwo):
    """Full size (config: 8 columns at log 24, blowup 4): interpolate then evaluate
    is the identity; evaluation is linear (checked on a sampled subset)."""
    B = stwo.CudaBackend
    r = rng(24)
    tree = B.precompute_twiddles(stwo.CanonicCoset(26).half_coset())
    v = m31(r, 1 << 24)
    col = stwo.BaseFieldVec.from_numpy(v)
    poly = B.interpolate(stwo.CircleEvaluation(stwo.CanonicCoset(24).circle_domain(), col), tree)
    ev = B.evaluate(stwo.CirclePoly(poly.coeffs.clone()), stwo.CanonicCoset(24).circle_domain(), tree)
    assert (ev.values.to_numpy() == v).all()
    # extension: the first 2^24 evaluations of the blown-up domain relate by bit-reversal
    # structure; instead check that interpolating the 2^26 evaluation returns the
    # zero-padded coefficients.
    big = B.evaluate_polynomials([poly], 2, tree)[0]
    back = B.interpolate(big, tree).coeffs.to_numpy()
    c = poly.coeffs.to_numpy()
    assert (back[: 1 << 24] == c).all() and not back[1 << 24:].any()


@pytest.mark.parametrize("log_size", [0, 1, 3, 8, 11, 12, 13, 20])
def test_eval_at_point(stwo, oracle, log_size):
    """poly.rs:372 (eval_at_point vs CpuBackend)."""
    r = rng(300 + log_size)
    c = m31(r, 1 << log_size)
    px, py = random_circle_point(r)
    got = stwo.CudaBackend.eval_at_point(stwo.CirclePoly(stwo.BaseFieldVec.from_numpy(c)), (px, py))
    assert got == oracle.eval_at_point(c, px, py)


def test_eval_at_points_batched(stwo, oracle):
    L = stwo._lib
    r = rng(77)
    logs = [4, 9, 12, 15, 15, 18]
    cs = [m31(r, 1 << lg) for lg in logs]
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cs]
    pts = [random_circle_point(r) for _ in logs]
    sp = (L.SPoint * len(logs))(*[L.SPoint(L.QM31(*x), L.QM31(*y)) for x, y in pts])
    scratch_n = L.lib().stwo_eval_at_points_scratch_bytes(L.u32_array(logs), len(logs))
    scratch = stwo.BaseFieldVec.new_uninitialized(scratch_n // 4 + 1)
    res = stwo.SecureFieldVec.new_uninitialized(len(logs))
    for _ in range(2):  # tickets are left zeroed for a second call on the same scratch
        L.check(L.lib().stwo_eval_at_points(L.ptr_array([b.device_ptr for b in bufs]), L.u32_array(logs), len(logs),
                                            sp, res.device_ptr, scratch.device_ptr, scratch_n, None))
        L.check(L.lib().stwo_stream_synchronize(None))
        got = res.to_numpy()
        for i, (c, (x, y)) in enumerate(zip(cs, pts)):
            assert tuple(int(v) for v in got[i]) == oracle.eval_at_point(c, x, y)


@pytest.mark.parametrize("groups_log", [0, 2, 3, 4])
def test_eval_at_points_every_chunk_size(stwo, oracle, groups_log):
    """Each forced CTA chunk (2^(13 + groups_log) coefficients) and the per-launch
    choice (0) give the oracle's values: sizes below a warp's 1024 coefficients
    (ragged), single groups, chunks with empty trailing groups and several chunks a
    polynomial."""
    L = stwo._lib
    lib = L.lib()
    r = rng(91 + groups_log)
    logs = [0, 3, 9, 10, 13, 14, 16, 17, 18, 19]
    cs = [m31(r, 1 << lg) for lg in logs]
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cs]
    pts = [random_circle_point(r) for _ in logs]
    sp = (L.SPoint * len(logs))(*[L.SPoint(L.QM31(*x), L.QM31(*y)) for x, y in pts])
    scratch_n = lib.stwo_eval_at_points_scratch_bytes(L.u32_array(logs), len(logs))
    scratch = stwo.BaseFieldVec.new_uninitialized(scratch_n // 4 + 1)
    res = stwo.SecureFieldVec.new_uninitialized(len(logs))
    L.check(lib.stwo_set_tunable(b"eval_at_point_groups_log", groups_log))
    try:
        for _ in range(2):  # tickets left zeroed by the first call serve the second
            L.check(lib.stwo_eval_at_points(L.ptr_array([b.device_ptr for b in bufs]), L.u32_array(logs), len(logs),
                                            sp, res.device_ptr, scratch.device_ptr, scratch_n, None))
            L.check(lib.stwo_stream_synchronize(None))
            got = res.to_numpy()
            for i, (c, (x, y)) in enumerate(zip(cs, pts)):
                assert tuple(int(v) for v in got[i]) == oracle.eval_at_point(c, x, y), logs[i]
    finally:
        lib.stwo_set_tunable(b"eval_at_point_groups_log", 0)
    with pytest.raises(L.StwoError):
        L.check(lib.stwo_set_tunable(b"eval_at_point_groups_log", 5))


def test_butterfly_probe_counts_and_checks_its_sink(stwo):
    """stwo_probe_m31_butterflies runs 16 chains a thread, 2048 threads an SM, and
    refuses a sink smaller than one word a thread."""
    import ctypes as C
    import torch
    L = stwo._lib
    lib = L.lib()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    sink = torch.zeros(2048 * sms, dtype=torch.int32, device="cuda")
    n = C.c_uint64()
    L.check(lib.stwo_probe_m31_butterflies(8, sink.data_ptr(), sink.numel(), C.byref(n), None))
    L.check(lib.stwo_stream_synchronize(None))
    assert n.value == 2048 * sms * 16 * 8
    assert int(torch.count_nonzero(sink)) > 0
    with pytest.raises(L.StwoError):
        L.check(lib.stwo_probe_m31_butterflies(8, sink.data_ptr(), sink.numel() - 1, C.byref(n), None))
