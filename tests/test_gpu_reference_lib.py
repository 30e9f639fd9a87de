"""Cross-check against the reference's own CUDA library (built unmodified from its
sources into oracle/_ref by oracle/ref.mk): on the same device inputs our kernels and
the reference kernels must agree element for element. The reference's Rust tests
assert these reference functions equal CpuBackend, so this pins our GPU path to the
reference itself, in addition to the oracle. Sizes stay where the reference's memory
accesses are in bounds (see oracle/reflib.py)."""
import ctypes as C

import numpy as np
import pytest

from helpers import m31, m31_nonzero, random_circle_point, random_qm31, rng

pytestmark = pytest.mark.gpu

import reflib  # noqa: E402  (oracle/reflib.py)

if not reflib.available():
    pytest.skip("oracle/_ref/libgpubackend_ref.so not built (make -f oracle/ref.mk)", allow_module_level=True)


def _ptrs(vecs):
    return (C.c_void_p * len(vecs))(*[v.device_ptr for v in vecs])


@pytest.fixture(scope="module")
def R():
    return reflib.lib()


def test_precompute_twiddles_matches_reference(stwo, R):
    coset = stwo.CanonicCoset(13).half_coset()
    ours = stwo.CudaBackend.precompute_twiddles(coset).twiddles.to_numpy()
    p = R.precompute_twiddles(reflib.Point(*coset.initial), reflib.Point(*coset.step), coset.size())
    ref = stwo.BaseFieldVec(p, coset.size()).to_numpy()
    assert (ours == ref).all()


@pytest.mark.parametrize("log_size", [3, 10, 16])
def test_fft_matches_reference(stwo, R, log_size):
    B = stwo.CudaBackend
    r = rng(log_size)
    coset = stwo.CanonicCoset(log_size)
    tree = B.precompute_twiddles(stwo.CanonicCoset(log_size + 1).half_coset())
    vals = m31(r, 1 << log_size)
    ours = B.interpolate(stwo.CircleEvaluation(coset.circle_domain(), stwo.BaseFieldVec.from_numpy(vals)), tree)
    ref = stwo.BaseFieldVec.from_numpy(vals)
    R.interpolate(1 << (log_size - 1), ref.device_ptr, tree.itwiddles.device_ptr, len(tree.itwiddles), 1 << log_size)
    assert (ours.coeffs.to_numpy() == ref.to_numpy()).all()
    ev = B.evaluate(stwo.CirclePoly(ref.clone()), coset.circle_domain(), tree)
    R.evaluate(1 << (log_size - 1), ref.device_ptr, tree.twiddles.device_ptr, len(tree.twiddles), 1 << log_size)
    assert (ev.values.to_numpy() == ref.to_numpy()).all()


def test_fft_columns_match_reference(stwo, R):
    B = stwo.CudaBackend
    r = rng(9)
    log_size, ncols, blow = 12, 16, 2
    tree = B.precompute_twiddles(stwo.CanonicCoset(log_size + blow).half_coset())
    vals = [m31(r, 1 << log_size) for _ in range(ncols)]
    ours = B.interpolate_columns([stwo.CircleEvaluation(stwo.CanonicCoset(log_size).circle_domain(),
                                                        stwo.BaseFieldVec.from_numpy(v)) for v in vals], tree)
    refs = [stwo.BaseFieldVec.from_numpy(v) for v in vals]
    R.interpolate_columns(1 << (log_size - 1), _ptrs(refs), tree.itwiddles.device_ptr, len(tree.itwiddles), ncols,
                          1 << log_size)
    for o, f in zip(ours, refs):
        assert (o.coeffs.to_numpy() == f.to_numpy()).all()
    evals = B.evaluate_polynomials(ours, blow, tree)
    ext = [B.extend(p, log_size + blow).coeffs for p in ours]
    sizes = (C.c_int * ncols)(*([1 << (log_size + blow)] * ncols))
    dom = (C.c_int * ncols)(*([1 << (log_size + blow - 1)] * ncols))
    R.evaluate_columns(dom, _ptrs(ext), tree.twiddles.device_ptr, len(tree.twiddles), ncols, sizes)
    for e, f in zip(evals, ext):
        assert (e.values.to_numpy() == f.to_numpy()).all()


def test_batch_inverse_and_bit_reverse_match_reference(stwo, R):
    B = stwo.CudaBackend
    r = rng(3)
    v = m31_nonzero(r, 1 << 16)
    src = stwo.BaseFieldVec.from_numpy(v)
    ours, ref = stwo.BaseFieldVec.new_uninitialized(len(v)), stwo.BaseFieldVec.new_uninitialized(len(v))
    B.batch_inverse(src, ours)
    R.batch_inverse_base_field(src.device_ptr, ref.device_ptr, len(v))
    assert (ours.to_numpy() == ref.to_numpy()).all()
    q = m31(r, 4 << 14).reshape(-1, 4)
    q[:, 0] |= 1
    qs = stwo.SecureFieldVec.from_numpy(q)
    qo, qr = stwo.SecureFieldVec.new_uninitialized(len(q)), stwo.SecureFieldVec.new_uninitialized(len(q))
    B.batch_inverse(qs, qo)
    R.batch_inverse_secure_field(qs.device_ptr, qr.device_ptr, len(q))
    assert (qo.to_numpy() == qr.to_numpy()).all()
    a, b = stwo.BaseFieldVec.from_numpy(v), stwo.BaseFieldVec.from_numpy(v)
    B.bit_reverse_column(a)
    R.bit_reverse_base_field(b.device_ptr, len(v))
    assert (a.to_numpy() == b.to_numpy()).all()
    qa, qb = stwo.SecureFieldVec.from_numpy(q), stwo.SecureFieldVec.from_numpy(q)
    B.bit_reverse_column(qa)
    R.bit_reverse_secure_field(qb.device_ptr, len(q))
    assert (qa.to_numpy() == qb.to_numpy()).all()


def test_folds_match_reference(stwo, R):
    B = stwo.CudaBackend
    r = rng(4)
    n = 1 << 14
    alpha = random_qm31(r)
    cols = [m31(r, n) for _ in range(4)]
    domain = stwo.LineDomain(stwo.CanonicCoset(15).half_coset())
    tree = B.precompute_twiddles(domain.coset)
    ours = B.fold_line(stwo.LineEvaluation(domain, stwo.SecureColumnByCoords.from_numpy(cols)), alpha, tree)
    src = stwo.SecureColumnByCoords.from_numpy(cols)
    out = stwo.SecureColumnByCoords.uninitialized(n // 2)
    R.fold_line(tree.itwiddles.device_ptr, len(tree.itwiddles) - n, n, src.ptrs(), reflib.QM31(*alpha), out.ptrs())
    for a, b in zip(ours.values.to_numpy(), out.to_numpy()):
        assert (a == b).all()
    circle = stwo.CanonicCoset(14).circle_domain()
    line = stwo.LineDomain(circle.half_coset)
    ctree = B.precompute_twiddles(line.coset)
    dst0 = [m31(r, n // 2) for _ in range(4)]
    d1 = stwo.LineEvaluation(line, stwo.SecureColumnByCoords.from_numpy(dst0))
    B.fold_circle_into_line(d1, stwo.SecureEvaluation(circle, stwo.SecureColumnByCoords.from_numpy(cols)), alpha, ctree)
    d2 = stwo.SecureColumnByCoords.from_numpy(dst0)
    src2 = stwo.SecureColumnByCoords.from_numpy(cols)  # kept alive until the reference call returns
    R.fold_circle_into_line(ctree.itwiddles.device_ptr, ctree.root_coset.size() - line.size(), n, src2.ptrs(),
                            reflib.QM31(*alpha), d2.ptrs())
    for a, b in zip(d1.values.to_numpy(), d2.to_numpy()):
        assert (a == b).all()


def test_merkle_matches_reference(stwo, R):
    r = rng(5)
    cols = [m31(r, 1 << 12) for _ in range(35)]
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cols]
    prev = stwo.CudaBackend.commit_on_layer(12, None, bufs)
    dev = R.copy_device_pointer_vec_from_host_to_device(_ptrs(bufs), len(bufs))
    ref_prev = stwo.Blake2sHashVec.new_uninitialized(1 << 12)
    R.commit_on_first_layer(1 << 12, len(bufs), dev, ref_prev.device_ptr)
    R.cuda_free_memory(dev)
    assert (prev.to_numpy() == ref_prev.to_numpy()).all()
    cols2 = [m31(r, 1 << 11) for _ in range(16)]
    bufs2 = [stwo.BaseFieldVec.from_numpy(c) for c in cols2]
    ours = stwo.CudaBackend.commit_on_layer(11, prev, bufs2)
    dev = R.copy_device_pointer_vec_from_host_to_device(_ptrs(bufs2), len(bufs2))
    ref = stwo.Blake2sHashVec.new_uninitialized(1 << 11)
    R.commit_on_layer_with_previous(1 << 11, len(bufs2), dev, ref_prev.device_ptr, ref.device_ptr)
    R.cuda_free_memory(dev)
    assert (ours.to_numpy() == ref.to_numpy()).all()


def test_accumulate_and_quotients_match_reference(stwo, R):
    B = stwo.CudaBackend
    r = rng(6)
    n = 1 << 14
    l0, r0 = [m31(r, n) for _ in range(4)], [m31(r, n) for _ in range(4)]
    a = stwo.SecureColumnByCoords.from_numpy(l0)
    B.accumulate(a, stwo.SecureColumnByCoords.from_numpy(r0))
    b = stwo.SecureColumnByCoords.from_numpy(l0)
    rb = stwo.SecureColumnByCoords.from_numpy(r0)  # kept alive until the reference call returns
    R.accumulate(n, b.ptrs(), rb.ptrs())
    for x, y in zip(a.to_numpy(), b.to_numpy()):
        assert (x == y).all()
    # quotients: equal batch sizes (the reference mis-indexes line coefficients otherwise)
    log_size, ncols = 13, 6
    domain = stwo.CanonicCoset(log_size).circle_domain()
    cols = [stwo.CircleEvaluation(domain, stwo.BaseFieldVec.from_numpy(m31(r, 1 << log_size))) for _ in range(ncols)]
    rc = random_qm31(r)
    batches = []
    for _ in range(3):
        pt = random_circle_point(r)
        batches.append(stwo.ColumnSampleBatch(pt, [(i, random_qm31(r)) for i in range(ncols)]))
    ours = B.accumulate_quotients(domain, cols, rc, batches).values.to_numpy()
    out = stwo.SecureColumnByCoords.uninitialized(1 << log_size)
    dev = R.copy_device_pointer_vec_from_host_to_device(_ptrs([c.values for c in cols]), ncols)
    pts = (C.c_uint32 * (8 * len(batches)))(*[v for b in batches for v in list(b.point[0]) + list(b.point[1])])
    idx = (C.c_uint32 * (ncols * len(batches)))(*[i for b in batches for i, _ in b.columns_and_values])
    vals = (reflib.QM31 * (ncols * len(batches)))(*[reflib.QM31(*v) for b in batches for _, v in b.columns_and_values])
    sizes = (C.c_uint32 * len(batches))(*([ncols] * len(batches)))
    R.accumulate_quotients(domain.half_coset.initial_index, domain.half_coset.step_size, 1 << log_size, dev, ncols,
                           reflib.QM31(*rc), pts, idx, ncols * len(batches), vals, sizes, len(batches),
                           *[c.device_ptr for c in out.columns], ncols * len(batches) * 3)
    R.cuda_free_memory(dev)
    for x, y in zip(ours, out.to_numpy()):
        assert (x == y).all()


def test_wide_fib_composition_matches_reference(stwo, R):
    L = stwo._lib
    r = rng(7)
    ext, ncols = 1 << 16, 24
    trace = [stwo.BaseFieldVec.from_numpy(m31(r, ext)) for _ in range(ncols)]
    powers = np.array([random_qm31(r) for _ in range(ncols - 2)], np.uint32)
    pdev = stwo.SecureFieldVec.from_numpy(powers)
    di = stwo.BaseFieldVec.from_numpy(m31(r, ext))
    ours = stwo.SecureColumnByCoords.uninitialized(ext)
    L.lib().evaluate_wide_fibonacci_constraint_quotients_on_domain(
        *[c.device_ptr for c in ours.columns], L.ptr_array([t.device_ptr for t in trace]), pdev.device_ptr,
        di.device_ptr, ext, ncols)
    L.check_last()
    ref = stwo.SecureColumnByCoords.uninitialized(ext)
    # the reference copies `extended_domain_size` pointers from this host array
    host_ptrs = (C.c_void_p * ext)(*([t.device_ptr for t in trace] + [None] * (ext - ncols)))
    R.evaluate_wide_fibonacci_constraint_quotients_on_domain(*[c.device_ptr for c in ref.columns], host_ptrs,
                                                             pdev.device_ptr, di.device_ptr, ext, ncols)
    for x, y in zip(ours.to_numpy(), ref.to_numpy()):
        assert (x == y).all()
