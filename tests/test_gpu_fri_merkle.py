"""FriOps, MerkleOps and AccumulationOps on the GPU vs the oracle."""
import json
import os

import numpy as np
import pytest

from helpers import m31, random_qm31, rng

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_literals.json")))


def _oc(o, c):
    return o.coset(c.initial_index, c.step_size, c.log_size)


@pytest.mark.parametrize("log_size", [1, 2, 3, 10, 13, 20])
def test_fold_line(stwo, oracle, log_size):
    """fri.rs:100 (2^20 random values, alpha (1,3,5,7))."""
    B = stwo.CudaBackend
    r = rng(400 + log_size)
    cols = [m31(r, 1 << log_size) for _ in range(4)]
    alpha = (1, 3, 5, 7) if log_size == 20 else random_qm31(r)
    domain = stwo.LineDomain(stwo.CanonicCoset(log_size + 1).half_coset())
    tree = B.precompute_twiddles(domain.coset)
    out = B.fold_line(stwo.LineEvaluation(domain, stwo.SecureColumnByCoords.from_numpy(cols)), alpha, tree)
    expect = oracle.fold_line(cols, _oc(oracle, domain.coset), alpha)
    for g, e in zip(out.values.to_numpy(), expect):
        assert (g == e).all()


def test_fold_line_more_than_once(stwo, oracle):
    """fri.rs:195: three successive folds at 2^13."""
    B = stwo.CudaBackend
    r = rng(13)
    cols = [m31(r, 1 << 13) for _ in range(4)]
    alpha = (1, 3, 5, 7)
    domain = stwo.LineDomain(stwo.CanonicCoset(14).half_coset())
    tree = B.precompute_twiddles(domain.coset)
    ev = stwo.LineEvaluation(domain, stwo.SecureColumnByCoords.from_numpy(cols))
    dom = _oc(oracle, domain.coset)
    for _ in range(3):
        ev = B.fold_line(ev, alpha, tree)
        cols = oracle.fold_line(cols, dom, alpha)
        dom = oracle.coset_double(dom)
    for g, e in zip(ev.values.to_numpy(), cols):
        assert (g == e).all()


@pytest.mark.parametrize("log_size", [1, 2, 3, 13, 21])
def test_fold_circle_into_line(stwo, oracle, log_size):
    """fri.rs:260 (2^13, values 4i..4i+3, alpha (1,3,5,7)) plus random sizes."""
    B = stwo.CudaBackend
    n = 1 << log_size
    if log_size == 13:
        i = np.arange(n, dtype=np.uint32)
        src = [4 * i, 4 * i + 1, 4 * i + 2, 4 * i + 3]
        alpha = (1, 3, 5, 7)
        dst0 = [np.zeros(n // 2, np.uint32) for _ in range(4)]
    else:
        r = rng(500 + log_size)
        src = [m31(r, n) for _ in range(4)]
        alpha = random_qm31(r)
        dst0 = [m31(r, n // 2) for _ in range(4)]
    circle = stwo.CanonicCoset(log_size).circle_domain()
    line = stwo.LineDomain(circle.half_coset)
    # For 2- and 4-point circle domains the tree must also cover the 8-point domain
    # (the circle twiddle 1/y is derived from it); larger folds use the reference's tree.
    tree = B.precompute_twiddles(line.coset if log_size > 2 else stwo.CanonicCoset(4).half_coset())
    dst = stwo.LineEvaluation(line, stwo.SecureColumnByCoords.from_numpy(dst0))
    B.fold_circle_into_line(dst, stwo.SecureEvaluation(circle, stwo.SecureColumnByCoords.from_numpy(src)), alpha, tree)
    expect = oracle.fold_circle_into_line(dst0, src, _oc(oracle, circle.half_coset), alpha)
    for g, e in zip(dst.values.to_numpy(), expect):
        assert (g == e).all()


def test_fold_circle_into_line_tiny_domain_needs_larger_tree(stwo):
    circle = stwo.CanonicCoset(2).circle_domain()
    line = stwo.LineDomain(circle.half_coset)
    tree = stwo.CudaBackend.precompute_twiddles(line.coset)
    dst = stwo.LineEvaluation(line, stwo.SecureColumnByCoords.zeros(2))
    src = stwo.SecureEvaluation(circle, stwo.SecureColumnByCoords.zeros(4))
    with pytest.raises(stwo._lib.StwoError, match="8-point"):
        stwo.CudaBackend.fold_circle_into_line(dst, src, (1, 2, 3, 4), tree)


def test_fold_circle_into_line_fibonacci_literals(stwo, oracle):
    """fri.rs:313-940: literal dst/src/alpha/domains with the literal twiddle tree
    (root coset larger than the folded domain: twiddle offset 32)."""
    f = GOLDEN["fold_circle_into_line_fib"]
    rc, sd, dd = f["root_coset"], f["src_circle_half_coset"], f["dst_line_domain"]
    tree = stwo.TwiddleTree(stwo.Coset(rc["initial_index"], rc["step_size"], rc["log_size"]),
                            stwo.BaseFieldVec.from_numpy(np.array(f["twiddles"], np.uint32)),
                            stwo.BaseFieldVec.from_numpy(np.array(f["itwiddles"], np.uint32)))
    src_dom = stwo.CircleDomain(stwo.Coset(sd["initial_index"], sd["step_size"], sd["log_size"]))
    dst_dom = stwo.LineDomain(stwo.Coset(dd["initial_index"], dd["step_size"], dd["log_size"]))
    src = [np.array(c, np.uint32) for c in f["src"]]
    dst0 = [np.array(c, np.uint32) for c in f["dst"]]
    dst = stwo.LineEvaluation(dst_dom, stwo.SecureColumnByCoords.from_numpy(dst0))
    stwo.CudaBackend.fold_circle_into_line(dst, stwo.SecureEvaluation(src_dom, stwo.SecureColumnByCoords.from_numpy(src)),
                                           tuple(f["alpha"]), tree)
    expect = oracle.fold_circle_into_line(dst0, src, oracle.coset(sd["initial_index"], sd["step_size"], sd["log_size"]),
                                          tuple(f["alpha"]))
    for g, e in zip(dst.values.to_numpy(), expect):
        assert (g == e).all()


def _cols_test_vector(ncols, size):
    """blake2s.rs:181-192: column j holds M31(i * j)."""
    i = np.arange(size, dtype=np.uint64)
    return [((i * j) % ((1 << 31) - 1)).astype(np.uint32) for j in range(ncols)]


@pytest.mark.parametrize("ncols", [0, 1, 15, 16, 17, 35, 64])
def test_merkle_first_layer(stwo, oracle, ncols):
    """blake2s.rs:110 (35 columns x 2^11)."""
    cols = _cols_test_vector(ncols, 1 << 11)
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cols]
    got = stwo.CudaBackend.commit_on_layer(11, None, bufs).to_numpy()
    assert (got == oracle.merkle_commit_on_layer(11, None, cols)).all()
    got_ref = stwo.CudaBackend.commit_on_layer_reference_abi(11, None, bufs).to_numpy()
    assert (got_ref == got).all()


def test_merkle_layer_with_previous(stwo, oracle):
    """blake2s.rs:132: 16 columns of 2^11 over a 35-column 2^12 layer."""
    prev_cols = _cols_test_vector(35, 1 << 12)
    prev_bufs = [stwo.BaseFieldVec.from_numpy(c) for c in prev_cols]
    prev = stwo.CudaBackend.commit_on_layer(12, None, prev_bufs)
    cols = _cols_test_vector(16, 1 << 11)
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cols]
    got = stwo.CudaBackend.commit_on_layer(11, prev, bufs).to_numpy()
    prev_o = oracle.merkle_commit_on_layer(12, None, prev_cols)
    assert (got == oracle.merkle_commit_on_layer(11, prev_o, cols)).all()
    got_ref = stwo.CudaBackend.commit_on_layer_reference_abi(11, prev, bufs).to_numpy()
    assert (got_ref == got).all()


def test_merkle_tree_mixed_sizes(stwo, oracle):
    """A whole tree over columns of log sizes 4..12 (MerkleProver::commit order:
    largest first, each layer hashes children then that size's columns)."""
    r = rng(21)
    logs = [12, 12, 11, 9, 9, 9, 6, 4]
    cols = [m31(r, 1 << lg) for lg in logs]
    bufs = {i: stwo.BaseFieldVec.from_numpy(c) for i, c in enumerate(cols)}
    layers_o = oracle.merkle_commit(cols)
    prev = None
    got_layers = []
    for lg in range(12, -1, -1):
        layer_cols = [bufs[i] for i, l in enumerate(logs) if l == lg]
        prev = stwo.CudaBackend.commit_on_layer(lg, prev, layer_cols)
        got_layers.append(prev.to_numpy())
    got_layers.reverse()
    for g, e in zip(got_layers, layers_o):
        assert (g == e).all()


@pytest.mark.parametrize("logs", [[12, 12, 11, 9, 9, 9, 6, 4], [20] * 3 + [18] * 20 + [15] * 33 + [3, 0],
                                  [14, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1]])
def test_merkle_commit_tree_matches_layer_by_layer_oracle(stwo, oracle, logs):
    """stwo_merkle_commit_tree hashes a whole mixed-size tree in one launch: every
    layer equals the oracle's MerkleProver::commit layer (columns of one size hashed in
    their order; sizes with no columns, more than 16 columns a layer, a 1-element
    column)."""
    L = stwo._lib
    r = rng(sum(logs))
    cols = [m31(r, 1 << lg) for lg in logs]
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cols]
    top = max(logs)
    layers = [stwo.BaseFieldVec.new_uninitialized(8 << l) for l in range(top + 1)]
    L.check(L.lib().stwo_merkle_commit_tree(L.ptr_array([b.device_ptr for b in bufs]), L.u32_array(logs), len(logs),
                                            top, L.ptr_array([x.device_ptr for x in layers]), None))
    L.check(L.lib().stwo_stream_synchronize(None))
    want = oracle.merkle_commit(cols)
    for l in range(top + 1):
        assert (layers[l].to_numpy().reshape(-1, 8) == want[l]).all(), l


@pytest.mark.parametrize("threads,spread", [(256, 3), (128, 0), (128, 5), (256, 0), (512, 1), (512, 5)])
def test_merkle_tree_one_launch_every_band_split(stwo, threads, spread):
    """The whole-tree kernel hashes every layer in one launch: the CTA that finishes the
    last unit under a node of the next band goes on to hash that band's unit. Each
    CTA size and spread cuts the layers into different bands (one to four); every
    layer must equal the layer-by-layer kernel's (pinned to the oracle above), the call
    must be a single launch, and a second call into zeroed buffers must give the same
    layers (the order in which CTAs finish does not change the tree)."""
    L = stwo._lib
    lib = L.lib()
    L.check(lib.stwo_set_tunable(b"merkle_sub_threads", threads))
    L.check(lib.stwo_set_tunable(b"merkle_sub_spread", spread))
    try:
        for nc, lg in [(4, 0), (1, 1), (4, 8), (8, 9), (4, 13), (20, 16), (4, 21), (64, 19)]:
            r = rng(lg * 1000 + nc + threads + spread)
            bufs = [stwo.BaseFieldVec.from_numpy(m31(r, 1 << lg)) for _ in range(nc)]
            want = [stwo.BaseFieldVec.new_uninitialized(8 << l) for l in range(lg + 1)]
            L.check(lib.stwo_merkle_commit_layer(lg, None, L.ptr_array([b.device_ptr for b in bufs]), nc,
                                                 want[lg].device_ptr, None))
            for l in range(lg - 1, -1, -1):
                L.check(lib.stwo_merkle_commit_layer(l, want[l + 1].device_ptr, None, 0, want[l].device_ptr, None))
            layers = [stwo.BaseFieldVec.new_uninitialized(8 << l) for l in range(lg + 1)]
            args = (L.ptr_array([b.device_ptr for b in bufs]), L.u32_array([lg] * nc), nc, lg,
                    L.ptr_array([x.device_ptr for x in layers]), None)
            n0 = lib.stwo_kernel_launches()
            L.check(lib.stwo_merkle_commit_tree(*args))
            assert lib.stwo_kernel_launches() - n0 == 1, (nc, lg)
            L.check(lib.stwo_stream_synchronize(None))
            first = [x.to_numpy() for x in layers]
            for l in range(lg + 1):
                assert (first[l] == want[l].to_numpy()).all(), (nc, lg, l)
            again = [stwo.BaseFieldVec.new_zeroes(8 << l) for l in range(lg + 1)]
            L.check(lib.stwo_merkle_commit_tree(*args[:4], L.ptr_array([x.device_ptr for x in again]), None))
            L.check(lib.stwo_stream_synchronize(None))
            assert all((x.to_numpy() == f).all() for x, f in zip(again, first)), (nc, lg)
    finally:
        lib.stwo_set_tunable(b"merkle_sub_threads", 256)
        lib.stwo_set_tunable(b"merkle_sub_spread", 3)


def test_merkle_64_columns_log22_root_property(stwo, oracle):
    """Config shape (64 columns at log 22): spot-check leaves against the oracle."""
    r = rng(22)
    n = 1 << 22
    cols = [m31(r, n) for _ in range(64)]
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in cols]
    got = stwo.CudaBackend.commit_on_layer(22, None, bufs).to_numpy()
    idx = r.integers(0, n, 64)
    sub = [c[idx] for c in cols]
    # the oracle hashes a 64-leaf layer built from the sampled rows
    expect = oracle.merkle_commit_on_layer(6, None, sub)
    assert (got[idx] == expect).all()


def test_accumulate(stwo, oracle):
    """accumulation.rs:32,68 literal cases at 2^21 plus random data."""
    for case in GOLDEN["accumulation"]:
        n = 2 << 20
        left = stwo.SecureColumnByCoords.from_numpy([np.full(n, v, np.uint32) for v in case["left"]])
        right = stwo.SecureColumnByCoords.from_numpy([np.full(n, v, np.uint32) for v in case["right"]])
        stwo.CudaBackend.accumulate(left, right)
        got = left.to_numpy()
        for g, e in zip(got, case["expected"]):
            assert (g == e).all()
    r = rng(3)
    for n in [1, 3, 5, 1000, 1 << 16]:
        l0 = [m31(r, n) for _ in range(4)]
        r0 = [m31(r, n) for _ in range(4)]
        left = stwo.SecureColumnByCoords.from_numpy(l0)
        stwo.CudaBackend.accumulate(left, stwo.SecureColumnByCoords.from_numpy(r0))
        for g, e in zip(left.to_numpy(), oracle.accumulate(l0, r0)):
            assert (g == e).all()
