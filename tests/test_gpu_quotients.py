"""QuotientOps::accumulate_quotients and the wide-Fibonacci composition on the GPU vs the oracle."""
import numpy as np
import pytest

from helpers import m31, random_circle_point, random_qm31, rng

pytestmark = pytest.mark.gpu


def _oc(o, c):
    return o.coset(c.initial_index, c.step_size, c.log_size)


def _run_quotients(stwo, oracle, log_size, ncols, batch_sizes, seed, reference_abi=False):
    B = stwo.CudaBackend
    r = rng(seed)
    domain = stwo.CanonicCoset(log_size).circle_domain()
    cols_np = [m31(r, 1 << log_size) for _ in range(ncols)]
    cols = [stwo.CircleEvaluation(domain, stwo.BaseFieldVec.from_numpy(c)) for c in cols_np]
    rc = random_qm31(r)
    batches, obatches = [], []
    for bs in batch_sizes:
        px, py = random_circle_point(r)
        cv = [(int(ci), random_qm31(r)) for ci in r.choice(ncols, size=bs, replace=bs > ncols)]
        batches.append(stwo.ColumnSampleBatch((px, py), cv))
        obatches.append((px, py, cv))
    expect = oracle.accumulate_quotients(_oc(oracle, domain.half_coset), cols_np, rc, obatches)
    if not reference_abi:
        got = B.accumulate_quotients(domain, cols, rc, batches).values.to_numpy()
    else:
        L = stwo._lib
        out = stwo.SecureColumnByCoords.uninitialized(1 << log_size)
        dev = L.lib().copy_device_pointer_vec_from_host_to_device(L.ptr_array([c.values.device_ptr for c in cols]),
                                                                  ncols)
        pts = []
        for b in batches:
            pts += list(b.point[0]) + list(b.point[1])
        idx = [ci for b in batches for ci, _ in b.columns_and_values]
        vals = (L.QM31 * len(idx))(*[L.QM31(*v) for b in batches for _, v in b.columns_and_values])
        L.clear_error()
        L.lib().accumulate_quotients(domain.half_coset.initial_index, domain.half_coset.step_size, 1 << log_size,
                                     dev, ncols, L.QM31(*rc), L.u32_array(pts), L.u32_array(idx), len(idx), vals,
                                     L.u32_array(batch_sizes), len(batches), *[c.device_ptr for c in out.columns],
                                     ncols * len(batches) * 3)
        L.check_last()
        L.lib().cuda_free_memory(dev)
        got = out.to_numpy()
    for g, e in zip(got, expect):
        assert (g == e).all()


def test_quotients_reference_shape(stwo, oracle):
    """quotient.rs:133: 2 columns over a 2^16 domain, 3 batches of 2 samples."""
    _run_quotients(stwo, oracle, 16, 2, [2, 2, 2], 1)


@pytest.mark.parametrize("log_size", [1, 2, 5, 12])
def test_quotients_small(stwo, oracle, log_size):
    _run_quotients(stwo, oracle, log_size, 5, [3, 1, 5], 10 + log_size)


def test_quotients_mixed_batch_sizes(stwo, oracle):
    # batches of different sizes (the case the reference kernel mis-indexes)
    _run_quotients(stwo, oracle, 13, 32, [32, 7, 1, 19], 3)


def test_quotients_reference_abi(stwo, oracle):
    _run_quotients(stwo, oracle, 12, 8, [8, 3, 8], 4, reference_abi=True)


def test_quotients_config_shape(stwo, oracle):
    """32 columns at log 22 with 4 sample points (each sampling all 32 columns):
    spot-checked against the oracle on a 2^14 subdomain of the same structure
    (the per-row formula is size-independent), full size checked for determinism."""
    _run_quotients(stwo, oracle, 14, 32, [32, 32, 32, 32], 5)


@pytest.fixture
def tensor_cores(stwo):
    """Sets the quotients_tensor_cores tunable for one test and restores the default."""
    L = stwo._lib

    def set_(v):
        L.check(L.lib().stwo_set_tunable(b"quotients_tensor_cores", v))
    yield set_
    set_(1)


def _faults(stwo):
    import ctypes as C
    n = C.c_uint32()
    stwo._lib.check(stwo._lib.lib().stwo_quotients_tc_faults(C.byref(n), 1))
    return n.value


# (log_size, columns, batch sizes): below one tile (2^7 rows: the CUDA cores), one tile
# (2^8 rows) up to many tiles per CTA, 1-4
# batches, partial column chunks (1, 5, 33, 100 columns), repeated columns within a batch
# (more samples than columns), the largest byte matrix the tensor form takes (250
# columns, rounded up to 256, x 4 batches), and 260 x 4, past it (the CUDA cores).
TC_SHAPES = [(7, 1, [1]), (8, 5, [3, 1, 5]), (8, 33, [33, 33]), (11, 100, [100]), (12, 8, [20, 3, 9, 8]),
             (13, 32, [32, 7, 1, 19]), (15, 250, [128, 128, 128, 128]), (9, 260, [130, 130, 130, 120]),
             (18, 64, [64])]


@pytest.mark.parametrize("log_size,ncols,batch_sizes", TC_SHAPES)
@pytest.mark.parametrize("tc", [2, 1, 0])
def test_quotients_tensor_and_cuda_cores(stwo, oracle, tensor_cores, log_size, ncols, batch_sizes, tc):
    """Both forms of the quotient kernel equal the oracle, through the native and the
    reference-compatible entry points (tc: the quotients_tensor_cores tunable; 2 takes
    the tensor cores wherever the form applies)."""
    tensor_cores(tc)
    _faults(stwo)
    seed = 100 * log_size + ncols
    _run_quotients(stwo, oracle, log_size, ncols, batch_sizes, seed)
    if ncols <= 100:
        _run_quotients(stwo, oracle, log_size, ncols, batch_sizes, seed + 1, reference_abi=True)
    assert _faults(stwo) == 0


def test_quotients_tensor_cores_full_size(stwo, tensor_cores):
    """32 columns x 2^22 with 4 points (the kernel sweep's shape): the tensor-core and
    CUDA-core forms give identical columns (each form is checked against the oracle
    above on the same per-row formula)."""
    B = stwo.CudaBackend
    r = rng(7)
    lg, nc = 22, 32
    domain = stwo.CanonicCoset(lg).circle_domain()
    cols = [stwo.CircleEvaluation(domain, stwo.BaseFieldVec.from_numpy(m31(r, 1 << lg))) for _ in range(nc)]
    rc = random_qm31(r)
    batches = [stwo.ColumnSampleBatch(random_circle_point(r), [(c, random_qm31(r)) for c in range(nc)])
               for _ in range(4)]
    got = {}
    for tc in (2, 0):
        tensor_cores(tc)
        got[tc] = B.accumulate_quotients(domain, cols, rc, batches).values.to_numpy()
    for a, b in zip(got[2], got[0]):
        assert (a == b).all()
    assert _faults(stwo) == 0


@pytest.fixture
def comp_tensor_cores(stwo):
    """Sets the composition_tensor_cores tunable for one test and restores the default (0)."""
    L = stwo._lib

    def set_(v):
        L.check(L.lib().stwo_set_tunable(b"composition_tensor_cores", v))
    yield set_
    set_(0)


def _comp_faults(stwo):
    import ctypes as C
    n = C.c_uint32()
    stwo._lib.check(stwo._lib.lib().stwo_composition_tc_faults(C.byref(n), 1))
    return n.value


# below one tile (2^6 rows: the CUDA cores), the fewest columns (3), constraint counts
# that are not a multiple of 32 (a stage), the most the tensor form takes (1024) and
# one past it (1025).
@pytest.mark.parametrize("n_cols,log_size", [(3, 1), (8, 5), (64, 13), (256, 8), (3, 7), (5, 9), (34, 8),
                                             (35, 8), (130, 10), (512, 8), (1024, 7), (1025, 7), (256, 12)])
@pytest.mark.parametrize("tc", [1, 0])
def test_wide_fib_composition(stwo, oracle, comp_tensor_cores, n_cols, log_size, tc):
    comp_tensor_cores(tc)
    _comp_faults(stwo)
    _wide_fib_composition(stwo, oracle, n_cols, log_size)
    assert _comp_faults(stwo) == 0


def _wide_fib_composition(stwo, oracle, n_cols, log_size):
    L = stwo._lib
    r = rng(n_cols + log_size)
    trace = [m31(r, 1 << log_size) for _ in range(n_cols)]
    powers = np.array([random_qm31(r) for _ in range(n_cols - 2)], np.uint32)
    den_inv = m31(r, 1 << log_size)
    expect = oracle.wide_fib_composition(trace, powers, den_inv)
    bufs = [stwo.BaseFieldVec.from_numpy(c) for c in trace]
    di = stwo.BaseFieldVec.from_numpy(den_inv)
    # native entry point (host powers)
    out = stwo.SecureColumnByCoords.uninitialized(1 << log_size)
    pw = (L.QM31 * len(powers))(*[L.QM31(*[int(x) for x in p]) for p in powers])
    L.check(L.lib().stwo_wide_fib_composition(L.ptr_array([b.device_ptr for b in bufs]), n_cols, log_size, pw,
                                              di.device_ptr, out.ptrs(), None))
    L.check(L.lib().stwo_stream_synchronize(None))
    for g, e in zip(out.to_numpy(), expect):
        assert (g == e).all()
    # reference-compatible entry point (device powers)
    out2 = stwo.SecureColumnByCoords.uninitialized(1 << log_size)
    pdev = stwo.SecureFieldVec.from_numpy(powers)
    L.clear_error()
    L.lib().evaluate_wide_fibonacci_constraint_quotients_on_domain(
        *[c.device_ptr for c in out2.columns], L.ptr_array([b.device_ptr for b in bufs]), pdev.device_ptr,
        di.device_ptr, 1 << log_size, n_cols)
    L.check_last()
    for g, e in zip(out2.to_numpy(), expect):
        assert (g == e).all()
