"""ColumnOps::bit_reverse_column and FieldOps::batch_inverse on the GPU vs the oracle."""
import numpy as np
import pytest

from helpers import P, m31, m31_nonzero, rng

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_size", [0, 1, 2, 5, 9, 10, 11, 16, 21])
def test_bit_reverse_base_field(stwo, oracle, log_size):
    """column.rs:157 (2^10 in the reference)."""
    v = m31(rng(log_size), 1 << log_size)
    col = stwo.BaseFieldVec.from_numpy(v)
    stwo.CudaBackend.bit_reverse_column(col)
    assert (col.to_numpy() == oracle.bit_reverse(v)).all()


@pytest.mark.parametrize("log_size", [0, 3, 10, 14, 16, 19])
def test_bit_reverse_secure_field(stwo, oracle, log_size):
    """column.rs:170 (2^16 QM31 in the reference)."""
    v = m31(rng(50 + log_size), 4 << log_size).reshape(-1, 4)
    col = stwo.SecureFieldVec.from_numpy(v)
    stwo.CudaBackend.bit_reverse_column(col)
    assert (col.to_numpy() == oracle.bit_reverse(v)).all()


def test_bit_reverse_is_an_involution_full_size(stwo):
    v = np.arange(1 << 26, dtype=np.uint32)
    col = stwo.BaseFieldVec.from_numpy(v)
    stwo.CudaBackend.bit_reverse_column(col)
    got = col.to_numpy()
    idx = rng(1).integers(0, 1 << 26, 4096)
    rev = np.array([int(format(int(i), "026b")[::-1], 2) for i in idx])
    assert (got[idx] == rev).all()
    stwo.CudaBackend.bit_reverse_column(col)
    assert (col.to_numpy() == v).all()


@pytest.mark.parametrize("n", [1, 7, 512, 2048, 2049, 100_000, 1 << 20])
def test_batch_inverse_base_field(stwo, oracle, n):
    """field.rs:42 (2^25 values 1..n in the reference; random nonzero here)."""
    v = m31_nonzero(rng(n), n)
    src = stwo.BaseFieldVec.from_numpy(v)
    dst = stwo.BaseFieldVec.new_uninitialized(n)
    stwo.CudaBackend.batch_inverse(src, dst)
    assert (dst.to_numpy() == oracle.batch_inverse_m31(v)).all()


@pytest.mark.parametrize("n", [1, 5, 1024, 3000, 8191, 8192, 8193, 1 << 18])
def test_batch_inverse_secure_field(stwo, oracle, n):
    """field.rs:59 (QM31 values from 1..4n in the reference)."""
    v = m31(rng(9 + n), 4 * n).reshape(n, 4)
    v[:, 0] |= 1  # nonzero
    src = stwo.SecureFieldVec.from_numpy(v)
    dst = stwo.SecureFieldVec.new_uninitialized(n)
    stwo.CudaBackend.batch_inverse(src, dst)
    assert (dst.to_numpy() == oracle.batch_inverse_qm31(v)).all()


@pytest.mark.parametrize("n", [7, 4096 + 33, 1 << 17])
def test_batch_inverse_in_place(stwo, oracle, n):
    """src == dst: each element is read before its inverse is written over it."""
    L = stwo._lib
    v = m31_nonzero(rng(700 + n), n)
    b = stwo.BaseFieldVec.from_numpy(v)
    L.check(L.lib().stwo_batch_inverse_m31(b.device_ptr, b.device_ptr, n, None))
    L.check(L.lib().stwo_stream_synchronize(None))
    assert (b.to_numpy() == oracle.batch_inverse_m31(v)).all()
    q = m31(rng(800 + n), 4 * n).reshape(n, 4)
    q[:, 0] |= 1
    qb = stwo.SecureFieldVec.from_numpy(q)
    L.check(L.lib().stwo_batch_inverse_qm31(qb.device_ptr, qb.device_ptr, n, None))
    L.check(L.lib().stwo_stream_synchronize(None))
    assert (qb.to_numpy() == oracle.batch_inverse_qm31(q)).all()


def test_batch_inverse_reference_pattern_full_size(stwo):
    """The reference's own pattern (values 1..2^25) checked by v * inv(v) == 1."""
    n = 1 << 25
    v = np.arange(1, n + 1, dtype=np.uint32)
    src = stwo.BaseFieldVec.from_numpy(v)
    dst = stwo.BaseFieldVec.new_uninitialized(n)
    stwo.CudaBackend.batch_inverse(src, dst)
    inv = dst.to_numpy().astype(np.uint64)
    assert ((v.astype(np.uint64) * inv) % P == 1).all()
