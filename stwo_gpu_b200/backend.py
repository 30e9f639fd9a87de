"""Host-side mirror of the reference's CudaBackend (stwo_gpu_backend/src/*.rs).

The reference implements stwo's backend traits in Rust over its C ABI
(backend.rs:9-20, column.rs:10-142, field.rs:8-30, poly.rs:20-193, fri.rs:15-75,
blake2s.rs:11-97, quotient.rs:17-115, accumulation.rs:9-19). No Rust toolchain is
available here, so this module restates those trait methods in Python over the
same C ABI (libstwo_b200.so): same method names, same argument meaning, same
device-resident column types. Every call runs on the GPU; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import _lib as L

P = (1 << 31) - 1
M31_CIRCLE_LOG_ORDER = 31


# ----------------------------------------------------------------------------- domains
def _index_mask(i):
    return i & ((1 << M31_CIRCLE_LOG_ORDER) - 1)


def _pt_mul(p, q):
    return ((p[0] * q[0] - p[1] * q[1]) % P, (p[0] * q[1] + p[1] * q[0]) % P)


M31_CIRCLE_GEN = (2, 1268011823)


def index_to_point(index):
    """CirclePointIndex -> CirclePoint<M31> (M31_CIRCLE_GEN^index)."""
    index = _index_mask(index)
    r, b = (1, 0), M31_CIRCLE_GEN
    while index:
        if index & 1:
            r = _pt_mul(r, b)
        b = _pt_mul(b, b)
        index >>= 1
    return r


def subgroup_gen(log_size):
    return 1 << (M31_CIRCLE_LOG_ORDER - log_size)


class Coset:
    """stwo core::circle::Coset (indices mod 2^31)."""

    def __init__(self, initial_index, step_size, log_size):
        self.initial_index = _index_mask(initial_index)
        self.step_size = _index_mask(step_size)
        self.log_size = log_size

    @classmethod
    def new(cls, initial_index, log_size):
        return cls(initial_index, subgroup_gen(log_size), log_size)

    @classmethod
    def odds(cls, log_size):
        return cls.new(subgroup_gen(log_size + 1), log_size)

    @classmethod
    def half_odds(cls, log_size):
        return cls.new(subgroup_gen(log_size + 2), log_size)

    def size(self):
        return 1 << self.log_size

    def index_at(self, i):
        return _index_mask(self.initial_index + self.step_size * i)

    def at(self, i):
        return index_to_point(self.index_at(i))

    @property
    def initial(self):
        return index_to_point(self.initial_index)

    @property
    def step(self):
        return index_to_point(self.step_size)

    def double(self):
        return Coset(self.initial_index * 2, self.step_size * 2, self.log_size - 1)

    def repeated_double(self, n):
        c = self
        for _ in range(n):
            c = c.double()
        return c

    def is_doubling_of(self, other):
        return self.log_size <= other.log_size and other.repeated_double(other.log_size - self.log_size) == self

    def __eq__(self, o):
        return (self.initial_index, self.step_size, self.log_size) == (o.initial_index, o.step_size, o.log_size)

    def __repr__(self):
        return f"Coset({self.initial_index}, {self.step_size}, log {self.log_size})"


class CircleDomain:
    def __init__(self, half_coset):
        self.half_coset = half_coset

    def log_size(self):
        return self.half_coset.log_size + 1

    def size(self):
        return 1 << self.log_size()

    def index_at(self, i):
        h = self.half_coset.size()
        return self.half_coset.index_at(i) if i < h else _index_mask(-self.half_coset.index_at(i - h))

    def at(self, i):
        return index_to_point(self.index_at(i))


class CanonicCoset:
    def __init__(self, log_size):
        self.log_size = log_size
        self.coset = Coset.odds(log_size)

    def half_coset(self):
        return Coset.half_odds(self.log_size - 1)

    def circle_domain(self):
        return CircleDomain(self.half_coset())

    def size(self):
        return 1 << self.log_size


class LineDomain:
    def __init__(self, coset):
        self.coset = coset

    def size(self):
        return self.coset.size()

    def log_size(self):
        return self.coset.log_size

    def double(self):
        return LineDomain(self.coset.double())


# ----------------------------------------------------------------------------- columns
class DeviceVec:
    """Owning device buffer of 32-bit words (BaseFieldVec / SecureFieldVec storage)."""

    words_per_elem = 1

    def __init__(self, device_ptr, size):
        self.device_ptr = device_ptr
        self.size = size

    @classmethod
    def new_uninitialized(cls, size):
        p = L.lib().cuda_malloc_uint32_t(max(1, size * cls.words_per_elem))
        if not p:
            L.check_last()
        return cls(p, size)

    @classmethod
    def new_zeroes(cls, size):
        p = L.lib().cuda_alloc_zeroes_uint32_t(max(1, size * cls.words_per_elem))
        if not p:
            L.check_last()
        return cls(p, size)

    @classmethod
    def from_numpy(cls, arr):
        a = np.ascontiguousarray(arr, dtype=np.uint32).reshape(-1)
        assert a.size % cls.words_per_elem == 0
        p = L.lib().copy_uint32_t_vec_from_host_to_device(a.ctypes.data, max(1, a.size))
        if not p:
            L.check_last()
        return cls(p, a.size // cls.words_per_elem)

    from_vec = from_numpy

    def to_numpy(self):
        out = np.empty(self.size * self.words_per_elem, np.uint32)
        if out.size:
            L.lib().copy_uint32_t_vec_from_device_to_host(self.device_ptr, out.ctypes.data, out.size)
            L.check_last()
        return out if self.words_per_elem == 1 else out.reshape(-1, self.words_per_elem)

    to_cpu = to_numpy

    def __len__(self):
        return self.size

    def clone(self):
        n = self.new_uninitialized(self.size)
        if self.size:
            L.lib().copy_uint32_t_vec_from_device_to_device(self.device_ptr, n.device_ptr,
                                                            self.size * self.words_per_elem)
            L.check_last()
        return n

    def copy_from(self, other):
        L.lib().copy_uint32_t_vec_from_device_to_device(other.device_ptr, self.device_ptr,
                                                        other.size * other.words_per_elem)
        L.check_last()

    def free(self):
        if self.device_ptr:
            L.lib().cuda_free_memory(self.device_ptr)
            self.device_ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class BaseFieldVec(DeviceVec):
    words_per_elem = 1


class SecureFieldVec(DeviceVec):
    words_per_elem = 4


class Blake2sHashVec(DeviceVec):
    words_per_elem = 8


class SecureColumnByCoords:
    """Four M31 coordinate columns (stwo SecureColumnByCoords<CudaBackend>)."""

    def __init__(self, columns):
        assert len(columns) == 4
        self.columns = columns

    @classmethod
    def zeros(cls, size):
        return cls([BaseFieldVec.new_zeroes(size) for _ in range(4)])

    @classmethod
    def uninitialized(cls, size):
        return cls([BaseFieldVec.new_uninitialized(size) for _ in range(4)])

    @classmethod
    def from_numpy(cls, cols4):
        return cls([BaseFieldVec.from_numpy(c) for c in cols4])

    def to_numpy(self):
        return [c.to_numpy() for c in self.columns]

    def __len__(self):
        return len(self.columns[0])

    def ptrs(self):
        return L.ptr_array([c.device_ptr for c in self.columns])


class TwiddleTree:
    def __init__(self, root_coset, twiddles, itwiddles):
        self.root_coset = root_coset
        self.twiddles = twiddles
        self.itwiddles = itwiddles


class CircleEvaluation:
    def __init__(self, domain, values):
        self.domain = domain
        self.values = values


class CirclePoly:
    def __init__(self, coeffs):
        self.coeffs = coeffs

    def log_size(self):
        return len(self.coeffs).bit_length() - 1


class LineEvaluation:
    def __init__(self, domain, values):
        self.domain = domain
        self.values = values


class SecureEvaluation:
    def __init__(self, domain, values):
        self.domain = domain
        self.values = values


class ColumnSampleBatch:
    def __init__(self, point, columns_and_values):
        self.point = point              # ((4 ints), (4 ints)) QM31 x, y
        self.columns_and_values = columns_and_values  # [(col index, (4 ints))]


def qm31(v):
    v = [int(x) for x in v]
    return L.QM31(v[0], v[1], v[2], v[3])


# ----------------------------------------------------------------------------- backend
class CudaBackend:
    """stwo backend traits over libstwo_b200.so (reference: stwo_gpu_backend/src/backend.rs:9-20)."""

    # ColumnOps (column.rs:10-34)
    @staticmethod
    def bit_reverse_column(column):
        n = len(column)
        assert n & (n - 1) == 0 and n < (1 << 32)
        L.clear_error()
        if isinstance(column, SecureFieldVec):
            L.lib().bit_reverse_secure_field(column.device_ptr, n)
        else:
            L.lib().bit_reverse_base_field(column.device_ptr, n)
        L.check_last()

    # FieldOps::batch_inverse (field.rs:8-30)
    @staticmethod
    def batch_inverse(column, dst):
        L.clear_error()
        if isinstance(column, SecureFieldVec):
            L.lib().batch_inverse_secure_field(column.device_ptr, dst.device_ptr, len(column))
        else:
            L.lib().batch_inverse_base_field(column.device_ptr, dst.device_ptr, len(column))
        L.check_last()

    # PolyOps (poly.rs:20-193)
    @staticmethod
    def new_canonical_ordered(coset, values):
        L.clear_error()
        p = L.lib().sort_values_and_permute_with_bit_reverse_order(values.device_ptr, len(values))
        if not p:
            L.check_last()
        return CircleEvaluation(coset.circle_domain(), BaseFieldVec(p, len(values)))

    @staticmethod
    def precompute_twiddles(coset):
        L.clear_error()
        n = coset.size()
        tw = BaseFieldVec.new_uninitialized(n)
        itw = BaseFieldVec.new_uninitialized(n)
        L.check(L.lib().stwo_precompute_twiddles(coset.initial_index, coset.step_size, coset.log_size,
                                                 tw.device_ptr, itw.device_ptr, None))
        L.check(L.lib().stwo_stream_synchronize(None))
        return TwiddleTree(coset, tw, itw)

    @staticmethod
    def precompute_twiddles_reference_abi(coset):
        """precompute_twiddles through the reference-compatible entry (poly.rs:170-192)."""
        L.clear_error()
        tw = L.lib().precompute_twiddles(L.Point(*coset.initial), L.Point(*coset.step), coset.size())
        if not tw:
            L.check_last()
        tw = BaseFieldVec(tw, coset.size())
        itw = BaseFieldVec.new_uninitialized(coset.size())
        L.lib().batch_inverse_base_field(tw.device_ptr, itw.device_ptr, coset.size())
        L.check_last()
        return TwiddleTree(coset, tw, itw)

    @staticmethod
    def interpolate(evaluation, twiddle_tree):
        assert evaluation.domain.half_coset.is_doubling_of(twiddle_tree.root_coset)
        v = evaluation.values
        L.clear_error()
        L.lib().interpolate(evaluation.domain.half_coset.size(), v.device_ptr, twiddle_tree.itwiddles.device_ptr,
                            len(twiddle_tree.itwiddles), len(v))
        L.check_last()
        return CirclePoly(v)

    @staticmethod
    def interpolate_columns(columns, twiddles):
        columns = list(columns)
        if not columns:
            return []
        logs = [len(c.values).bit_length() - 1 for c in columns]
        L.clear_error()
        L.check(L.lib().stwo_interpolate_columns(L.ptr_array([c.values.device_ptr for c in columns]),
                                                 L.u32_array(logs), len(columns), twiddles.itwiddles.device_ptr,
                                                 len(twiddles.itwiddles), None))
        L.check(L.lib().stwo_stream_synchronize(None))
        return [CirclePoly(c.values) for c in columns]

    @staticmethod
    def eval_at_point(poly, point):
        px, py = point
        L.clear_error()
        r = L.lib().eval_at_point(poly.coeffs.device_ptr, len(poly.coeffs), qm31(px), qm31(py))
        L.check_last()
        return r.tuple()

    @staticmethod
    def extend(poly, log_size):
        new = BaseFieldVec.new_zeroes(1 << log_size)
        assert len(new) >= len(poly.coeffs)
        new.copy_from(poly.coeffs)
        return CirclePoly(new)

    @staticmethod
    def evaluate(poly, domain, twiddle_tree):
        values = CudaBackend.extend(poly, domain.log_size()).coeffs
        assert domain.half_coset.is_doubling_of(twiddle_tree.root_coset)
        L.clear_error()
        L.lib().evaluate(domain.half_coset.size(), values.device_ptr, twiddle_tree.twiddles.device_ptr,
                         len(twiddle_tree.twiddles), len(values))
        L.check_last()
        return CircleEvaluation(domain, values)

    @staticmethod
    def evaluate_polynomials(polynomials, log_blowup_factor, twiddles):
        """Extend + evaluate fused: only the coefficients are read, the blown-up
        evaluations written (poly.rs:128-168 extends first, then transforms)."""
        outs, logs, doms = [], [], []
        for p in polynomials:
            lg = p.log_size()
            logs.append(lg)
            outs.append(BaseFieldVec.new_uninitialized(1 << (lg + log_blowup_factor)))
            doms.append(CanonicCoset(lg + log_blowup_factor).circle_domain())
        if polynomials:
            L.clear_error()
            L.check(L.lib().stwo_extend_evaluate_columns(
                L.ptr_array([p.coeffs.device_ptr for p in polynomials]), L.u32_array(logs),
                L.ptr_array([o.device_ptr for o in outs]), log_blowup_factor, len(outs),
                twiddles.twiddles.device_ptr, len(twiddles.twiddles), None))
            L.check(L.lib().stwo_stream_synchronize(None))
        return [CircleEvaluation(d, o) for d, o in zip(doms, outs)]

    # FriOps (fri.rs:15-75)
    @staticmethod
    def fold_line(evaluation, alpha, twiddles):
        n = len(evaluation.values)
        assert n >= 2, "Evaluation too small"
        remaining_folds = n.bit_length() - 1
        offset = len(twiddles.itwiddles) - (1 << remaining_folds)
        folded = SecureColumnByCoords.uninitialized(n >> 1)
        L.clear_error()
        L.lib().fold_line(twiddles.itwiddles.device_ptr, offset, n, evaluation.values.ptrs(), qm31(alpha),
                          folded.ptrs())
        L.check_last()
        return LineEvaluation(evaluation.domain.double(), folded)

    @staticmethod
    def fold_circle_into_line(dst, src, alpha, twiddles):
        n = len(src.values)
        assert n >> 1 == len(dst.values)
        offset = twiddles.root_coset.size() - dst.domain.size()
        L.clear_error()
        L.lib().fold_circle_into_line(twiddles.itwiddles.device_ptr, offset, n, src.values.ptrs(), qm31(alpha),
                                      dst.values.ptrs())
        L.check_last()

    # MerkleOps<Blake2sMerkleHasher> (blake2s.rs:19-97)
    @staticmethod
    def commit_on_layer(log_size, prev_layer, columns):
        size = 1 << log_size
        result = Blake2sHashVec.new_uninitialized(size)
        L.clear_error()
        L.check(L.lib().stwo_merkle_commit_layer(log_size, prev_layer.device_ptr if prev_layer else None,
                                                 L.ptr_array([c.device_ptr for c in columns]), len(columns),
                                                 result.device_ptr, None))
        L.check(L.lib().stwo_stream_synchronize(None))
        return result

    @staticmethod
    def commit_on_layer_reference_abi(log_size, prev_layer, columns):
        """Through commit_on_first_layer / commit_on_layer_with_previous, whose column
        pointer array lives in device memory (blake2s.rs:55-94)."""
        size = 1 << log_size
        result = Blake2sHashVec.new_uninitialized(size)
        L.clear_error()
        dev_ptrs = L.lib().copy_device_pointer_vec_from_host_to_device(
            L.ptr_array([c.device_ptr for c in columns]), max(1, len(columns)))
        try:
            if prev_layer is None:
                L.lib().commit_on_first_layer(size, len(columns), dev_ptrs, result.device_ptr)
            else:
                L.lib().commit_on_layer_with_previous(size, len(columns), dev_ptrs, prev_layer.device_ptr,
                                                      result.device_ptr)
            L.check_last()
        finally:
            L.lib().cuda_free_memory(dev_ptrs)
        return result

    # QuotientOps (quotient.rs:17-115)
    @staticmethod
    def accumulate_quotients(domain, columns, random_coeff, sample_batches, log_blowup_factor=1):
        n = domain.size()
        out = SecureColumnByCoords.uninitialized(n)
        pts = (L.SPoint * max(1, len(sample_batches)))()
        for i, b in enumerate(sample_batches):
            pts[i] = L.SPoint(qm31(b.point[0]), qm31(b.point[1]))
        sizes = [len(b.columns_and_values) for b in sample_batches]
        idx = [ci for b in sample_batches for ci, _ in b.columns_and_values]
        vals = [v for b in sample_batches for _, v in b.columns_and_values]
        varr = (L.QM31 * max(1, len(vals)))(*[qm31(v) for v in vals])
        L.clear_error()
        L.check(L.lib().stwo_accumulate_quotients(
            domain.half_coset.initial_index, domain.half_coset.step_size, domain.log_size(),
            L.ptr_array([c.values.device_ptr for c in columns]), len(columns), qm31(random_coeff),
            C.cast(pts, C.c_void_p), L.u32_array(sizes), L.u32_array(idx), C.cast(varr, C.c_void_p),
            len(sample_batches), out.ptrs(), None))
        L.check(L.lib().stwo_stream_synchronize(None))
        return SecureEvaluation(domain, out)

    # AccumulationOps (accumulation.rs:9-19)
    @staticmethod
    def accumulate(column, other):
        L.clear_error()
        L.lib().accumulate(len(column), column.ptrs(), other.ptrs())
        L.check_last()
