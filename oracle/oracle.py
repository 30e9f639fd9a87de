"""ctypes front end of the CPU oracle (libstwo_oracle.so) — TEST INFRASTRUCTURE ONLY.

The oracle restates stwo CpuBackend (see stwo_oracle.c). Only tests/, the smoke
check and the CPU-baseline leg of bench.py may import this module, and only to
check or time the reference algorithm; the product never calls it.

Field elements travel as numpy uint32 arrays. QM31 values are numpy arrays of
shape (..., 4) in coordinate order (a.a, a.b, b.a, b.b), i.e. the order of the
reference's repr(C) CudaSecureField {a, b, c, d} (stwo_gpu_backend/src/cuda/bindings.rs:8-14).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstwo_oracle.so")
P = (1 << 31) - 1

_u32p = C.POINTER(C.c_uint32)


class CM31(C.Structure):
    _fields_ = [("a", C.c_uint32), ("b", C.c_uint32)]


class QM31(C.Structure):
    _fields_ = [("a", CM31), ("b", CM31)]


class CPoint(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32)]


class SPoint(C.Structure):
    _fields_ = [("x", QM31), ("y", QM31)]


class Coset(C.Structure):
    _fields_ = [("initial_index", C.c_uint32), ("step_size", C.c_uint32), ("log_size", C.c_uint32)]


class WideFibJob(C.Structure):
    _fields_ = [("log_n_rows", C.c_uint32), ("n_columns", C.c_uint32), ("log_blowup", C.c_uint32),
                ("n_queries", C.c_uint32), ("pow_bits", C.c_uint32)]


def build():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_m31_mul.restype = C.c_uint32
        L.or_m31_inv.restype = C.c_uint32
        L.or_qm31_mul.restype = QM31
        L.or_qm31_mul.argtypes = [QM31, QM31]
        L.or_qm31_inv.restype = QM31
        L.or_qm31_inv.argtypes = [QM31]
        L.or_qm31_pow.restype = QM31
        L.or_qm31_pow.argtypes = [QM31, C.c_uint64]
        L.or_index_to_point.restype = CPoint
        L.or_index_to_point.argtypes = [C.c_uint32]
        L.or_coset_at.restype = CPoint
        L.or_coset_at.argtypes = [Coset, C.c_uint64]
        L.or_circle_domain_at.restype = CPoint
        L.or_circle_domain_at.argtypes = [Coset, C.c_uint64]
        L.or_bit_reverse_index.restype = C.c_uint32
        L.or_canonic_half_coset.restype = Coset
        L.or_canonic_coset.restype = Coset
        L.or_interpolate.argtypes = [Coset, _u32p, _u32p, C.c_size_t]
        L.or_evaluate.argtypes = [Coset, _u32p, _u32p, C.c_size_t]
        L.or_evaluate_direct.argtypes = [Coset, _u32p, C.c_uint32, _u32p]
        L.or_precompute_twiddles.argtypes = [Coset, _u32p, _u32p]
        L.or_wide_fib_prove.argtypes = [C.POINTER(WideFibJob), C.c_void_p, C.c_void_p,
                                        C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]
        L.or_free.argtypes = [C.c_void_p]
        L.or_eval_at_point.restype = QM31
        L.or_eval_at_point.argtypes = [_u32p, C.c_uint32, SPoint]
        L.or_line_eval_at_point.restype = QM31
        L.or_line_eval_at_point.argtypes = [C.c_void_p, C.c_uint32, QM31]
        L.or_fold_line.argtypes = [C.c_void_p, C.c_size_t, Coset, QM31, C.c_void_p]
        L.or_fold_circle_into_line.argtypes = [C.c_void_p, C.c_size_t, Coset, QM31, C.c_void_p]
        L.or_merkle_commit_on_layer.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        L.or_blake2s_std.argtypes = [C.c_char_p, C.c_size_t, C.c_void_p]
        L.or_blake2s_compress.argtypes = [C.c_void_p, C.c_void_p] + [C.c_uint32] * 4
        L.or_accumulate_quotients.argtypes = [Coset, C.c_void_p, C.c_size_t, QM31, C.c_size_t, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_accumulate.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.or_coset_vanishing_m31.restype = C.c_uint32
        L.or_coset_vanishing_m31.argtypes = [Coset, CPoint]
        L.or_wide_fib_trace_row.argtypes = [C.c_uint32, C.c_uint32, C.c_size_t, _u32p]
        L.or_wide_fib_composition.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, _u32p, C.c_void_p]
        L.or_new_canonical_ordered.argtypes = [C.c_uint32, _u32p, _u32p]
        L.or_batch_inverse_m31.argtypes = [_u32p, _u32p, C.c_size_t]
        L.or_batch_inverse_qm31.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.or_bit_reverse_u32.argtypes = [_u32p, C.c_size_t]
        L.or_bit_reverse_qm31.argtypes = [C.c_void_p, C.c_size_t]
        L.or_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


# ---------------------------------------------------------------- helpers
def _p(a):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def _ptr_array(cols):
    arr = (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])
    return arr


def qm31(v):
    v = [int(x) for x in v]
    return QM31(CM31(v[0], v[1]), CM31(v[2], v[3]))


def qm31_tuple(q):
    return (q.a.a, q.a.b, q.b.a, q.b.b)


def coset(initial_index, step_size, log_size):
    return Coset(initial_index, step_size, log_size)


def canonic_half_coset(domain_log_size):
    return lib().or_canonic_half_coset(domain_log_size)


def canonic_coset(log_size):
    return lib().or_canonic_coset(log_size)


def coset_double(c, times=1):
    for _ in range(times):
        c = Coset((c.initial_index * 2) & 0x7FFFFFFF, (c.step_size * 2) & 0x7FFFFFFF, c.log_size - 1)
    return c


def index_to_point(i):
    p = lib().or_index_to_point(i)
    return (p.x, p.y)


def set_threads(n):
    lib().or_set_threads(int(n))


# ---------------------------------------------------------------- ops
def precompute_twiddles(root):
    n = 1 << root.log_size
    tw = np.zeros(n, np.uint32)
    itw = np.zeros(n, np.uint32)
    lib().or_precompute_twiddles(root, _p(tw), _p(itw))
    return tw, itw


def interpolate(half_coset, values, itwiddles):
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    itw = np.ascontiguousarray(itwiddles, dtype=np.uint32)
    rc = lib().or_interpolate(half_coset, _p(v), _p(itw), itw.size)
    assert rc == 0
    return v


def evaluate(half_coset, coeffs, twiddles):
    n = 1 << (half_coset.log_size + 1)
    v = np.zeros(n, np.uint32)
    v[: len(coeffs)] = coeffs
    tw = np.ascontiguousarray(twiddles, dtype=np.uint32)
    rc = lib().or_evaluate(half_coset, _p(v), _p(tw), tw.size)
    assert rc == 0
    return v


def evaluate_direct(half_coset, coeffs):
    n = 1 << (half_coset.log_size + 1)
    c = np.ascontiguousarray(coeffs, dtype=np.uint32)
    out = np.zeros(n, np.uint32)
    lib().or_evaluate_direct(half_coset, _p(c), int(c.size).bit_length() - 1, _p(out))
    return out


def eval_at_point(coeffs, px, py):
    c = np.ascontiguousarray(coeffs, dtype=np.uint32)
    sp = SPoint(qm31(px), qm31(py))
    return qm31_tuple(lib().or_eval_at_point(_p(c), int(c.size).bit_length() - 1, sp))


def line_eval_at_point(coeffs_q, x):
    c = np.ascontiguousarray(coeffs_q, dtype=np.uint32).reshape(-1, 4)
    return qm31_tuple(lib().or_line_eval_at_point(c.ctypes.data, int(len(c)).bit_length() - 1, qm31(x)))


def new_canonical_ordered(log_size, values):
    src = np.ascontiguousarray(values, dtype=np.uint32)
    dst = np.zeros_like(src)
    lib().or_new_canonical_ordered(log_size, _p(src), _p(dst))
    return dst


def bit_reverse(values):
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    if v.ndim == 2:
        lib().or_bit_reverse_qm31(v.ctypes.data, len(v))
    else:
        lib().or_bit_reverse_u32(_p(v), v.size)
    return v


def batch_inverse_m31(values):
    src = np.ascontiguousarray(values, dtype=np.uint32)
    dst = np.zeros_like(src)
    lib().or_batch_inverse_m31(_p(src), _p(dst), src.size)
    return dst


def batch_inverse_qm31(values):
    src = np.ascontiguousarray(values, dtype=np.uint32).reshape(-1, 4)
    dst = np.zeros_like(src)
    lib().or_batch_inverse_qm31(src.ctypes.data, dst.ctypes.data, len(src))
    return dst


def fold_line(cols4, line_domain, alpha):
    src = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols4]
    n = src[0].size
    dst = [np.zeros(n // 2, np.uint32) for _ in range(4)]
    lib().or_fold_line(_ptr_array(src), n, line_domain, qm31(alpha), _ptr_array(dst))
    return dst


def fold_circle_into_line(dst4, src4, circle_half_coset, alpha):
    src = [np.ascontiguousarray(c, dtype=np.uint32) for c in src4]
    dst = [np.ascontiguousarray(c, dtype=np.uint32).copy() for c in dst4]
    lib().or_fold_circle_into_line(_ptr_array(src), src[0].size, circle_half_coset, qm31(alpha),
                                   _ptr_array(dst))
    return dst


def merkle_commit_on_layer(log_size, prev, cols):
    n = 1 << log_size
    out = np.zeros((n, 8), np.uint32)
    cs = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    prev_p = None
    if prev is not None:
        prev = np.ascontiguousarray(prev, dtype=np.uint32)
        prev_p = prev.ctypes.data
    lib().or_merkle_commit_on_layer(log_size, prev_p, _ptr_array(cs) if cs else None, len(cs),
                                    out.ctypes.data)
    return out


def merkle_commit(columns):
    """All layers of a Merkle tree over columns of (possibly) mixed power-of-two
    sizes: columns sorted by decreasing length, each layer hashes the previous
    layer's children, then that layer's columns (MerkleProver::commit)."""
    cols = sorted(columns, key=lambda c: -len(c))
    max_log = len(cols[0]).bit_length() - 1
    layers, prev = [], None
    for lg in range(max_log, -1, -1):
        layer_cols = [c for c in cols if len(c) == (1 << lg)]
        prev = merkle_commit_on_layer(lg, prev, layer_cols)
        layers.append(prev)
    layers.reverse()
    return layers


def blake2s_std(data: bytes):
    out = C.create_string_buffer(32)
    lib().or_blake2s_std(data, len(data), out)
    return out.raw


def accumulate_quotients(half_coset, columns, random_coeff, batches):
    """batches: list of (point_x(4), point_y(4), [(col_index, value(4)), ...])."""
    n = 1 << (half_coset.log_size + 1)
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in columns]
    pts = (SPoint * max(1, len(batches)))()
    sizes = np.array([len(b[2]) for b in batches] or [0], np.uint32)
    idx = np.array([ci for b in batches for ci, _ in b[2]] or [0], np.uint32)
    vals = np.array([v for b in batches for _, v in b[2]] or [[0, 0, 0, 0]], np.uint32).reshape(-1, 4)
    for i, b in enumerate(batches):
        pts[i] = SPoint(qm31(b[0]), qm31(b[1]))
    out = [np.zeros(n, np.uint32) for _ in range(4)]
    lib().or_accumulate_quotients(half_coset, _ptr_array(cols), len(cols), qm31(random_coeff), len(batches),
                                  C.cast(pts, C.c_void_p), sizes.ctypes.data, idx.ctypes.data,
                                  vals.ctypes.data, _ptr_array(out))
    return out


def accumulate(left4, right4):
    left = [np.ascontiguousarray(c, dtype=np.uint32).copy() for c in left4]
    right = [np.ascontiguousarray(c, dtype=np.uint32) for c in right4]
    lib().or_accumulate(_ptr_array(left), _ptr_array(right), left[0].size)
    return left


def coset_vanishing(c, p):
    return lib().or_coset_vanishing_m31(c, CPoint(*p))


def wide_fib_trace(n_columns, a, b):
    rows = len(a)
    trace = np.zeros((rows, n_columns), np.uint32)
    row = np.zeros(n_columns, np.uint32)
    for r in range(rows):
        lib().or_wide_fib_trace_row(int(a[r]), int(b[r]), n_columns, _p(row))
        trace[r] = row
    return np.ascontiguousarray(trace.T)


def wide_fib_composition(trace_evals, coeff_powers, den_inv):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in trace_evals]
    ext = cols[0].size
    pw = np.ascontiguousarray(coeff_powers, dtype=np.uint32).reshape(-1, 4)
    di = np.ascontiguousarray(den_inv, dtype=np.uint32)
    out = [np.zeros(ext, np.uint32) for _ in range(4)]
    lib().or_wide_fib_composition(_ptr_array(cols), len(cols), ext, pw.ctypes.data, _p(di), _ptr_array(out))
    return out


# ---------------------------------------------------------------- scalar field helpers (pure Python)
def m31_mul(a, b):
    return (a * b) % P


def qm31_mul(x, y):
    return qm31_tuple(lib().or_qm31_mul(qm31(x), qm31(y)))


def qm31_inv(x):
    return qm31_tuple(lib().or_qm31_inv(qm31(x)))


def qm31_pow(x, e):
    return qm31_tuple(lib().or_qm31_pow(qm31(x), e))


def wide_fib_prove(log_n_rows, n_columns, a0, a1, log_blowup=1, n_queries=3, pow_bits=5):
    """The oracle prover's proof bytes (stwo_oracle_prover.c) and its status (0, or
    -2 / -3 when the OODS / last-layer check failed)."""
    a0 = np.ascontiguousarray(a0, dtype=np.uint32)
    a1 = np.ascontiguousarray(a1, dtype=np.uint32)
    out = C.POINTER(C.c_uint8)()
    ln = C.c_size_t()
    job = WideFibJob(log_n_rows, n_columns, log_blowup, n_queries, pow_bits)
    rc = lib().or_wide_fib_prove(C.byref(job), a0.ctypes.data, a1.ctypes.data, C.byref(out), C.byref(ln))
    if rc == -1:
        raise ValueError("unsupported wide-Fibonacci job")
    try:
        return C.string_at(out, ln.value), rc
    finally:
        lib().or_free(out)
