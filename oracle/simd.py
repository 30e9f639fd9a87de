"""ctypes front end of the SIMD CPU baseline (libstwo_simd_avx512.so / _avx2.so) —
BASELINE AND TEST INFRASTRUCTURE ONLY.

The library is the oracle prover's protocol code on vectorised, multi-threaded
restatements of its heavy functions (stwo_simd.cc): a stand-in for stwo's
SimdBackend, whose proof bytes equal the oracle prover's. The benchmark times it as
the reference CPU path; the tests compare each function with the scalar oracle. The
AVX-512 build is loaded where the host has AVX-512, else the AVX2 build.
"""
import ctypes as C
import os

import numpy as np

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return {"avx512f", "avx512bw", "avx512dq", "avx512vl"} <= flags
    except OSError:
        pass
    return False


def variant():
    return "avx512" if _cpu_has_avx512() else "avx2"


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, f"libstwo_simd_{variant()}.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", HERE])
        L = C.CDLL(path)
        _u32p = C.POINTER(C.c_uint32)
        L.simd_set_threads.argtypes = [C.c_int]
        L.simd_lane_count.restype = C.c_int
        L.simd_wide_fib_prove.argtypes = [C.POINTER(O.WideFibJob), C.c_void_p, C.c_void_p,
                                          C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_size_t)]
        L.simd_free.argtypes = [C.c_void_p]
        L.simd_interpolate.argtypes = [O.Coset, _u32p, _u32p, C.c_size_t]
        L.simd_evaluate.argtypes = [O.Coset, _u32p, _u32p, C.c_size_t]
        L.simd_precompute_twiddles.argtypes = [O.Coset, _u32p, _u32p]
        L.simd_merkle_commit_on_layer.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
        L.simd_accumulate_quotients.argtypes = [O.Coset, C.c_void_p, C.c_size_t, O.QM31, C.c_size_t, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.simd_wide_fib_composition.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, _u32p, C.c_void_p]
        L.simd_eval_at_point.restype = O.QM31
        L.simd_eval_at_point.argtypes = [_u32p, C.c_uint32, O.SPoint]
        L.simd_fold_line.argtypes = [C.c_void_p, C.c_size_t, O.Coset, O.QM31, C.c_void_p]
        L.simd_fold_circle_into_line.argtypes = [C.c_void_p, C.c_size_t, O.Coset, O.QM31, C.c_void_p]
        L.simd_vanishing_inverses.argtypes = [C.c_uint32, _u32p]
        L.simd_wide_fib_trace.argtypes = [_u32p, _u32p, C.c_size_t, C.c_size_t, C.c_void_p]
        _lib = L
    return _lib


def set_threads(n):
    lib().simd_set_threads(int(n))


def lanes():
    return lib().simd_lane_count()


def _p(a):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _ptrs(cols):
    return (C.c_void_p * len(cols))(*[c.ctypes.data for c in cols])


def wide_fib_prove(log_n_rows, n_columns, a0, a1, log_blowup=1, n_queries=3, pow_bits=5):
    """Proof bytes of the SIMD prover and its status (as oracle.wide_fib_prove)."""
    a0 = np.ascontiguousarray(a0, dtype=np.uint32)
    a1 = np.ascontiguousarray(a1, dtype=np.uint32)
    out = C.POINTER(C.c_uint8)()
    ln = C.c_size_t()
    job = O.WideFibJob(log_n_rows, n_columns, log_blowup, n_queries, pow_bits)
    rc = lib().simd_wide_fib_prove(C.byref(job), a0.ctypes.data, a1.ctypes.data, C.byref(out), C.byref(ln))
    if rc == -1:
        raise ValueError("unsupported wide-Fibonacci job")
    try:
        return C.string_at(out, ln.value), rc
    finally:
        lib().simd_free(out)


def precompute_twiddles(root):
    n = 1 << root.log_size
    tw, itw = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    lib().simd_precompute_twiddles(root, _p(tw), _p(itw))
    return tw, itw


def interpolate(half_coset, values, itwiddles):
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    itw = np.ascontiguousarray(itwiddles, dtype=np.uint32)
    assert lib().simd_interpolate(half_coset, _p(v), _p(itw), itw.size) == 0
    return v


def evaluate(half_coset, coeffs, twiddles):
    v = np.zeros(1 << (half_coset.log_size + 1), np.uint32)
    v[: len(coeffs)] = coeffs
    tw = np.ascontiguousarray(twiddles, dtype=np.uint32)
    assert lib().simd_evaluate(half_coset, _p(v), _p(tw), tw.size) == 0
    return v


def merkle_commit_on_layer(log_size, prev, cols):
    out = np.zeros((1 << log_size, 8), np.uint32)
    cs = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols]
    prev_p = None if prev is None else np.ascontiguousarray(prev, dtype=np.uint32).ctypes.data
    lib().simd_merkle_commit_on_layer(log_size, prev_p, _ptrs(cs) if cs else None, len(cs), out.ctypes.data)
    return out


def accumulate_quotients(half_coset, columns, random_coeff, batches):
    n = 1 << (half_coset.log_size + 1)
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in columns]
    pts = (O.SPoint * max(1, len(batches)))()
    sizes = np.array([len(b[2]) for b in batches] or [0], np.uint32)
    idx = np.array([ci for b in batches for ci, _ in b[2]] or [0], np.uint32)
    vals = np.array([v for b in batches for _, v in b[2]] or [[0, 0, 0, 0]], np.uint32).reshape(-1, 4)
    for i, b in enumerate(batches):
        pts[i] = O.SPoint(O.qm31(b[0]), O.qm31(b[1]))
    out = [np.zeros(n, np.uint32) for _ in range(4)]
    lib().simd_accumulate_quotients(half_coset, _ptrs(cols), len(cols), O.qm31(random_coeff), len(batches),
                                    C.cast(pts, C.c_void_p), sizes.ctypes.data, idx.ctypes.data, vals.ctypes.data,
                                    _ptrs(out))
    return out


def wide_fib_composition(trace_evals, coeff_powers, den_inv):
    cols = [np.ascontiguousarray(c, dtype=np.uint32) for c in trace_evals]
    ext = cols[0].size
    pw = np.ascontiguousarray(coeff_powers, dtype=np.uint32).reshape(-1, 4)
    di = np.ascontiguousarray(den_inv, dtype=np.uint32)
    out = [np.zeros(ext, np.uint32) for _ in range(4)]
    lib().simd_wide_fib_composition(_ptrs(cols), len(cols), ext, pw.ctypes.data, _p(di), _ptrs(out))
    return out


def eval_at_point(coeffs, px, py):
    c = np.ascontiguousarray(coeffs, dtype=np.uint32)
    return O.qm31_tuple(lib().simd_eval_at_point(_p(c), int(c.size).bit_length() - 1,
                                                 O.SPoint(O.qm31(px), O.qm31(py))))


def fold_line(cols4, line_domain, alpha):
    src = [np.ascontiguousarray(c, dtype=np.uint32) for c in cols4]
    n = src[0].size
    dst = [np.zeros(n // 2, np.uint32) for _ in range(4)]
    lib().simd_fold_line(_ptrs(src), n, line_domain, O.qm31(alpha), _ptrs(dst))
    return dst


def fold_circle_into_line(dst4, src4, circle_half_coset, alpha):
    src = [np.ascontiguousarray(c, dtype=np.uint32) for c in src4]
    dst = [np.ascontiguousarray(c, dtype=np.uint32).copy() for c in dst4]
    lib().simd_fold_circle_into_line(_ptrs(src), src[0].size, circle_half_coset, O.qm31(alpha), _ptrs(dst))
    return dst


def vanishing_inverses(log_n_rows):
    out = np.zeros(2 << log_n_rows, np.uint32)
    lib().simd_vanishing_inverses(log_n_rows, _p(out))
    return out


def wide_fib_trace(n_columns, a0, a1):
    a0 = np.ascontiguousarray(a0, dtype=np.uint32)
    a1 = np.ascontiguousarray(a1, dtype=np.uint32)
    cols = [np.zeros(a0.size, np.uint32) for _ in range(n_columns)]
    lib().simd_wide_fib_trace(_p(a0), _p(a1), a0.size, n_columns, _ptrs(cols))
    return cols
