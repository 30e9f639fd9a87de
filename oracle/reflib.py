"""ctypes binding of the reference's own CUDA library (oracle/_ref/libgpubackend_ref.so,
built unmodified from the reference sources by oracle/ref.mk) — TEST INFRASTRUCTURE ONLY.

Used by the GPU tests as a second, independent cross-check of our kernels (the
reference's Rust tests assert these functions equal CpuBackend) and by bench.py to
time the reference's GPU path on the same box. Signatures follow the reference's C
headers (cuda/include/*.cuh). Only calls whose memory accesses stay in bounds are made:
the reference reads out of bounds for FFTs of fewer than 8 points, batch inverses of
fewer than 512 (M31) / 1024 (QM31) elements and eval_at_point below 512
coefficients, and clones `extended_domain_size` column pointers in the wide-Fibonacci
entry point (callers pass a host array of that length).
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libgpubackend_ref.so")

i32, u32, vp = C.c_int, C.c_uint32, C.c_void_p


class Point(C.Structure):
    _fields_ = [("x", u32), ("y", u32)]


class QM31(C.Structure):
    _fields_ = [("a", u32), ("b", u32), ("c", u32), ("d", u32)]


SIGS = [
    ("interpolate", None, [i32, vp, vp, i32, i32]),
    ("interpolate_columns", None, [i32, vp, vp, i32, i32, i32]),
    ("evaluate", None, [i32, vp, vp, i32, i32]),
    ("evaluate_columns", None, [vp, vp, vp, i32, i32, vp]),
    ("precompute_twiddles", vp, [Point, Point, i32]),
    ("batch_inverse_base_field", None, [vp, vp, i32]),
    ("batch_inverse_secure_field", None, [vp, vp, i32]),
    ("bit_reverse_base_field", None, [vp, i32]),
    ("bit_reverse_secure_field", None, [vp, i32]),
    ("fold_line", None, [vp, u32, u32, vp, QM31, vp]),
    ("fold_circle_into_line", None, [vp, u32, u32, vp, QM31, vp]),
    ("accumulate", None, [i32, vp, vp]),
    ("commit_on_first_layer", None, [u32, u32, vp, vp]),
    ("commit_on_layer_with_previous", None, [u32, u32, vp, vp, vp]),
    ("accumulate_quotients", None, [u32, u32, u32, vp, u32, QM31, vp, vp, u32, vp, vp, u32, vp, vp, vp, vp, u32]),
    ("evaluate_wide_fibonacci_constraint_quotients_on_domain", None, [vp, vp, vp, vp, vp, vp, vp, u32, u32]),
    ("cuda_alloc_zeroes_uint32_t", vp, [i32]),
    ("copy_uint32_t_vec_from_device_to_device", None, [vp, vp, i32]),
    ("cuda_free_memory", None, [vp]),
    ("copy_device_pointer_vec_from_host_to_device", vp, [vp, u32]),
]

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
