"""ctypes binding of libstwo_b200.so (the C ABI declared in include/stwo_b200.h).

Loading fails loudly when the library is missing or was built without CUDA: the
package has no CPU fallback.
"""
import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
# STWO_B200_LIB selects another build of the library (for A/B measurements).
LIB_PATH = os.environ.get("STWO_B200_LIB") or os.path.join(PKG, "lib", "libstwo_b200.so")

u32 = C.c_uint32
u64 = C.c_uint64
sz = C.c_size_t
vp = C.c_void_p
u32p = C.POINTER(C.c_uint32)
vpp = C.POINTER(C.c_void_p)


class Point(C.Structure):
    _fields_ = [("x", u32), ("y", u32)]


class QM31(C.Structure):
    _fields_ = [("a", u32), ("b", u32), ("c", u32), ("d", u32)]

    def tuple(self):
        return (self.a, self.b, self.c, self.d)


class SPoint(C.Structure):
    _fields_ = [("x", QM31), ("y", QM31)]


class WideFibJob(C.Structure):
    """stwo_wide_fib_job: one wide-Fibonacci proof's parameters."""
    _fields_ = [("log_n_rows", u32), ("n_columns", u32), ("log_blowup", u32), ("n_queries", u32),
                ("pow_bits", u32)]


class ProveStats(C.Structure):
    """stwo_prove_stats: per-phase wall-clock times and resources of one proof."""
    _fields_ = [("trace_ms", C.c_double), ("composition_ms", C.c_double), ("oods_ms", C.c_double),
                ("fri_ms", C.c_double), ("decommit_ms", C.c_double), ("total_ms", C.c_double),
                ("device_bytes", u64), ("kernel_launches", u64), ("proof_bytes", u64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerResult(C.Structure):
    """stwo_server_result: one finished job of the proof server."""
    _fields_ = [("job_id", u64), ("status", C.c_int), ("error", C.c_char * 256), ("proof", C.POINTER(C.c_uint8)),
                ("proof_len", u64), ("submit_ms", C.c_double), ("start_ms", C.c_double), ("done_ms", C.c_double),
                ("device_done_ms", C.c_double), ("stats", ProveStats)]


class StwoError(RuntimeError):
    pass


# status codes (include/stwo_b200.h)
OK, ERR_INVALID_ARGUMENT, ERR_UNSUPPORTED_SIZE, ERR_OUT_OF_MEMORY, ERR_CUDA, ERR_CANCELLED, ERR_TIMEOUT = range(7)


# (name, restype, argtypes); every symbol declared in include/stwo_b200.h.
SIGNATURES = [
    # reference-compatible tier (stwo_gpu_backend/src/cuda/bindings.rs:75-271)
    ("copy_uint32_t_vec_from_device_to_host", None, [vp, vp, u32]),
    ("copy_uint32_t_vec_from_host_to_device", vp, [vp, u32]),
    ("copy_uint32_t_vec_from_device_to_device", vp, [vp, vp, u32]),
    ("cuda_malloc_uint32_t", vp, [u32]),
    ("cuda_malloc_blake_2s_hash", vp, [sz]),
    ("cuda_alloc_zeroes_uint32_t", vp, [u32]),
    ("cuda_alloc_zeroes_blake_2s_hash", vp, [sz]),
    ("cuda_free_memory", None, [vp]),
    ("copy_blake_2s_hash_vec_from_host_to_device", vp, [vp, sz]),
    ("copy_blake_2s_hash_vec_from_device_to_host", None, [vp, vp, sz]),
    ("copy_blake_2s_hash_vec_from_device_to_device", None, [vp, vp, sz]),
    ("copy_device_pointer_vec_from_host_to_device", vp, [vp, sz]),
    ("bit_reverse_base_field", None, [vp, sz]),
    ("bit_reverse_secure_field", None, [vp, sz]),
    ("batch_inverse_base_field", None, [vp, vp, sz]),
    ("batch_inverse_secure_field", None, [vp, vp, sz]),
    ("sort_values_and_permute_with_bit_reverse_order", vp, [vp, sz]),
    ("precompute_twiddles", vp, [Point, Point, sz]),
    ("interpolate", None, [u32, vp, vp, u32, u32]),
    ("interpolate_columns", None, [u32, vp, vp, u32, u32, u32]),
    ("evaluate", None, [u32, vp, vp, u32, u32]),
    ("evaluate_columns", None, [vp, vp, vp, u32, u32, vp]),
    ("eval_at_point", QM31, [vp, u32, QM31, QM31]),
    ("fold_line", None, [vp, sz, sz, vp, QM31, vp]),
    ("fold_circle_into_line", None, [vp, sz, sz, vp, QM31, vp]),
    ("accumulate", None, [u32, vp, vp]),
    ("commit_on_first_layer", None, [sz, sz, vp, vp]),
    ("commit_on_layer_with_previous", None, [sz, sz, vp, vp, vp]),
    ("accumulate_quotients", None, [u32, u32, u32, vp, sz, QM31, vp, vp, u32, vp, vp, u32, vp, vp, vp, vp, u32]),
    ("evaluate_wide_fibonacci_constraint_quotients_on_domain", None, [vp, vp, vp, vp, vp, vp, vp, u32, u32]),
    # native tier
    ("stwo_last_error", C.c_char_p, []),
    ("stwo_clear_last_error", None, []),
    ("stwo_stream_synchronize", C.c_int, [vp]),
    ("stwo_precompute_twiddles", C.c_int, [u32, u32, u32, vp, vp, vp]),
    ("stwo_interpolate_columns", C.c_int, [vp, vp, u32, vp, u64, vp]),
    ("stwo_evaluate_columns", C.c_int, [vp, vp, u32, vp, u64, vp]),
    ("stwo_extend_evaluate_columns", C.c_int, [vp, vp, vp, u32, u32, vp, u64, vp]),
    ("stwo_bit_reverse_m31", C.c_int, [vp, u64, vp]),
    ("stwo_bit_reverse_qm31", C.c_int, [vp, u64, vp]),
    ("stwo_new_canonical_ordered", C.c_int, [vp, vp, u32, vp]),
    ("stwo_batch_inverse_m31", C.c_int, [vp, vp, u64, vp]),
    ("stwo_batch_inverse_qm31", C.c_int, [vp, vp, u64, vp]),
    ("stwo_eval_at_points_scratch_bytes", sz, [vp, u32]),
    ("stwo_eval_at_points", C.c_int, [vp, vp, u32, vp, vp, vp, sz, vp]),
    ("stwo_eval_at_point_no_alloc", C.c_int, [vp, u32, QM31, QM31, vp, vp]),
    ("stwo_fold_line", C.c_int, [vp, u64, QM31, vp, u64, vp, vp]),
    ("stwo_fold_circle_into_line", C.c_int, [vp, u64, QM31, vp, u64, vp, vp]),
    ("stwo_accumulate", C.c_int, [vp, vp, u64, vp]),
    ("stwo_merkle_commit_layer", C.c_int, [u32, vp, vp, u32, vp, vp]),
    ("stwo_merkle_commit_tree", C.c_int, [vp, vp, u32, u32, vp, vp]),
    ("stwo_accumulate_quotients", C.c_int, [u32, u32, u32, vp, u32, QM31, vp, vp, vp, vp, u32, vp, vp]),
    ("stwo_quotients_tc_faults", C.c_int, [C.POINTER(u32), C.c_int]),
    ("stwo_composition_tc_faults", C.c_int, [C.POINTER(u32), C.c_int]),
    ("stwo_wide_fib_composition", C.c_int, [vp, u32, u32, vp, vp, vp, vp]),
    ("stwo_kernel_launches", u64, []),
    ("stwo_reserve_device_memory", C.c_int, [u64]),
    ("stwo_autotune", C.c_int, [C.c_char_p, sz]),
    ("stwo_set_tunable", C.c_int, [C.c_char_p, C.c_int]),
    # prover tier
    ("stwo_wide_fib_prove_device_bytes", u64, [C.POINTER(WideFibJob), C.c_int]),
    ("stwo_wide_fib_prove", C.c_int, [C.POINTER(WideFibJob), vp, vp, vp, vp, u64, C.POINTER(C.POINTER(C.c_uint8)),
                                      C.POINTER(u64), C.POINTER(ProveStats), vp]),
    ("stwo_wide_fib_prove_batch", C.c_int, [C.POINTER(WideFibJob), u32, vp, vp, vp, vp, u64,
                                            C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(u64), C.POINTER(C.c_int),
                                            C.POINTER(ProveStats), vp]),
    ("stwo_free_proof", None, [vp]),
    ("stwo_prove_cache_create", vp, []),
    ("stwo_wide_fib_prove_cached", C.c_int, [vp, C.POINTER(WideFibJob), vp, vp, vp, vp, u64,
                                             C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(u64),
                                             C.POINTER(ProveStats), vp]),
    ("stwo_prove_cache_stats", None, [vp, C.POINTER(u64), C.POINTER(u64)]),
    ("stwo_prove_cache_destroy", None, [vp, vp]),
    ("stwo_server_create", vp, [u32, u64, u32]),
    ("stwo_server_submit", C.c_int, [vp, u64, C.POINTER(WideFibJob), vp, vp]),
    ("stwo_server_submit_device", C.c_int, [vp, u64, C.POINTER(WideFibJob), vp, vp]),
    ("stwo_server_poll", u32, [vp, C.POINTER(ServerResult), u32, C.c_int32]),
    ("stwo_server_stats", None, [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u64)]),
    ("stwo_server_graph_stats", None, [vp, C.POINTER(u64), C.POINTER(u64)]),
    ("stwo_server_batch_stats", None, [vp, C.POINTER(u64), C.POINTER(u64)]),
    ("stwo_server_now_ms", C.c_double, []),
    ("stwo_server_mark_epoch", C.c_int, [vp]),
    ("stwo_probe_m31_butterflies", C.c_int, [u32, vp, u64, C.POINTER(u64), vp]),
    ("stwo_server_destroy", None, [vp]),
    ("stwo_server_cancel", C.c_int, [vp, u64]),
    ("stwo_server_pause", C.c_int, [vp, C.c_int]),
    ("stwo_server_set_queue_timeout", C.c_int, [vp, C.c_double]),
    ("stwo_debug_fail_allocations", None, [u32]),
]

_lib = None


def lib():
    """The loaded library; raises if it is absent (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m stwo_gpu_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().stwo_last_error().decode()


def check(status):
    """Raise on a non-zero status; the raise consumes the recorded message, so a later
    check_last() does not see it again."""
    if status != 0:
        msg = last_error()
        clear_error()
        raise StwoError(f"stwo_b200 status {status}: {msg}")


def clear_error():
    lib().stwo_clear_last_error()


def check_last():
    """After a reference-compatible (void) call: raise if it recorded an error."""
    msg = last_error()
    if msg:
        clear_error()
        raise StwoError(msg)


def ptr_array(ptrs):
    return (C.c_void_p * max(1, len(ptrs)))(*ptrs)


def u32_array(vals):
    return (C.c_uint32 * max(1, len(vals)))(*vals)
