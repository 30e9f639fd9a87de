"""The C ABI: the library builds for sm_100a, loads, and exports every entry point
include/stwo_b200.h declares (CPU-only; no kernel is launched)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "stwo_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "sizeof")))


def test_header_declares_reference_bindings():
    names = set(declared_functions())
    # every function the reference's Rust FFI binds for the hot path (bindings.rs:75-271),
    # minus the GKR/MLE lookups that are out of scope
    ref = {
        "copy_uint32_t_vec_from_device_to_host", "copy_uint32_t_vec_from_host_to_device",
        "copy_uint32_t_vec_from_device_to_device", "cuda_malloc_uint32_t", "cuda_malloc_blake_2s_hash",
        "cuda_alloc_zeroes_uint32_t", "cuda_alloc_zeroes_blake_2s_hash", "cuda_free_memory",
        "bit_reverse_base_field", "bit_reverse_secure_field", "batch_inverse_base_field",
        "batch_inverse_secure_field", "sort_values_and_permute_with_bit_reverse_order", "precompute_twiddles",
        "interpolate", "interpolate_columns", "evaluate", "evaluate_columns", "eval_at_point", "fold_line",
        "fold_circle_into_line", "accumulate", "commit_on_first_layer", "commit_on_layer_with_previous",
        "copy_blake_2s_hash_vec_from_host_to_device", "copy_blake_2s_hash_vec_from_device_to_host",
        "copy_blake_2s_hash_vec_from_device_to_device", "copy_device_pointer_vec_from_host_to_device",
        "accumulate_quotients", "evaluate_wide_fibonacci_constraint_quotients_on_domain",
    }
    assert ref <= names, ref - names


def test_library_exports_every_declared_symbol(stwo):
    lib = stwo._lib.lib()  # loads libstwo_b200.so (no GPU needed to load)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", stwo._lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    assert set(declared_functions()) <= exported


def test_python_binding_covers_header(stwo):
    bound = {name for name, _, _ in stwo._lib.SIGNATURES}
    assert set(declared_functions()) <= bound, set(declared_functions()) - bound


def test_library_is_built_for_sm100a_only():
    """Every object and the link step are compiled for sm_100a and nothing else."""
    from stwo_gpu_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert build.FLAGS[:2] == build.ARCH
    assert not any("compute_" in f or "sm_" in f for f in build.FLAGS[2:])


def test_last_error_roundtrip_without_gpu(stwo):
    L = stwo._lib
    L.clear_error()
    assert L.last_error() == ""
    # a bad argument is rejected on the host before any CUDA call
    rc = L.lib().stwo_fold_line(L.ptr_array([0, 0, 0, 0]), 3, L.QM31(0, 0, 0, 0), None, 0,
                                L.ptr_array([0, 0, 0, 0]), None)
    assert rc == 1 and "fold" in L.last_error()
    L.clear_error()
