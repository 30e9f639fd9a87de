"""stwo_gpu_b200 — Blackwell-native CUDA backend for the Stwo prover's hot path.

The compute lives in libstwo_b200.so (CUDA for sm_100a behind the C ABI of
include/stwo_b200.h); this package is the host-side mirror of the reference's
backend traits (backend.py), the wide-Fibonacci prover and proof server
(prover.py), a plain-Python verifier (verifier.py) and the ctypes binding (_lib.py).
"""
from . import _lib  # noqa: F401
from .backend import (  # noqa: F401
    BaseFieldVec, Blake2sHashVec, CanonicCoset, CircleDomain, CircleEvaluation, CirclePoly, ColumnSampleBatch,
    Coset, CudaBackend, LineDomain, LineEvaluation, SecureColumnByCoords, SecureEvaluation, SecureFieldVec,
    TwiddleTree, index_to_point,
)
from .prover import (  # noqa: F401
    ProofServer, ProveCache, WideFibJob, kernel_launches, prove_wide_fib, prove_wide_fib_batch, wide_fib_inputs)
from .verifier import VerificationError, verify  # noqa: F401
