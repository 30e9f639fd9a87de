"""The oracle prover (oracle/stwo_oracle_prover.c) against the plain-Python verifier
(stwo_gpu_b200/verifier.py): honest proofs verify, every tampered byte is rejected,
proofs are deterministic. CPU only."""
import numpy as np
import pytest

from conftest import load_package

JOBS = [
    # (log_n_rows, n_columns, log_blowup, n_queries, pow_bits)
    (2, 3, 1, 1, 0),
    (4, 8, 1, 3, 5),
    (5, 3, 1, 3, 0),
    (6, 16, 2, 5, 3),
    (3, 20, 3, 9, 2),
    (7, 33, 4, 20, 8),
    (12, 64, 1, 3, 5),  # the reference CpuBackend's single-proof case: 64 columns, 2^12 rows
]


def inputs(log_n_rows, seed):
    stwo = load_package()
    return stwo.wide_fib_inputs(log_n_rows, seed)


@pytest.mark.parametrize("job", JOBS, ids=lambda j: "L%d_N%d_B%d_q%d_pow%d" % j)
def test_oracle_proof_verifies(oracle, job):
    L, N, B, Q, PW = job
    stwo = load_package()
    a0, a1 = inputs(L, 1000 + L)
    proof, rc = oracle.wide_fib_prove(L, N, a0, a1, B, Q, PW)
    assert rc == 0
    assert stwo.verify(proof, L, N, B, Q, PW)


def test_oracle_proof_is_deterministic(oracle):
    a0, a1 = inputs(6, 7)
    p1, _ = oracle.wide_fib_prove(6, 10, a0, a1)
    p2, _ = oracle.wide_fib_prove(6, 10, a0, a1)
    assert p1 == p2
    a0b = a0.copy()
    a0b[3] = (a0b[3] + 1) % ((1 << 31) - 1)
    p3, _ = oracle.wide_fib_prove(6, 10, a0b, a1)
    assert p3 != p1


def test_every_tampered_byte_is_rejected(oracle):
    stwo = load_package()
    L, N, B, Q, PW = 4, 6, 1, 4, 4
    a0, a1 = inputs(L, 11)
    proof, _ = oracle.wide_fib_prove(L, N, a0, a1, B, Q, PW)
    positions = sorted(set(list(range(0, len(proof), max(1, len(proof) // 150))) + [len(proof) - 1]))
    for pos in positions:
        for bit in (0, 5):
            bad = bytearray(proof)
            bad[pos] ^= 1 << bit
            with pytest.raises(stwo.VerificationError):
                stwo.verify(bytes(bad), L, N, B, Q, PW)
    with pytest.raises(stwo.VerificationError):
        stwo.verify(proof + b"\0", L, N, B, Q, PW)
    with pytest.raises(stwo.VerificationError):
        stwo.verify(proof[:-1], L, N, B, Q, PW)


def test_proof_does_not_verify_under_other_parameters(oracle):
    stwo = load_package()
    a0, a1 = inputs(5, 3)
    proof, _ = oracle.wide_fib_prove(5, 8, a0, a1, 1, 3, 2)
    assert stwo.verify(proof, 5, 8, 1, 3, 2)
    for args in [(5, 9, 1, 3, 2), (5, 8, 1, 4, 2), (5, 8, 1, 3, 12), (6, 8, 1, 3, 2)]:
        with pytest.raises(stwo.VerificationError):
            stwo.verify(proof, *args)


def test_wide_fib_inputs_are_seeded_splitmix64():
    stwo = load_package()
    # independent scalar SplitMix64 (Steele, Lea, Flood 2014)
    M = (1 << 64) - 1

    def sm(seed, k):
        z = (seed + k * 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    a0, a1 = stwo.wide_fib_inputs(3, 42)
    want = [v for v in (sm(42, k) >> 33 for k in range(1, 40)) if v < (1 << 31) - 1][:16]
    assert [int(x) for x in a0] == want[:8]
    assert [int(x) for x in a1] == want[8:16]
    b0, b1 = stwo.wide_fib_inputs(3, 42)
    assert np.array_equal(a0, b0) and np.array_equal(a1, b1)
    c0, _ = stwo.wide_fib_inputs(3, 43)
    assert not np.array_equal(a0, c0)


def test_verifier_channel_matches_blake2s_reference():
    """The verifier's Merkle compression, run as a standard BLAKE2s (parameter block,
    counter, final flag), equals hashlib's BLAKE2s."""
    import hashlib
    import struct
    stwo = load_package()
    V = stwo.verifier
    msg = bytes(range(37))
    h = list(V._IV)
    h[0] ^= 0x01010020
    m = list(struct.unpack("<16I", msg + bytes(64 - len(msg))))
    # one final block: t = len, f0 = all ones (xor into v[12], v[14])
    v = list(h) + list(V._IV)
    v[12] ^= len(msg)
    v[14] ^= 0xFFFFFFFF

    def g(a, b, c, d, x, y):
        v[a] = (v[a] + v[b] + x) & V.M32
        v[d] = V._rotr(v[d] ^ v[a], 16)
        v[c] = (v[c] + v[d]) & V.M32
        v[b] = V._rotr(v[b] ^ v[c], 12)
        v[a] = (v[a] + v[b] + y) & V.M32
        v[d] = V._rotr(v[d] ^ v[a], 8)
        v[c] = (v[c] + v[d]) & V.M32
        v[b] = V._rotr(v[b] ^ v[c], 7)

    for s in V._SIGMA:
        g(0, 4, 8, 12, m[s[0]], m[s[1]]); g(1, 5, 9, 13, m[s[2]], m[s[3]])
        g(2, 6, 10, 14, m[s[4]], m[s[5]]); g(3, 7, 11, 15, m[s[6]], m[s[7]])
        g(0, 5, 10, 15, m[s[8]], m[s[9]]); g(1, 6, 11, 12, m[s[10]], m[s[11]])
        g(2, 7, 8, 13, m[s[12]], m[s[13]]); g(3, 4, 9, 14, m[s[14]], m[s[15]])
    out = struct.pack("<8I", *[h[i] ^ v[i] ^ v[i + 8] for i in range(8)])
    assert out == hashlib.blake2s(msg, digest_size=32).digest()
    # and the zero-counter compression the Merkle hasher uses equals the oracle's
    import oracle as O
    import ctypes as C
    hh = (C.c_uint32 * 8)(*range(8))
    mm = (C.c_uint32 * 16)(*range(100, 116))
    O.lib().or_blake2s_compress(hh, mm, 0, 0, 0, 0)
    assert list(hh) == V.compress(list(range(8)), list(range(100, 116)))
