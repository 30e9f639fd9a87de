"""Wide-Fibonacci proving on the GPU: one proof (`prove_wide_fib`) and the proof
server (`ProofServer`, continuous batching of many jobs on one device).

These wrap the prover tier of include/stwo_b200.h. The reference runs the same proof
through stwo's Rust prove() over its CudaBackend
(stwo_gpu_backend/src/examples/wide_fibonacci.rs:205-250); here the whole prover is
native (csrc/prover.cu, csrc/server.cu) and the proof bytes are checked by
`verifier.verify`.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

P = (1 << 31) - 1


@dataclass(frozen=True)
class WideFibJob:
    """PcsConfig{pow_bits, FriConfig{0, log_blowup, n_queries}} over a wide-Fibonacci
    trace of 2^log_n_rows rows and n_columns columns."""
    log_n_rows: int
    n_columns: int
    log_blowup: int = 1
    n_queries: int = 3
    pow_bits: int = 5

    def c(self):
        return L.WideFibJob(self.log_n_rows, self.n_columns, self.log_blowup, self.n_queries, self.pow_bits)

    def device_bytes(self, own_twiddles=True):
        return int(L.lib().stwo_wide_fib_prove_device_bytes(C.byref(self.c()), int(own_twiddles)))


def splitmix64(seed, count):
    """SplitMix64 outputs 1..count for `seed` (uint64 numpy array)."""
    k = np.arange(1, count + 1, dtype=np.uint64)
    z = np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def wide_fib_inputs(log_n_rows, seed):
    """Seeded trace inputs: 2 * 2^log_n_rows uniform M31 values in [0, P), the top 31
    bits of SplitMix64 outputs with the value P rejected; a0 takes the first half,
    a1 the second."""
    n = 1 << log_n_rows
    need, draw = 2 * n, 2 * n + 64
    while True:
        v = (splitmix64(seed, draw) >> np.uint64(33)).astype(np.uint32)
        v = v[v < P]
        if v.size >= need:
            return np.ascontiguousarray(v[:n]), np.ascontiguousarray(v[n:need])
        draw *= 2


class ProveCache:
    """Device memory (and the CUDA graph of the launch sequence) kept between proofs of
    one job shape: pass it to prove_wide_fib with a twiddle tree; the second proof of
    a shape captures the graph, later ones replay it (include/stwo_b200.h)."""

    def __init__(self):
        self._c = L.lib().stwo_prove_cache_create()
        if not self._c:
            raise MemoryError("proof cache allocation failed")

    def stats(self):
        b, r = C.c_uint64(), C.c_uint64()
        L.lib().stwo_prove_cache_stats(self._c, C.byref(b), C.byref(r))
        return {"device_bytes": b.value, "graph_replays": r.value}

    def close(self, stream=None):
        if self._c:
            L.lib().stwo_prove_cache_destroy(self._c, stream)
            self._c = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def prove_wide_fib(job, a0, a1, twiddles=None, stream=None, cache=None):
    """Proves one job; returns (proof bytes, per-phase stats dict). a0, a1: host
    uint32 arrays of 2^log_n_rows M31 values. twiddles: optional TwiddleTree covering
    CanonicCoset(log_n_rows + 1 + log_blowup). cache: optional ProveCache (needs
    twiddles) for repeated proofs of one shape."""
    a0 = np.ascontiguousarray(a0, dtype=np.uint32)
    a1 = np.ascontiguousarray(a1, dtype=np.uint32)
    n = 1 << job.log_n_rows
    if a0.size != n or a1.size != n:
        raise ValueError(f"a0 and a1 need {n} values")
    out = C.POINTER(C.c_uint8)()
    ln = C.c_uint64()
    st = L.ProveStats()
    tw = itw = None
    tsz = 0
    if twiddles is not None:
        tw, itw, tsz = twiddles.twiddles.device_ptr, twiddles.itwiddles.device_ptr, len(twiddles.twiddles)
    L.clear_error()
    if cache is not None:
        L.check(L.lib().stwo_wide_fib_prove_cached(cache._c, C.byref(job.c()), a0.ctypes.data, a1.ctypes.data, tw,
                                                   itw, tsz, C.byref(out), C.byref(ln), C.byref(st), stream))
    else:
        L.check(L.lib().stwo_wide_fib_prove(C.byref(job.c()), a0.ctypes.data, a1.ctypes.data, tw, itw, tsz,
                                            C.byref(out), C.byref(ln), C.byref(st), stream))
    try:
        proof = C.string_at(out, ln.value)
    finally:
        L.lib().stwo_free_proof(out)
    return proof, st.as_dict()


def prove_wide_fib_batch(job, inputs, twiddles, stream=None):
    """Proves len(inputs) jobs of one shape in one launch sequence (every kernel of the
    proof launched once for all of them); inputs: a list of (a0, a1) host uint32
    arrays. Returns (list of proof bytes, or None for a job that failed, list of
    statuses, stats dict of the whole sequence). The proofs are byte for byte those of
    prove_wide_fib. twiddles: a TwiddleTree covering CanonicCoset(log_n_rows + 1 +
    log_blowup)."""
    n = 1 << job.log_n_rows
    arrays = []
    for a0, a1 in inputs:
        a0 = np.ascontiguousarray(a0, dtype=np.uint32)
        a1 = np.ascontiguousarray(a1, dtype=np.uint32)
        if a0.size != n or a1.size != n:
            raise ValueError(f"a0 and a1 need {n} values")
        arrays.append((a0, a1))
    k = len(arrays)
    a0p = (C.c_void_p * k)(*[a[0].ctypes.data for a in arrays])
    a1p = (C.c_void_p * k)(*[a[1].ctypes.data for a in arrays])
    outs = (C.POINTER(C.c_uint8) * k)()
    lens = (C.c_uint64 * k)()
    status = (C.c_int * k)()
    st = L.ProveStats()
    L.clear_error()
    L.check(L.lib().stwo_wide_fib_prove_batch(C.byref(job.c()), k, a0p, a1p, twiddles.twiddles.device_ptr,
                                              twiddles.itwiddles.device_ptr, len(twiddles.twiddles), outs, lens,
                                              status, C.byref(st), stream))
    proofs = []
    for i in range(k):
        if outs[i]:
            try:
                proofs.append(C.string_at(outs[i], lens[i]))
            finally:
                L.lib().stwo_free_proof(outs[i])
        else:
            proofs.append(None)
    return proofs, list(status), st.as_dict()


def kernel_launches():
    """Kernel launches the library has made in this process."""
    return int(L.lib().stwo_kernel_launches())


class ProofServer:
    """Continuous-batching proof server on the current device (csrc/server.cu):
    up to n_workers jobs in flight, admitted in arrival order while their device bound
    fits the budget, each on its own stream, sharing one twiddle tree."""

    def __init__(self, n_workers=8, device_budget_bytes=150 << 30, max_domain_log=22):
        L.clear_error()
        self._s = L.lib().stwo_server_create(n_workers, device_budget_bytes, max_domain_log)
        if not self._s:
            raise L.StwoError(f"server creation failed: {L.last_error()}")

    def submit(self, job_id, job, a0, a1):
        a0 = np.ascontiguousarray(a0, dtype=np.uint32)
        a1 = np.ascontiguousarray(a1, dtype=np.uint32)
        n = 1 << job.log_n_rows
        if a0.size != n or a1.size != n:
            raise ValueError(f"a0 and a1 need {n} values")
        L.clear_error()
        L.check(L.lib().stwo_server_submit(self._s, job_id, C.byref(job.c()), a0.ctypes.data, a1.ctypes.data))

    def submit_device(self, job_id, job, a0_dev, a1_dev):
        """Queues a job whose inputs are device pointers (ints); they must stay valid
        until the job's result has been polled."""
        L.clear_error()
        L.check(L.lib().stwo_server_submit_device(self._s, job_id, C.byref(job.c()), a0_dev, a1_dev))

    def cancel(self, job_id):
        """Removes a job that is still queued (its result reports STWO_ERR_CANCELLED);
        raises if the job is running, finished or unknown."""
        L.check(L.lib().stwo_server_cancel(self._s, job_id))

    def pause(self):
        """Workers start no queued job until resume() (running jobs finish)."""
        L.check(L.lib().stwo_server_pause(self._s, 1))

    def resume(self):
        L.check(L.lib().stwo_server_pause(self._s, 0))

    def set_queue_timeout(self, ms):
        """Queued jobs that wait longer than ms (0: no limit) are not started; their
        results report STWO_ERR_TIMEOUT."""
        L.check(L.lib().stwo_server_set_queue_timeout(self._s, float(ms)))

    def mark_epoch(self):
        """Sets the device epoch of device_done_ms (records and waits for an event on an
        idle stream of the server's): call it with nothing running, before a batch."""
        L.check(L.lib().stwo_server_mark_epoch(self._s))

    def poll(self, max_results=64, timeout_ms=-1):
        """Finished jobs as dicts: job_id, status, error, proof, submit/start/done ms (host
        clock), device_done_ms (device time of the job's last GPU operation after the
        last mark_epoch, or -1), stats."""
        buf = (L.ServerResult * max_results)()
        n = L.lib().stwo_server_poll(self._s, buf, max_results, timeout_ms)
        out = []
        for r in buf[:n]:
            proof = C.string_at(r.proof, r.proof_len) if r.proof else None
            if r.proof:
                L.lib().stwo_free_proof(r.proof)
            out.append({"job_id": r.job_id, "status": r.status, "error": r.error.decode(errors="replace"),
                        "proof": proof, "submit_ms": r.submit_ms, "start_ms": r.start_ms, "done_ms": r.done_ms,
                        "device_done_ms": r.device_done_ms, "stats": r.stats.as_dict()})
        return out

    def stats(self):
        p, r, b = C.c_uint32(), C.c_uint32(), C.c_uint64()
        L.lib().stwo_server_stats(self._s, C.byref(p), C.byref(r), C.byref(b))
        return {"pending": p.value, "running": r.value, "device_bytes_in_use": b.value}

    def graph_stats(self):
        """Proofs that reused a worker's retained slab, and those that replayed the
        proof's CUDA graph (same-shape jobs in a row on one worker)."""
        a, b = C.c_uint64(), C.c_uint64()
        L.lib().stwo_server_graph_stats(self._s, C.byref(a), C.byref(b))
        return {"slab_reuses": a.value, "graph_replays": b.value}

    def batch_stats(self):
        """Launch sequences that proved several queued jobs of one shape at once, and
        the jobs they proved."""
        a, b = C.c_uint64(), C.c_uint64()
        L.lib().stwo_server_batch_stats(self._s, C.byref(a), C.byref(b))
        return {"batches": a.value, "batched_jobs": b.value}

    @staticmethod
    def now_ms():
        return L.lib().stwo_server_now_ms()

    def close(self):
        if self._s:
            L.lib().stwo_server_destroy(self._s)
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
