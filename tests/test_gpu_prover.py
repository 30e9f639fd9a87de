"""The GPU prover (csrc/prover.cu) and proof server (csrc/server.cu): proof bytes
identical to the oracle prover's, proofs that verify, identical proofs alone and in a
concurrent mix."""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu

JOBS = [
    # (log_n_rows, n_columns, log_blowup, n_queries, pow_bits)
    (2, 3, 1, 1, 0),
    (3, 4, 1, 3, 5),
    (4, 8, 1, 3, 5),
    (5, 3, 1, 3, 0),
    (6, 16, 2, 5, 3),
    (3, 20, 3, 9, 2),
    (7, 33, 4, 20, 8),
    (9, 17, 1, 7, 11),
    (10, 20, 1, 3, 5),   # first FRI layer of log size 11: the fused tail starts at layer 1
    (10, 100, 2, 3, 5),
    (11, 64, 1, 30, 1),
    (12, 64, 1, 3, 5),   # 64 columns, 2^12 rows: the reference CpuBackend's single proof
    (14, 16, 1, 3, 10),
]


def job_of(t):
    stwo = load_package()
    return stwo.WideFibJob(*t)


@pytest.mark.parametrize("t", JOBS, ids=lambda j: "L%d_N%d_B%d_q%d_pow%d" % j)
def test_gpu_proof_equals_oracle_proof(oracle, t):
    stwo = load_package()
    a0, a1 = stwo.wide_fib_inputs(t[0], 2000 + t[0] * 7 + t[1])
    proof, stats = stwo.prove_wide_fib(job_of(t), a0, a1)
    want, rc = oracle.wide_fib_prove(t[0], t[1], a0, a1, t[2], t[3], t[4])
    assert rc == 0
    assert proof == want
    assert stats["proof_bytes"] == len(proof)
    assert stats["kernel_launches"] > 0
    assert 0 < stats["device_bytes"] <= job_of(t).device_bytes(own_twiddles=True)
    assert stats["total_ms"] >= stats["trace_ms"] > 0
    assert stwo.verify(proof, *t)


def test_gpu_proof_with_shared_twiddles_is_identical():
    stwo = load_package()
    t = (8, 12, 1, 3, 5)
    a0, a1 = stwo.wide_fib_inputs(8, 5)
    own, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
    tree = stwo.CudaBackend.precompute_twiddles(stwo.CanonicCoset(16).half_coset())
    shared, _ = stwo.prove_wide_fib(job_of(t), a0, a1, twiddles=tree)
    assert own == shared


def test_gpu_prover_accepts_device_inputs():
    stwo = load_package()
    t = (6, 9, 1, 3, 5)
    a0, a1 = stwo.wide_fib_inputs(6, 8)
    host, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
    d0, d1 = stwo.BaseFieldVec.from_numpy(a0), stwo.BaseFieldVec.from_numpy(a1)
    import ctypes as C
    L = stwo._lib
    out, ln, st = C.POINTER(C.c_uint8)(), C.c_uint64(), L.ProveStats()
    L.check(L.lib().stwo_wide_fib_prove(C.byref(job_of(t).c()), d0.device_ptr, d1.device_ptr, None, None, 0,
                                        C.byref(out), C.byref(ln), C.byref(st), None))
    dev = C.string_at(out, ln.value)
    L.lib().stwo_free_proof(out)
    assert dev == host


@pytest.mark.parametrize("bad", [(2, 2, 1, 3, 5), (1, 8, 1, 3, 5), (4, 8, 0, 3, 5), (4, 8, 5, 3, 5),
                                 (4, 8, 1, 0, 5), (4, 2000, 1, 3, 5), (26, 8, 1, 3, 5), (4, 8, 1, 3, 33)])
def test_gpu_prover_rejects_unsupported_jobs(bad):
    stwo = load_package()
    n = 1 << min(bad[0], 4)
    with pytest.raises((stwo._lib.StwoError, ValueError)):
        stwo.prove_wide_fib(job_of(bad), np.zeros(n, np.uint32), np.zeros(n, np.uint32))
    # the library stays usable
    a0, a1 = stwo.wide_fib_inputs(4, 1)
    proof, _ = stwo.prove_wide_fib(job_of((4, 8, 1, 3, 5)), a0, a1)
    assert stwo.verify(proof, 4, 8, 1, 3, 5)


LARGE_JOBS = [
    # serving-stream shapes above 2^14 rows (log_n_rows 12..20, 16..256 columns)
    (15, 64, 1, 3, 5),
    (16, 128, 1, 3, 5),
    (17, 32, 1, 3, 5),
    (19, 16, 1, 3, 5),
    # the reference's own end-to-end shape: 1024 columns, 2^16 rows
    # (examples/wide_fibonacci.rs:19-20, 211-249)
    (16, 1024, 1, 3, 5),
]


@pytest.mark.parametrize("t", LARGE_JOBS, ids=lambda j: "L%d_N%d_B%d_q%d_pow%d" % j)
def test_large_gpu_proof_equals_oracle_proof(oracle, t):
    """Proof bytes above 2^14 rows: the oracle prover runs on every host thread."""
    import os
    stwo = load_package()
    a0, a1 = stwo.wide_fib_inputs(t[0], 3000 + t[0] * 7 + t[1])
    proof, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
    oracle.set_threads(os.cpu_count() or 1)
    try:
        want, rc = oracle.wide_fib_prove(t[0], t[1], a0, a1, t[2], t[3], t[4])
    finally:
        oracle.set_threads(1)
    assert rc == 0
    assert proof == want
    assert stwo.verify(proof, *t)


def test_large_proof_verifies():
    """256 columns, 2^18 rows: checked by the verifier (the oracle is too slow here)."""
    stwo = load_package()
    t = (18, 256, 1, 3, 10)
    a0, a1 = stwo.wide_fib_inputs(18, 99)
    proof, stats = stwo.prove_wide_fib(job_of(t), a0, a1)
    assert stwo.verify(proof, *t)
    proof2, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
    assert proof2 == proof


def _mixed_jobs(n, seed):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        L = int(rng.integers(4, 13))
        N = int(rng.choice([3, 8, 16, 33, 64]))
        B = int(rng.choice([1, 1, 2]))
        jobs.append((i, (L, N, B, int(rng.integers(1, 8)), int(rng.integers(0, 9))), 500 + i))
    return jobs


@pytest.mark.parametrize("priorities", ["1", "0"])
def test_server_proofs_equal_single_job_proofs(priorities, monkeypatch):
    """Every proof of a concurrent mix equals the same job proved alone, with per-job
    stream priorities (the default) and without (STWO_SERVER_PRIORITY=0)."""
    monkeypatch.setenv("STWO_SERVER_PRIORITY", priorities)
    stwo = load_package()
    jobs = _mixed_jobs(24, 3)
    alone = {}
    for jid, t, seed in jobs:
        a0, a1 = stwo.wide_fib_inputs(t[0], seed)
        alone[jid] = stwo.prove_wide_fib(job_of(t), a0, a1)[0]
    with stwo.ProofServer(n_workers=8, device_budget_bytes=8 << 30, max_domain_log=16) as srv:
        for jid, t, seed in jobs:
            a0, a1 = stwo.wide_fib_inputs(t[0], seed)
            srv.submit(jid, job_of(t), a0, a1)
        got = {}
        while len(got) < len(jobs):
            for r in srv.poll(timeout_ms=-1):
                assert r["status"] == 0, r["error"]
                got[r["job_id"]] = r
        assert srv.stats()["running"] == 0
    for jid, t, _ in jobs:
        assert got[jid]["proof"] == alone[jid], (jid, t)
        r = got[jid]
        assert r["submit_ms"] <= r["start_ms"] <= r["done_ms"]


def test_server_device_completion_times():
    """Before any epoch mark a result carries device_done_ms = -1; after mark_epoch each
    finished job carries the device time of its last GPU operation, after the mark and
    no later than the host saw the job finish."""
    stwo = load_package()
    jobs = [(0, (9, 24, 1, 3, 5), 11), (1, (11, 16, 1, 3, 5), 12), (2, (10, 40, 1, 3, 5), 13)]
    with stwo.ProofServer(n_workers=2, device_budget_bytes=8 << 30, max_domain_log=16) as srv:
        a0, a1 = stwo.wide_fib_inputs(9, 10)
        srv.submit(99, job_of((9, 24, 1, 3, 5)), a0, a1)
        (r,) = srv.poll(timeout_ms=-1)
        assert r["status"] == 0 and r["device_done_ms"] == -1.0
        t0 = srv.now_ms()
        srv.mark_epoch()
        for jid, t, seed in jobs:
            a0, a1 = stwo.wide_fib_inputs(t[0], seed)
            srv.submit(jid, job_of(t), a0, a1)
        got = {}
        while len(got) < len(jobs):
            for r in srv.poll(timeout_ms=-1):
                assert r["status"] == 0, r["error"]
                got[r["job_id"]] = r
    for r in got.values():
        assert 0.0 < r["device_done_ms"] <= r["done_ms"] - t0 + 1.0, r


@pytest.mark.parametrize("graphs", ["1", "0"])
@pytest.mark.parametrize("workers", [1, 3])
def test_server_same_shape_runs_replay_equal_proofs(graphs, workers, monkeypatch):
    """Runs of same-shape jobs: a worker keeps its slab for the next job of the same
    shape, captures the proof's launch sequence as a CUDA graph on the second and
    replays it from the third. Every proof (each job with its own inputs) equals the
    same job proved alone; STWO_SERVER_GRAPHS=0 turns the reuse off. (Batching of
    queued same-shape jobs is off here: it would take these runs as batches.)"""
    monkeypatch.setenv("STWO_SERVER_GRAPHS", graphs)
    monkeypatch.setenv("STWO_SERVER_BATCH", "1")
    stwo = load_package()
    shapes = [(9, 24, 1, 3, 5), (11, 16, 2, 4, 3), (3, 5, 1, 2, 1), (2, 3, 1, 1, 0)]
    jobs = []
    for k in range(28):
        t = shapes[0] if k < 10 else shapes[1] if k < 19 else shapes[2] if k < 25 else shapes[3]
        jobs.append((k, t, 700 + k))
    alone = {}
    for jid, t, seed in jobs:
        a0, a1 = stwo.wide_fib_inputs(t[0], seed)
        alone[jid] = stwo.prove_wide_fib(job_of(t), a0, a1)[0]
    with stwo.ProofServer(n_workers=workers, device_budget_bytes=8 << 30, max_domain_log=16) as srv:
        for jid, t, seed in jobs:
            a0, a1 = stwo.wide_fib_inputs(t[0], seed)
            srv.submit(jid, job_of(t), a0, a1)
        got = {}
        while len(got) < len(jobs):
            for r in srv.poll(timeout_ms=-1):
                assert r["status"] == 0, r["error"]
                got[r["job_id"]] = r
        assert srv.stats()["running"] == 0 and srv.stats()["device_bytes_in_use"] == 0
        gs = srv.graph_stats()
    for jid, t, _ in jobs:
        assert got[jid]["proof"] == alone[jid], (jid, t)
        assert got[jid]["stats"]["kernel_launches"] > 0
    if graphs == "0":
        assert gs == {"slab_reuses": 0, "graph_replays": 0}
    elif workers == 1:
        # runs of 10, 9 and 6 jobs of cacheable shapes (log_n_rows >= 3): every job but a
        # run's first reuses the slab; every job but a run's first two replays the graph
        assert gs == {"slab_reuses": 9 + 8 + 5, "graph_replays": 8 + 7 + 4}
    else:
        assert gs["slab_reuses"] > 0 and gs["graph_replays"] > 0


@pytest.mark.parametrize("stream_kind", ["own", "default"])
def test_cached_proofs_replay_and_equal_plain_proofs(stream_kind):
    """stwo_wide_fib_prove_cached: the first proof of a shape keeps its memory, the
    second captures the launch sequence as a CUDA graph, later ones replay it; a new
    shape replaces the cached one. On the legacy default stream the memory is reused
    but nothing is captured. Every proof equals the plain call's."""
    import torch
    stwo = load_package()
    s = torch.cuda.Stream() if stream_kind == "own" else None
    sptr = s.cuda_stream if s is not None else None
    tree = stwo.CudaBackend.precompute_twiddles(stwo.CanonicCoset(16).half_coset())
    seq = [(10, 24, 1, 3, 5)] * 4 + [(12, 16, 2, 4, 2)] * 3 + [(2, 3, 1, 1, 0)] * 2 + [(10, 24, 1, 3, 5)] * 2
    with stwo.ProveCache() as cache:
        replays = []
        for k, t in enumerate(seq):
            a0, a1 = stwo.wide_fib_inputs(t[0], 3000 + k)
            want, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
            got, st = stwo.prove_wide_fib(job_of(t), a0, a1, twiddles=tree, stream=sptr, cache=cache)
            assert got == want, (k, t)
            assert st["trace_ms"] > 0 and st["kernel_launches"] > 0
            replays.append(cache.stats()["graph_replays"])
        # replays from the third proof of a run on; log_n_rows 2 is not cached
        if stream_kind == "own":
            assert replays == [0, 0, 1, 2, 2, 2, 3, 3, 3, 3, 3]
        else:
            assert replays == [0] * len(seq)
        assert cache.stats()["device_bytes"] == job_of(seq[-1]).device_bytes(own_twiddles=False)
        cache.close(sptr)
    with pytest.raises(stwo._lib.StwoError):  # the cache needs the caller's tree
        with stwo.ProveCache() as c2:
            a0, a1 = stwo.wide_fib_inputs(10, 1)
            stwo.prove_wide_fib(job_of(seq[0]), a0, a1, cache=c2)


def test_cached_proofs_recapture_after_a_tunable_changes():
    """Changing a tunable between cached proofs of one shape retires the captured
    sequence (the eval_at_point chunking changes its descriptors and grid): the next
    proof runs afresh, the one after captures again, and every proof equals the plain
    call's."""
    import torch
    stwo = load_package()
    lib = stwo._lib.lib()
    s = torch.cuda.Stream()
    tree = stwo.CudaBackend.precompute_twiddles(stwo.CanonicCoset(16).half_coset())
    t = (13, 300, 1, 3, 5)  # 300 polynomials: the per-launch choice is 4 groups a CTA
    plan = [None, None, None, 2, None, None, 0, None]  # a tunable set at proofs 3 and 6
    try:
        with stwo.ProveCache() as cache:
            replays = []
            for k, g in enumerate(plan):
                if g is not None:
                    stwo._lib.check(lib.stwo_set_tunable(b"eval_at_point_groups_log", g))
                a0, a1 = stwo.wide_fib_inputs(t[0], 4000 + k)
                want, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
                got, _ = stwo.prove_wide_fib(job_of(t), a0, a1, twiddles=tree, stream=s.cuda_stream, cache=cache)
                assert got == want, (k, g)
                replays.append(cache.stats()["graph_replays"])
            assert replays == [0, 0, 1, 1, 1, 2, 2, 2]
            cache.close(s.cuda_stream)
    finally:
        lib.stwo_set_tunable(b"eval_at_point_groups_log", 0)


def test_server_respects_the_memory_budget():
    stwo = load_package()
    t = (10, 32, 1, 3, 5)
    need = job_of(t).device_bytes(own_twiddles=False)
    with stwo.ProofServer(n_workers=4, device_budget_bytes=need + need // 2, max_domain_log=12) as srv:
        for i in range(6):
            a0, a1 = stwo.wide_fib_inputs(10, i)
            srv.submit(i, job_of(t), a0, a1)
        results = []
        while len(results) < 6:
            st = srv.stats()
            assert st["device_bytes_in_use"] <= need + need // 2
            assert st["running"] <= 1
            results += srv.poll(timeout_ms=5)
        # one job at a time fits: their runs do not overlap
        spans = sorted((r["start_ms"], r["done_ms"]) for r in results)
        for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
            assert s1 >= e0 - 1e-6
        with pytest.raises(stwo._lib.StwoError):
            big = (11, 64, 1, 3, 5)
            a0, a1 = stwo.wide_fib_inputs(11, 0)
            srv.submit(99, job_of(big), a0, a1)


def test_concurrent_prove_calls_on_separate_streams_match():
    """prove_wide_fib from several host threads, each on its own stream, gives each
    job the same bytes as proving it alone."""
    import threading
    import torch
    stwo = load_package()
    jobs = [(7 + i % 5, 8 + 3 * i, 1 + (i % 2), 3, i % 6) for i in range(8)]
    alone = []
    for i, t in enumerate(jobs):
        a0, a1 = stwo.wide_fib_inputs(t[0], 300 + i)
        alone.append(stwo.prove_wide_fib(job_of(t), a0, a1)[0])
    got = [None] * len(jobs)

    def run(i):
        torch.cuda.set_device(0)
        s = torch.cuda.Stream()
        a0, a1 = stwo.wide_fib_inputs(jobs[i][0], 300 + i)
        for _ in range(2):
            got[i] = stwo.prove_wide_fib(job_of(jobs[i]), a0, a1, stream=s.cuda_stream)[0]

    th = [threading.Thread(target=run, args=(i,)) for i in range(len(jobs))]
    for x in th:
        x.start()
    for x in th:
        x.join()
    assert got == alone


def test_server_shutdown_with_queued_jobs_is_clean():
    stwo = load_package()
    srv = stwo.ProofServer(n_workers=2, device_budget_bytes=4 << 30, max_domain_log=16)
    for i in range(12):
        a0, a1 = stwo.wide_fib_inputs(12, i)
        srv.submit(i, job_of((12, 32, 1, 3, 5)), a0, a1)
    srv.close()  # drops queued jobs, waits for running ones
    # the library stays usable
    a0, a1 = stwo.wide_fib_inputs(5, 2)
    proof, _ = stwo.prove_wide_fib(job_of((5, 6, 1, 3, 5)), a0, a1)
    assert stwo.verify(proof, 5, 6, 1, 3, 5)


def test_tunables_change_speed_not_results():
    """Every FFT elements-per-thread, Merkle layers-per-launch, Merkle nodes-per-thread
    and eval_at_point chunk setting gives the same proof bytes; stwo_autotune reports
    its choices as JSON."""
    import ctypes as C
    import json
    stwo = load_package()
    lib = stwo._lib.lib()
    t = (16, 40, 2, 3, 5)
    a0, a1 = stwo.wide_fib_inputs(16, 77)
    base, _ = stwo.prove_wide_fib(job_of(t), a0, a1)
    # trees of 2^20 and 2^21 leaves, large enough for several nodes per thread
    tb = (19, 24, 1, 3, 5)
    b0, b1 = stwo.wide_fib_inputs(19, 78)
    base_b, _ = stwo.prove_wide_fib(job_of(tb), b0, b1)
    settings = [("fft_ept_contig_small", 5), ("fft_ept_contig_large", 5), ("fft_ept_strided", 5),
                ("merkle_sub_threads", 128), ("merkle_sub_threads", 512), ("merkle_sub_spread", 0),
                ("merkle_sub_spread", 5), ("eval_at_point_groups_log", 2), ("eval_at_point_groups_log", 3),
                ("eval_at_point_groups_log", 4), ("fft_max_strided_layers", 4), ("fft_max_strided_layers", 7)]
    try:
        for name, value in settings:
            stwo._lib.check(lib.stwo_set_tunable(name.encode(), value))
            assert stwo.prove_wide_fib(job_of(t), a0, a1)[0] == base, (name, value)
            assert stwo.prove_wide_fib(job_of(tb), b0, b1)[0] == base_b, (name, value)
        with pytest.raises(stwo._lib.StwoError):
            stwo._lib.check(lib.stwo_set_tunable(b"merkle_sub_threads", 100))
        with pytest.raises(stwo._lib.StwoError):
            stwo._lib.check(lib.stwo_set_tunable(b"merkle_sub_spread", 6))
        with pytest.raises(stwo._lib.StwoError):
            stwo._lib.check(lib.stwo_set_tunable(b"fft_max_strided_layers", 11))
        buf = C.create_string_buffer(4096)
        stwo._lib.check(lib.stwo_autotune(buf, 4096))
        rep = json.loads(buf.value.decode())
        assert set(rep) == {"fft_ept_contig_small", "fft_ept_contig_large", "fft_ept_strided", "fft_max_strided_layers",
                            "merkle_sub_threads", "merkle_sub_spread"}
        assert stwo.prove_wide_fib(job_of(t), a0, a1)[0] == base
        assert stwo.prove_wide_fib(job_of(tb), b0, b1)[0] == base_b
    finally:
        for name, value in [("fft_ept_contig_small", 6), ("fft_ept_contig_large", 6), ("fft_ept_strided", 6),
                            ("merkle_sub_threads", 256), ("merkle_sub_spread", 3), ("eval_at_point_groups_log", 0),
                            ("fft_max_strided_layers", 10)]:
            lib.stwo_set_tunable(name.encode(), value)


def _collect(srv, n):
    got = {}
    while len(got) < n:
        for r in srv.poll(timeout_ms=-1):
            got[r["job_id"]] = r
    return got


def _wait_running(srv):
    import time
    t0 = time.time()
    while srv.stats()["running"] == 0:
        assert time.time() - t0 < 30, "the first job never started"
        time.sleep(0.0005)


BUSY_JOB = (19, 256, 1, 3, 5)  # keeps a single worker busy for several milliseconds


def _small_jobs(n):
    return [(8 + (i % 3), 16, 1, 3, 5) for i in range(n)]


def test_server_cancels_queued_jobs_only():
    """A queued job leaves the queue with STWO_ERR_CANCELLED and never runs; the running
    job and unknown ids cannot be cancelled; every other job proves exactly as alone."""
    stwo = load_package()
    L = stwo._lib
    small = _small_jobs(3)
    alone = [stwo.prove_wide_fib(job_of(t), *stwo.wide_fib_inputs(t[0], 50 + i))[0] for i, t in enumerate(small)]
    with stwo.ProofServer(n_workers=1, device_budget_bytes=16 << 30, max_domain_log=21) as srv:
        srv.submit(0, job_of(BUSY_JOB), *stwo.wide_fib_inputs(BUSY_JOB[0], 5))
        _wait_running(srv)
        for i, t in enumerate(small):
            srv.submit(1 + i, job_of(t), *stwo.wide_fib_inputs(t[0], 50 + i))
        srv.cancel(2)
        with pytest.raises(L.StwoError):
            srv.cancel(2)  # no longer queued
        with pytest.raises(L.StwoError):
            srv.cancel(99)  # unknown
        got = _collect(srv, 4)
        assert srv.stats() == {"pending": 0, "running": 0, "device_bytes_in_use": 0}
    assert got[0]["status"] == L.OK
    assert got[2]["status"] == L.ERR_CANCELLED and got[2]["proof"] is None
    assert got[1]["status"] == got[3]["status"] == L.OK
    assert got[1]["proof"] == alone[0] and got[3]["proof"] == alone[2]


def test_server_queue_timeout():
    """Jobs that wait in the queue past the server's queue timeout end with
    STWO_ERR_TIMEOUT without running (reported while the worker is still busy); with
    the limit lifted, jobs run again."""
    stwo = load_package()
    L = stwo._lib
    small = _small_jobs(3)
    with stwo.ProofServer(n_workers=1, device_budget_bytes=16 << 30, max_domain_log=21) as srv:
        srv.submit(0, job_of(BUSY_JOB), *stwo.wide_fib_inputs(BUSY_JOB[0], 6))
        _wait_running(srv)
        srv.set_queue_timeout(0.2)
        for i, t in enumerate(small):
            srv.submit(1 + i, job_of(t), *stwo.wide_fib_inputs(t[0], 60 + i))
        got = _collect(srv, 4)
        assert got[0]["status"] == L.OK and stwo.verify(got[0]["proof"], *BUSY_JOB)
        for k in (1, 2, 3):
            assert got[k]["status"] == L.ERR_TIMEOUT and got[k]["proof"] is None
        srv.set_queue_timeout(0)
        t = small[0]
        srv.submit(7, job_of(t), *stwo.wide_fib_inputs(t[0], 70))
        r = _collect(srv, 1)[7]
        assert r["status"] == L.OK and stwo.verify(r["proof"], *t)
        assert srv.stats()["device_bytes_in_use"] == 0


def test_server_job_survives_injected_allocation_failure():
    """An allocation failure of one job (injected on the host: the pool call fails as if
    the device were full) fails that job alone with STWO_ERR_OUT_OF_MEMORY; its budget
    returns and the following jobs prove exactly as alone."""
    stwo = load_package()
    L = stwo._lib
    jobs = [(9, 16, 1, 3, 5), (10, 32, 1, 3, 5), (9, 20, 2, 4, 3)]
    alone = [stwo.prove_wide_fib(job_of(t), *stwo.wide_fib_inputs(t[0], 80 + i))[0] for i, t in enumerate(jobs)]
    with stwo.ProofServer(n_workers=1, device_budget_bytes=8 << 30, max_domain_log=16) as srv:
        L.lib().stwo_debug_fail_allocations(1)
        try:
            for i, t in enumerate(jobs):
                srv.submit(i, job_of(t), *stwo.wide_fib_inputs(t[0], 80 + i))
            got = _collect(srv, len(jobs))
        finally:
            L.lib().stwo_debug_fail_allocations(0)
        assert srv.stats() == {"pending": 0, "running": 0, "device_bytes_in_use": 0}
    failed = [k for k, r in got.items() if r["status"] != L.OK]
    assert failed == [0] and got[0]["status"] == L.ERR_OUT_OF_MEMORY and "injected" in got[0]["error"]
    assert got[1]["proof"] == alone[1] and got[2]["proof"] == alone[2]


def test_server_submit_checks_before_copying_inputs():
    """A job whose domain exceeds the server's twiddle tree is refused at submission,
    before its inputs are read: the input arrays may be shorter than 2^log_n_rows."""
    import numpy as np
    stwo = load_package()
    L = stwo._lib
    with stwo.ProofServer(n_workers=1, device_budget_bytes=1 << 30, max_domain_log=12) as srv:
        tiny = np.zeros(4, np.uint32)
        L.clear_error()
        rc = L.lib().stwo_server_submit(srv._s, 1, stwo.WideFibJob(28, 16).c(), tiny.ctypes.data, tiny.ctypes.data)
        assert rc == L.ERR_UNSUPPORTED_SIZE and "exceeds" in L.last_error()
        L.clear_error()


@pytest.mark.parametrize("shape,k", [((4, 8, 1, 3, 5), 3), ((10, 100, 2, 3, 5), 2), ((12, 64, 1, 3, 5), 8),
                                     ((13, 70, 1, 5, 5), 5), ((16, 16, 1, 3, 5), 2)],
                         ids=lambda v: str(v))
def test_batch_of_one_shape_in_one_launch_sequence(stwo, shape, k):
    """stwo_wide_fib_prove_batch proves k jobs of one shape with every kernel of the proof
    launched once for all of them (their device memory laid out alike, job k's at job
    0's plus k slabs): each proof equals the one-job prover's byte for byte, and the
    sequence launches about as many kernels as one proof (the transforms of more than
    64 columns stage their table; nothing scales with k)."""
    L, N, B, q, pw = shape
    job = stwo.WideFibJob(L, N, B, q, pw)
    tree = stwo.CudaBackend.precompute_twiddles(stwo.CanonicCoset(L + 1 + B).half_coset())
    inputs = [stwo.wide_fib_inputs(L, 900 + 17 * i + L) for i in range(k)]
    n0 = stwo.kernel_launches()
    single = [stwo.prove_wide_fib(job, a0, a1, twiddles=tree)[0] for a0, a1 in inputs]
    one = (stwo.kernel_launches() - n0) // k
    n0 = stwo.kernel_launches()
    proofs, status, stats = stwo.prove_wide_fib_batch(job, inputs, tree)
    batched = stwo.kernel_launches() - n0
    assert status == [0] * k
    for i in range(k):
        assert proofs[i] == single[i], f"job {i}"
    assert batched <= one + 4, (batched, one)
    stwo.verify(proofs[-1], L, N, log_blowup=B, n_queries=q, pow_bits=pw)


def test_server_pause_holds_the_queue():
    """While paused, the server accepts jobs but starts none; resumed, its one worker
    takes the first and the 9 queued jobs of its shape behind it as one batch (exactly
    one launch sequence of 10), every proof equal to the job's proof alone."""
    stwo = load_package()
    L = stwo._lib
    sh = (12, 64, 1, 3, 5)
    seeds = [1700 + i for i in range(10)]
    alone = [stwo.prove_wide_fib(job_of(sh), *stwo.wide_fib_inputs(sh[0], sd))[0] for sd in seeds]
    with stwo.ProofServer(n_workers=1, device_budget_bytes=16 << 30, max_domain_log=21) as srv:
        srv.pause()
        for i, sd in enumerate(seeds):
            srv.submit(i, job_of(sh), *stwo.wide_fib_inputs(sh[0], sd))
        import time
        time.sleep(0.2)
        assert srv.stats()["pending"] == 10 and srv.stats()["running"] == 0
        assert srv.poll(timeout_ms=0) == []
        srv.resume()
        got = _collect(srv, 10)
        assert srv.batch_stats() == {"batches": 1, "batched_jobs": 10}
    for i in range(10):
        assert got[i]["status"] == L.OK, got[i]["error"]
        assert got[i]["proof"] == alone[i], i


@pytest.mark.parametrize("batch", ["32", "5"])
def test_server_batches_queued_jobs_of_one_shape(batch, monkeypatch):
    """A worker that takes a small job also takes the queued jobs of its shape that
    arrival-order admission would take next (up to STWO_SERVER_BATCH) and proves them in
    one launch sequence. A larger job keeps the one worker busy while 40 jobs of one
    shape and then 3 of another queue behind it: they come back in batches, every proof
    equal to the job's proof alone, the other shape's jobs after them."""
    monkeypatch.setenv("STWO_SERVER_BATCH", batch)
    stwo = load_package()
    L = stwo._lib
    t, u = (12, 64, 1, 3, 5), (11, 16, 1, 3, 5)
    jobs = [(1 + i, t, 900 + i) for i in range(40)] + [(41 + i, u, 990 + i) for i in range(3)]
    alone = {jid: stwo.prove_wide_fib(job_of(sh), *stwo.wide_fib_inputs(sh[0], seed))[0] for jid, sh, seed in jobs}
    with stwo.ProofServer(n_workers=1, device_budget_bytes=16 << 30, max_domain_log=21) as srv:
        srv.submit(0, job_of(BUSY_JOB), *stwo.wide_fib_inputs(BUSY_JOB[0], 9))
        _wait_running(srv)
        for jid, sh, seed in jobs:
            srv.submit(jid, job_of(sh), *stwo.wide_fib_inputs(sh[0], seed))
        got = _collect(srv, len(jobs) + 1)
        bs = srv.batch_stats()
        assert srv.stats() == {"pending": 0, "running": 0, "device_bytes_in_use": 0}
    for jid, sh, _ in jobs:
        assert got[jid]["status"] == L.OK, got[jid]["error"]
        assert got[jid]["proof"] == alone[jid], jid
    k = int(batch)
    assert bs["batches"] >= 40 // k and bs["batched_jobs"] >= 40 - 1
    assert max(got[jid]["start_ms"] for jid in range(1, 41)) <= min(got[jid]["start_ms"] for jid in (41, 42, 43))
