"""Benchmark: wide-Fibonacci proof serving on one B200 (the headline metric:
"bit-exact proofs/s & p99 latency: batched server vs per-job; FFT % HBM peak").

Workload: a seeded stream of wide-Fibonacci proof jobs shaped like the serving
config: log_n_rows uniform in {12..20} (log-uniform row counts), columns uniform in
{16..256}, log_blowup 1, 3 queries, pow_bits 5, Blake2s channel. A step is one batch
of --jobs jobs (default 48) admitted at once to the proof server (csrc/server.cu:
--workers jobs in flight, 150 GB device budget). `value` is the server's proofs/s
with the job inputs already resident in HBM; `e2e` submits host inputs instead.
Alongside: the same jobs proved one at a time (per_job), every batched proof
compared byte for byte with its one-at-a-time proof, Poisson-arrival latency
(p50/p99/p99.9) at three loads for both modes, the single proofs of the 64-column x
2^12 and 256-column x 2^20 cases with their phase breakdown, the M31 circle FFT
roofline (8 columns at log 24, blowup 4; roofline.frac = FFT % HBM peak) and the
per-kernel sweep against the reference's own CUDA library.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the oracle port of the reference's CPU prover (CpuBackend
restated in C, oracle/stwo_oracle_prover.c) on the same job stream on all host
cores, a bounded sample per step. Prints one JSON line (rank 0).
"""
import argparse
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
P = (1 << 31) - 1
METRIC = "bit-exact proofs/s & p99 latency: batched server vs per-job; FFT % HBM peak"
UNIT = "proofs/s"
FFT_UNIT = "columns/s"
BUDGET = 150 << 30  # device-memory budget of the serving config


def load_package():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import stwo_gpu_b200
    return stwo_gpu_b200


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    return O


def load_simd():
    """The SIMD CPU baseline (oracle/simd.py: the oracle prover on vectorised, threaded
    functions; a stand-in for stwo's SimdBackend with the same proof bytes)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import simd as S
    S.lib()
    return S


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        for line in self._proc.stdout:
            if self._stop.is_set():
                break
            fields = [x.strip() for x in line.strip().split(",")]
            if len(fields) >= 9:
                self.samples.append(fields)

    def __enter__(self):
        # One nvidia-smi process printing a line every 100 ms for the whole region.
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                           "--format=csv,noheader,nounits", "-lms", "100"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._proc = None
        if self._proc is not None:
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except Exception:
                self._proc.kill()
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        smax = max(float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i] == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(self.samples)}


def cpu_baseline(O, log_size, log_blowup, threads):
    """The oracle (CpuBackend restated in C) on one column: interpolate + evaluate."""
    import numpy as np
    O.set_threads(threads)
    r = np.random.default_rng(1)
    N = log_size + log_blowup
    hc_big = O.canonic_half_coset(N)
    tw, itw = O.precompute_twiddles(hc_big)
    vals = r.integers(0, P, 1 << log_size, dtype=np.uint64).astype(np.uint32)
    hc = O.canonic_half_coset(log_size)
    t0 = time.perf_counter()
    coeffs = O.interpolate(hc, vals, itw)
    O.evaluate(hc_big, coeffs, tw)
    dt = time.perf_counter() - t0
    O.set_threads(1)
    return dt


def reference_gpu_timing(args, evals, lg, lb, ncols, tw, itw, tree_size):
    """The reference's own CUDA library (oracle/_ref, built unmodified from its sources)
    on the same step through its own API path: interpolate_columns, then, as
    PolyOps::evaluate_polynomials does (poly.rs:128-168), extend every polynomial into
    a fresh zeroed buffer and evaluate_columns. Reported beside our numbers."""
    import ctypes as C
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import reflib
    except ImportError:
        return None
    if not reflib.available():
        return None
    R = reflib.lib()
    N = lg + lb
    ptrs = (C.c_void_p * ncols)(*[t.data_ptr() for t in evals])

    def step():
        R.interpolate_columns(1 << (lg - 1), ptrs, itw.data_ptr(), tree_size, ncols, 1 << lg)
        ext = []
        for t in evals:
            d = R.cuda_alloc_zeroes_uint32_t(1 << N)
            R.copy_uint32_t_vec_from_device_to_device(t.data_ptr(), d, 1 << lg)
            ext.append(d)
        eptr = (C.c_void_p * ncols)(*ext)
        sizes = (C.c_int * ncols)(*([1 << N] * ncols))
        dom = (C.c_int * ncols)(*([1 << (N - 1)] * ncols))
        R.evaluate_columns(dom, eptr, tw.data_ptr(), tree_size, ncols, sizes)
        for d in ext:
            R.cuda_free_memory(d)

    # Equality first, on fresh copies of the step's inputs: our interpolate_columns +
    # extend_evaluate_columns against the reference library's path above.
    stwo = load_package()
    L, lib = stwo._lib, stwo._lib.lib()
    ours = [t.clone() for t in evals]
    theirs = [t.clone() for t in evals]
    ours_ext = [torch.empty(1 << N, dtype=torch.int32, device=t.device) for t in evals]
    theirs_ext = [torch.zeros(1 << N, dtype=torch.int32, device=t.device) for t in evals]
    logs = L.u32_array([lg] * ncols)
    torch.cuda.synchronize()
    L.check(lib.stwo_interpolate_columns(L.ptr_array([t.data_ptr() for t in ours]), logs, ncols, itw.data_ptr(),
                                         tree_size, None))
    L.check(lib.stwo_extend_evaluate_columns(L.ptr_array([t.data_ptr() for t in ours]), logs,
                                             L.ptr_array([t.data_ptr() for t in ours_ext]), lb, ncols, tw.data_ptr(),
                                             tree_size, None))
    L.check(lib.stwo_stream_synchronize(None))
    R.interpolate_columns(1 << (lg - 1), (C.c_void_p * ncols)(*[t.data_ptr() for t in theirs]), itw.data_ptr(),
                          tree_size, ncols, 1 << lg)
    for t, x in zip(theirs, theirs_ext):
        R.copy_uint32_t_vec_from_device_to_device(t.data_ptr(), x.data_ptr(), 1 << lg)
    R.evaluate_columns((C.c_int * ncols)(*([1 << (N - 1)] * ncols)),
                       (C.c_void_p * ncols)(*[x.data_ptr() for x in theirs_ext]), tw.data_ptr(), tree_size, ncols,
                       (C.c_int * ncols)(*([1 << N] * ncols)))
    torch.cuda.synchronize()
    equal_interp = all(torch.equal(a, b) for a, b in zip(ours, theirs))
    equal_eval = all(torch.equal(a, b) for a, b in zip(ours_ext, theirs_ext))
    del ours, theirs, ours_ext, theirs_ext
    torch.cuda.empty_cache()

    torch.cuda.synchronize()
    step()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    s.record(torch.cuda.default_stream())
    for _ in range(reps):
        step()
    e.record(torch.cuda.default_stream())
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    return {"ms_per_step": ms, "value": ncols / (ms / 1e3), "unit": FFT_UNIT,
            "equal": equal_interp and equal_eval, "equal_interpolate": equal_interp, "equal_evaluate": equal_eval,
            "what": "reference CUDA library (oracle/_ref) on this GPU: interpolate_columns + extend + "
                    "evaluate_columns, same 8 x 2^24 step; outputs compared element for element with ours"}


def replica_throughput(local_ms, units_per_rank, world, device=None):
    """Whole-job throughput of `world` independent replicas (no data-path collective):
    the step time is the maximum over ranks, and every rank processed
    `units_per_rank` units. Returns (max_ms, units per second)."""
    if world > 1:
        import torch
        t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        local_ms = float(t.item())
    return local_ms, world * units_per_rank / (local_ms / 1e3)


def kernel_suite(stwo, reps=5):
    """Config-1 per-kernel sweep (seeded uniform data) on cuda:0, ours and the reference
    CUDA library (oracle/_ref) on the same device inputs. Times are CUDA-event means over
    `reps` runs after one warm-up; algorithmic bytes are defined per kernel below."""
    import ctypes as C
    import torch
    L = stwo._lib
    lib = L.lib()
    dev = torch.device("cuda", 0)
    peak, _ = measured_peaks()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    R = None
    try:
        import reflib
        if reflib.available():
            R = reflib.lib()
    except ImportError:
        pass
    gen = torch.Generator(device=dev)
    gen.manual_seed(99)

    def rand(n, nonzero=False):
        lo = 1 if nonzero else 0
        return torch.randint(lo, P, (n,), dtype=torch.int64, device=dev, generator=gen).to(torch.int32)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(torch.cuda.current_stream())
        for _ in range(reps):
            fn()
        e.record(torch.cuda.current_stream())
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    def ptrs(ts):
        return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])

    out = {}
    sptr = torch.cuda.current_stream(dev).cuda_stream

    # (b) Blake2s Merkle tree over 64 columns of 2^22 (leaf = 64 words): leaf layer + 22 node layers.
    lg, nc = 22, 64
    cols = [rand(1 << lg) for _ in range(nc)]
    layers = [torch.empty((1 << l) * 8, dtype=torch.int32, device=dev) for l in range(lg + 1)]
    cptr = ptrs(cols)

    def merkle_ours():
        L.check(lib.stwo_merkle_commit_layer(lg, None, cptr, nc, layers[lg].data_ptr(), sptr))
        for l in range(lg - 1, -1, -1):
            L.check(lib.stwo_merkle_commit_layer(l, layers[l + 1].data_ptr(), None, 0, layers[l].data_ptr(), sptr))

    t = timed(merkle_ours)
    nodes = (1 << (lg + 1)) - 1
    b = nc * (1 << lg) * 4 + nodes * 32 + ((1 << lg) - 1) * 64
    comp = (1 << lg) * (nc // 16) + ((1 << lg) - 1)
    # The compression's own ALU-pipe bound: the xors and rotations of its 80 G functions
    # (640 instructions) at 64 ALU lanes per SM per clock, at the maximum SM clock.
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    alu_bound = sms * 64 * 1965e6 / 640
    rec = {"ms": t, "gbs": b / t / 1e6, "frac_hbm": b / t / 1e6 / peak, "compressions_per_s": comp / (t / 1e3),
           "alu_bound_compressions_per_s": alu_bound, "frac_alu_bound": comp / (t / 1e3) / alu_bound,
           "alu_bound_basis": f"{sms} SMs x 64 ALU lanes x 1965 MHz / 640 ALU instructions per compression",
           "workload": "64 cols x 2^22, full tree",
           "path": "stwo_merkle_commit_layer per layer (the reference's commit_on_layer calls)"}
    # The same tree through stwo_merkle_commit_tree, the prover's path: one launch.
    layers_t = [torch.empty((1 << l) * 8, dtype=torch.int32, device=dev) for l in range(lg + 1)]
    tlogs, tlay = L.u32_array([lg] * nc), L.ptr_array([x.data_ptr() for x in layers_t])

    def merkle_tree():
        L.check(lib.stwo_merkle_commit_tree(cptr, tlogs, nc, lg, tlay, sptr))

    n0 = lib.stwo_kernel_launches()
    merkle_tree()
    tree_launches = lib.stwo_kernel_launches() - n0
    tt = timed(merkle_tree)
    rec["tree_one_call"] = {"ms": tt, "compressions_per_s": comp / (tt / 1e3),
                            "frac_alu_bound": comp / (tt / 1e3) / alu_bound, "kernel_launches": tree_launches,
                            "equal": all(bool(torch.equal(x, y)) for x, y in zip(layers_t, layers))}
    rec["tree_frac_alu_bound"] = rec["tree_one_call"]["frac_alu_bound"]
    del layers_t
    if R is not None:
        dcols = R.copy_device_pointer_vec_from_host_to_device(cptr, nc)
        rl = [torch.empty((1 << l) * 8, dtype=torch.int32, device=dev) for l in range(lg + 1)]

        def merkle_ref():
            R.commit_on_first_layer(1 << lg, nc, dcols, rl[lg].data_ptr())
            for l in range(lg - 1, -1, -1):
                R.commit_on_layer_with_previous(1 << l, 0, dcols, rl[l + 1].data_ptr(), rl[l].data_ptr())

        rec["reference_ms"] = timed(merkle_ref)
        rec["root_equal"] = bool(torch.equal(rl[0], layers[0]))
        R.cuda_free_memory(dcols)
    out["merkle"] = rec
    del cols, layers

    # (c) batch inverse of 2^24 nonzero QM31 (AoS).
    n = 1 << 24
    src = rand(4 * n, nonzero=True)
    dst = torch.empty_like(src)
    t = timed(lambda: L.check(lib.stwo_batch_inverse_qm31(src.data_ptr(), dst.data_ptr(), n, sptr)))
    rec = {"ms": t, "gbs": n * 32 / t / 1e6, "frac_hbm": n * 32 / t / 1e6 / peak, "workload": "2^24 QM31"}
    if R is not None:
        rdst = torch.empty_like(src)
        rec["reference_ms"] = timed(lambda: R.batch_inverse_secure_field(src.data_ptr(), rdst.data_ptr(), n))
        rec["equal"] = bool(torch.equal(rdst, dst))
    out["batch_inverse_qm31"] = rec
    del src, dst

    # (d) FRI: fold_circle_into_line 2^24 -> 2^23, then fold_line down to 2^4.
    lg = 24
    hc = stwo.CanonicCoset(lg).half_coset()  # circle domain 2^24; line domain = its half coset
    tree = torch.empty(1 << hc.log_size, dtype=torch.int32, device=dev)
    itree = torch.empty_like(tree)
    L.check(lib.stwo_precompute_twiddles(hc.initial_index, hc.step_size, hc.log_size, tree.data_ptr(),
                                         itree.data_ptr(), sptr))
    src = [rand(1 << lg) for _ in range(4)]
    bufs = [[torch.empty(1 << l, dtype=torch.int32, device=dev) for _ in range(4)] for l in range(lg)]
    alpha = L.QM31(12345, 678, 91011, 1213)
    tsz = 1 << hc.log_size

    def fri_ours():
        L.check(lib.stwo_fold_circle_into_line(ptrs(src), 1 << lg, alpha, itree.data_ptr(), 0, ptrs(bufs[lg - 1]),
                                               sptr))
        for l in range(lg - 1, 4, -1):
            L.check(lib.stwo_fold_line(ptrs(bufs[l]), 1 << l, alpha, itree.data_ptr(), tsz - (1 << l),
                                       ptrs(bufs[l - 1]), sptr))

    t = timed(fri_ours)
    b = (1 << (lg - 1)) * 68 + sum((1 << (l - 1)) * 52 for l in range(lg - 1, 4, -1))
    rec = {"ms": t, "gbs": b / t / 1e6, "frac_hbm": b / t / 1e6 / peak, "workload": "circle fold 2^24 + line folds to 2^4"}
    if R is not None:
        rb_ = [[torch.empty(1 << l, dtype=torch.int32, device=dev) for _ in range(4)] for l in range(lg)]

        def fri_ref():
            R.fold_circle_into_line(itree.data_ptr(), 0, 1 << lg, ptrs(src), reflib.QM31(12345, 678, 91011, 1213),
                                    ptrs(rb_[lg - 1]))
            for l in range(lg - 1, 4, -1):
                R.fold_line(itree.data_ptr(), tsz - (1 << l), 1 << l, ptrs(rb_[l]),
                            reflib.QM31(12345, 678, 91011, 1213), ptrs(rb_[l - 1]))

        for bb in rb_[lg - 1]:
            bb.zero_()
        for bb in bufs[lg - 1]:
            bb.zero_()
        fri_ref()
        fri_ours()
        torch.cuda.synchronize()
        rec["equal_after_one_chain"] = all(torch.equal(a, c) for a, c in zip(rb_[4], bufs[4]))
        rec["reference_ms"] = timed(fri_ref)
    out["fri_fold_chain"] = rec
    del src, bufs

    # (e) DEEP quotients: 32 columns over a 2^22 domain, 4 sample points each sampling all 32 columns.
    lg, nc, nb = 22, 32, 4
    dom = stwo.CanonicCoset(lg).circle_domain()
    cols = [rand(1 << lg) for _ in range(nc)]
    outq = [torch.empty(1 << lg, dtype=torch.int32, device=dev) for _ in range(4)]
    import random
    rr = random.Random(5)

    def rq():
        return L.QM31(*[rr.randrange(P) for _ in range(4)])

    sp = (L.SPoint * nb)(*[L.SPoint(rq(), rq()) for _ in range(nb)])  # any QM31 pair works for timing
    sizes = (C.c_uint32 * nb)(*([nc] * nb))
    idx = (C.c_uint32 * (nc * nb))(*(list(range(nc)) * nb))
    vals = (L.QM31 * (nc * nb))(*[rq() for _ in range(nc * nb)])
    rcoef = rq()
    cp = ptrs(cols)

    def quot_ours():
        L.check(lib.stwo_accumulate_quotients(dom.half_coset.initial_index, dom.half_coset.step_size, lg, cp, nc,
                                              rcoef, sp, sizes, idx, vals, nb, ptrs(outq), sptr))

    t = timed(quot_ours)
    b = (1 << lg) * (4 * nc + 16)
    rec = {"ms": t, "gbs": b / t / 1e6, "frac_hbm": b / t / 1e6 / peak, "workload": "32 cols x 2^22, 4 points",
           "form": "tensor cores (tcgen05 kind::i8)"}
    # the same call on the CUDA cores (the kernel the tensor-core form replaces)
    tc_out = [o.clone() for o in outq]
    L.check(lib.stwo_set_tunable(b"quotients_tensor_cores", 0))
    try:
        rec["cuda_cores_ms"] = timed(quot_ours)
        rec["equal_cuda_cores"] = all(torch.equal(a, c) for a, c in zip(tc_out, outq))
    finally:
        L.check(lib.stwo_set_tunable(b"quotients_tensor_cores", 1))
    del tc_out
    nf = C.c_uint32()
    L.check(lib.stwo_quotients_tc_faults(C.byref(nf), 1))
    rec["tc_faults"] = nf.value
    if R is not None:
        dcols = R.copy_device_pointer_vec_from_host_to_device(cp, nc)
        rout = [torch.empty(1 << lg, dtype=torch.int32, device=dev) for _ in range(4)]
        flat_pts = (C.c_uint32 * (8 * nb))(*[v for q in sp for v in (q.x.a, q.x.b, q.x.c, q.x.d,
                                                                      q.y.a, q.y.b, q.y.c, q.y.d)])
        rvals = (reflib.QM31 * (nc * nb))(*[reflib.QM31(v.a, v.b, v.c, v.d) for v in vals])

        def quot_ref():
            R.accumulate_quotients(dom.half_coset.initial_index, dom.half_coset.step_size, 1 << lg, dcols, nc,
                                   reflib.QM31(rcoef.a, rcoef.b, rcoef.c, rcoef.d), flat_pts, idx, nc * nb, rvals,
                                   sizes, nb, *[o.data_ptr() for o in rout], nc * nb * 3)

        rec["reference_ms"] = timed(quot_ref)
        rec["equal"] = all(torch.equal(a, c) for a, c in zip(rout, outq))
        R.cuda_free_memory(dcols)
    out["quotients"] = rec
    del cols, outq

    # (f) eval_at_point: 32 polynomials of 2^22 coefficients, each at its own point, in
    # one batched call (the OODS step's shape). The reference library's kernel is not
    # run: its shared-memory arrays alias (eval_at_point.cu:17-18).
    lg, npoly = 22, 32
    polys = [rand(1 << lg) for _ in range(npoly)]
    logs = (C.c_uint32 * npoly)(*([lg] * npoly))
    spts = (L.SPoint * npoly)(*[L.SPoint(rq(), rq()) for _ in range(npoly)])
    eap_scratch_n = lib.stwo_eval_at_points_scratch_bytes(logs, npoly)
    eap_scratch = torch.zeros(eap_scratch_n // 4 + 1, dtype=torch.int32, device=dev)
    eap_res = torch.empty(4 * npoly, dtype=torch.int32, device=dev)
    pp = ptrs(polys)
    t = timed(lambda: L.check(lib.stwo_eval_at_points(pp, logs, npoly, spts, eap_res.data_ptr(),
                                                      eap_scratch.data_ptr(), eap_scratch_n, sptr)))
    b = npoly * 4 * (1 << lg)
    out["eval_at_point"] = {"ms": t, "gbs": b / t / 1e6, "frac_hbm": b / t / 1e6 / peak,
                            "workload": "32 polynomials x 2^22 coefficients, one point each"}
    del polys
    out["fft_many_columns"] = many_columns_fft(stwo, R, timed, ptrs, rand, dev, peak)
    for k, v in out.items():
        if "reference_ms" in v:
            v["speedup_vs_reference"] = v["reference_ms"] / v["ms"]
    return out


def many_columns_fft(stwo, R, timed, ptrs, rand, dev, peak):
    """The reference's own FFT harness shape (benches/evaluate_columns.rs:11-13,
    interpolate_columns.rs:10-11): 2^16 columns of 2^10 values, interpolated, and 2^16
    polynomials of 2^10 coefficients evaluated at blowup 4. Ours through the native
    column entry points (one launch per pass over a device table of the columns);
    the reference library's interpolate_columns and evaluate_columns on the same
    inputs, its evaluation on buffers already zero-extended (the extension copies of
    its evaluate_polynomials are not timed). Outputs compared on sampled columns."""
    import ctypes as C
    import torch
    L = stwo._lib
    lib = L.lib()
    lg, lb, ncols = 10, 2, 1 << 16
    N = lg + lb
    sptr = torch.cuda.current_stream(dev).cuda_stream
    hc = stwo.CanonicCoset(N).half_coset()
    tsz = 1 << hc.log_size
    tw = torch.empty(tsz, dtype=torch.int32, device=dev)
    itw = torch.empty_like(tw)
    L.check(lib.stwo_precompute_twiddles(hc.initial_index, hc.step_size, hc.log_size, tw.data_ptr(), itw.data_ptr(),
                                         sptr))
    src = rand(ncols << lg)
    work = src.clone()
    ext = torch.empty(ncols << N, dtype=torch.int32, device=dev)
    col_p = L.ptr_array([work.data_ptr() + 4 * (i << lg) for i in range(ncols)])
    ext_p = L.ptr_array([ext.data_ptr() + 4 * (i << N) for i in range(ncols)])
    logs = L.u32_array([lg] * ncols)

    def interp():
        L.check(lib.stwo_interpolate_columns(col_p, logs, ncols, itw.data_ptr(), tsz, sptr))

    def evaluate():
        L.check(lib.stwo_extend_evaluate_columns(col_p, logs, ext_p, lb, ncols, tw.data_ptr(), tsz, sptr))

    n0 = lib.stwo_kernel_launches()
    interp()
    evaluate()
    torch.cuda.synchronize()
    launches = lib.stwo_kernel_launches() - n0
    work.copy_(src)
    t_i = timed(interp)
    t_e = timed(evaluate)
    rec = {"workload": "2^16 columns x 2^10: interpolate_columns; evaluate_polynomials at blowup 4",
           "interpolate_ms": t_i, "evaluate_ms": t_e, "launches_per_step": launches,
           "interpolate_gbs": ncols * (8 << lg) / t_i / 1e6,
           "evaluate_gbs": ncols * ((4 << lg) + (4 << N)) / t_e / 1e6}
    rec["evaluate_frac_hbm"] = rec["evaluate_gbs"] / peak
    if R is not None:
        # equality on the same inputs: ours and the reference's interpolation, then the
        # reference's evaluation of its own zero-extended coefficients
        ours = src.clone()
        theirs = src.clone()
        o_p = L.ptr_array([ours.data_ptr() + 4 * (i << lg) for i in range(ncols)])
        t_p = (C.c_void_p * ncols)(*[theirs.data_ptr() + 4 * (i << lg) for i in range(ncols)])
        L.check(lib.stwo_interpolate_columns(o_p, logs, ncols, itw.data_ptr(), tsz, sptr))
        L.check(lib.stwo_extend_evaluate_columns(o_p, logs, ext_p, lb, ncols, tw.data_ptr(), tsz, sptr))
        torch.cuda.synchronize()
        R.interpolate_columns(1 << (lg - 1), t_p, itw.data_ptr(), tsz, ncols, 1 << lg)
        rext = torch.zeros(ncols << N, dtype=torch.int32, device=dev)
        rext.view(ncols, 1 << N)[:, : 1 << lg].copy_(theirs.view(ncols, 1 << lg))
        re_p = (C.c_void_p * ncols)(*[rext.data_ptr() + 4 * (i << N) for i in range(ncols)])
        dom = (C.c_int * ncols)(*([1 << (N - 1)] * ncols))
        szs = (C.c_int * ncols)(*([1 << N] * ncols))
        R.evaluate_columns(dom, re_p, tw.data_ptr(), tsz, ncols, szs)
        torch.cuda.synchronize()
        sample = [0, 1, 63, 64, 1000, ncols // 2, ncols - 1]
        ov, tv = ours.view(ncols, -1), theirs.view(ncols, -1)
        oe, te = ext.view(ncols, -1), rext.view(ncols, -1)
        rec["equal_sampled_columns"] = all(torch.equal(ov[k], tv[k]) and torch.equal(oe[k], te[k]) for k in sample)
        rec["reference_interpolate_ms"] = timed(
            lambda: R.interpolate_columns(1 << (lg - 1), t_p, itw.data_ptr(), tsz, ncols, 1 << lg))
        rec["reference_evaluate_ms"] = timed(lambda: R.evaluate_columns(dom, re_p, tw.data_ptr(), tsz, ncols, szs))
        rec["reference_ms"] = rec["reference_interpolate_ms"] + rec["reference_evaluate_ms"]
        del ours, theirs, rext
    rec["ms"] = t_i + t_e
    del src, work, ext
    torch.cuda.empty_cache()
    return rec


def job_stream(n, seed):
    """n seeded jobs: (log_n_rows, n_columns, input seed)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(12, 21)), int(rng.integers(16, 257)), int(rng.integers(0, 1 << 62))) for _ in range(n)]


def job_of(stwo, t):
    return stwo.WideFibJob(t[0], t[1], 1, 3, 5)


def job_desc(n_jobs):
    return (f"seeded wide-Fibonacci proof stream: log_n_rows U{{12..20}}, columns U{{16..256}}, log_blowup 1, "
            f"3 queries, pow_bits 5; {n_jobs} jobs per step admitted at once")


def cpu_stream_sample(S, stwo, jobs, budget_s, threads, min_jobs=32):
    """The SIMD CPU prover (S: oracle/simd.py) on jobs of the stream, in order, until
    min_jobs are done or budget_s of CPU work has gone by (at least one job). Returns
    (jobs done, seconds, description)."""
    S.set_threads(threads)
    done, t0 = 0, time.perf_counter()
    for t in jobs:
        a0, a1 = stwo.wide_fib_inputs(t[0], t[2])
        S.wide_fib_prove(t[0], t[1], a0, a1, 1, 3, 5)
        done += 1
        if done >= min_jobs or time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return done, dt, (f"first {done} jobs of the stream, SIMD CPU prover ({S.variant()}, {S.lanes()} lanes) on "
                      f"{threads} host threads")


def run_reference(args, rank, world):
    if rank != 0:
        return
    S = load_simd()
    stwo = load_package()
    threads = os.cpu_count() or 1
    for w in range(args.warmup):  # warm-up: one 64-column x 2^12 job each
        cpu_stream_sample(S, stwo, [(12, 64, 7000 + w)], 0.0, threads, 1)
    # Each step: the stream's first jobs until 32 are done or --cpu-budget seconds have
    # gone by (at least one job); steps stop once --cpu-total-budget seconds have gone
    # by, so the whole run stays within a few minutes.
    n_total, t_total, steps_done = 0, 0.0, 0
    for s in range(args.steps):
        if steps_done and t_total >= args.cpu_total_budget:
            break
        n, dt, _ = cpu_stream_sample(S, stwo, job_stream(args.jobs, 1000 + s), args.cpu_budget, threads)
        n_total += n
        t_total += dt
        steps_done += 1
    value = n_total / t_total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "m31 (u32)",
        "data": "synthetic (seeded SplitMix64 M31 trace inputs)",
        "config": {"workload": job_desc(args.jobs) + f" (CPU: a bounded sample of each step, ~{args.cpu_budget:.0f} s)",
                   "jobs_per_step": args.jobs},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n_total} jobs over {steps_done} of {args.steps} steps (at most "
                                   f"{args.cpu_total_budget:.0f} s in all), each step the stream's first 32 jobs "
                                   f"or {args.cpu_budget:.0f} s of them; SIMD CPU prover (SimdBackend stand-in, "
                                   f"{S.variant()}, {S.lanes()} lanes, proof bytes equal to the oracle's), "
                                   f"{threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fft_roofline(stwo, dev, rank, args):
    """The M31 circle FFT step (8 columns at log 24: interpolate, extend-evaluate
    blowup 4), its HBM roofline and the reference CUDA library on the same step."""
    import ctypes as C
    import torch
    L = stwo._lib
    lib = L.lib()
    ncols, lg, lb = 8, 24, 2
    N = lg + lb
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    hc = stwo.CanonicCoset(N).half_coset()
    tree_size = 1 << hc.log_size
    tw = torch.empty(tree_size, dtype=torch.int32, device=dev)
    itw = torch.empty(tree_size, dtype=torch.int32, device=dev)
    L.check(lib.stwo_precompute_twiddles(hc.initial_index, hc.step_size, hc.log_size, tw.data_ptr(),
                                         itw.data_ptr(), sptr))
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    evals = [torch.randint(0, P, (1 << lg,), dtype=torch.int64, device=dev, generator=gen).to(torch.int32)
             for _ in range(ncols)]
    outs = [torch.empty(1 << N, dtype=torch.int32, device=dev) for _ in range(ncols)]
    ev_ptrs = L.ptr_array([t.data_ptr() for t in evals])
    out_ptrs = L.ptr_array([t.data_ptr() for t in outs])
    logs = L.u32_array([lg] * ncols)

    def interp():
        L.check(lib.stwo_interpolate_columns(ev_ptrs, logs, ncols, itw.data_ptr(), tree_size, sptr))

    def extend_eval():
        L.check(lib.stwo_extend_evaluate_columns(ev_ptrs, logs, out_ptrs, lb, ncols, tw.data_ptr(), tree_size, sptr))

    for _ in range(3):
        interp()
        extend_eval()
    torch.cuda.synchronize()
    reps = 5
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for e0, e1, e2 in ev:
        e0.record(stream)
        interp()
        e1.record(stream)
        extend_eval()
        e2.record(stream)
    torch.cuda.synchronize()
    t_interp = sum(a.elapsed_time(b) for a, b, _ in ev) / reps
    t_eval = sum(b.elapsed_time(c) for _, b, c in ev) / reps
    # algorithmic bytes: one read + one write per element (interpolate 8 B per element;
    # evaluate 4 B per coefficient read + 4 B per evaluation written); twiddles not counted
    b_interp = ncols * (1 << lg) * 8
    b_eval = ncols * ((1 << lg) * 4 + (1 << N) * 4)
    achieved = (b_interp + b_eval) / ((t_interp + t_eval) / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tf = os.path.join(ROOT, "profiles", "fft_traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get("dram_bytes_per_step")
    ref_gpu = None
    if rank == 0 and not args.no_suite:
        ns = argparse.Namespace(**vars(args))
        ref_gpu = reference_gpu_timing(ns, evals, lg, lb, ncols, tw, itw, tree_size)
    # The integer ceiling, measured live: the passes' own butterfly on register operands
    # (stwo_probe_m31_butterflies), against the step's butterflies (interpolate: lg
    # layers of 2^(lg-1); evaluate: lg layers of 2^(N-1), the lb top layers of the
    # zero-padded input being copies).
    bf_step = ncols * lg * ((1 << (lg - 1)) + (1 << (N - 1)))
    sink = torch.empty(2048 * torch.cuda.get_device_properties(dev).multi_processor_count, dtype=torch.int32,
                       device=dev)
    nbf = C.c_uint64()

    def probe():
        L.check(lib.stwo_probe_m31_butterflies(4096, sink.data_ptr(), sink.numel(), C.byref(nbf), sptr))

    probe()
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    for _ in range(3):
        probe()
    pe1.record(stream)
    torch.cuda.synchronize()
    ceiling = 3 * nbf.value / (pe0.elapsed_time(pe1) / 1e3)
    fft_rate = bf_step / ((t_interp + t_eval) / 1e3)
    roof = {"bound": "hbm", "kernel": "fftT_kernel / fft_pass_kernel (circle FFT, 8 columns x 2^24, blowup 4)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": traffic, "interpolate_ms": t_interp, "evaluate_ms": t_eval,
            "algorithmic_bytes_per_step": b_interp + b_eval,
            "integer_ceiling": {"butterflies_per_s": ceiling, "fft_butterflies_per_s": fft_rate,
                                "frac": fft_rate / ceiling, "butterflies_per_step": bf_step,
                                "what": "the passes' forward butterfly on register operands (probe kernel), "
                                        "the bound the passes meet before HBM"}}
    fft = {"columns_per_s": ncols / ((t_interp + t_eval) / 1e3), "unit": FFT_UNIT, "reference_gpu": ref_gpu}
    del evals, outs, tw, itw
    torch.cuda.empty_cache()
    return roof, fft


class StreamRunner:
    """Submits jobs to a ProofServer (resident device inputs or host inputs) and
    collects every result on a polling thread."""

    def __init__(self, stwo, workers, max_domain_log=22):
        self.stwo = stwo
        # One worker is the one-job-at-a-time reference: it proves queued jobs of one
        # shape one by one, not as a batch (STWO_SERVER_BATCH is read at creation).
        saved = os.environ.get("STWO_SERVER_BATCH")
        if workers == 1:
            os.environ["STWO_SERVER_BATCH"] = "1"
        try:
            self.srv = stwo.ProofServer(n_workers=workers, device_budget_bytes=BUDGET,
                                        max_domain_log=max_domain_log)
        finally:
            if saved is None:
                os.environ.pop("STWO_SERVER_BATCH", None)
            else:
                os.environ["STWO_SERVER_BATCH"] = saved

    def run(self, jobs, inputs, resident, arrivals_ms=None, device_time=False, hold=False):
        """jobs: list of (L, N, seed); inputs[i] = (host a0, host a1, dev a0, dev a1).
        arrivals_ms: offsets from the start (None: all at once). hold: the server is paused
        while the jobs are submitted and resumed after the last one, so all of them are
        queued when the workers start (and the clock starts at the resume). Returns
        (results by index, ms from the first submit to the last completion): host wall
        time, or with device_time the device time from an epoch event recorded just
        before the first submission to the end of the last job's final GPU operation
        (CUDA events)."""
        stwo, srv = self.stwo, self.srv
        results = {}
        done = threading.Event()
        if hold:
            srv.pause()
        if device_time and not hold:
            srv.mark_epoch()

        def poller():
            while len(results) < len(jobs):
                for r in srv.poll(timeout_ms=50):
                    results[int(r["job_id"])] = r
            done.set()

        th = threading.Thread(target=poller, daemon=True)
        th.start()
        t0 = srv.now_ms()
        for i, t in enumerate(jobs):
            if arrivals_ms is not None:
                wait = t0 + arrivals_ms[i] - srv.now_ms()
                if wait > 0:
                    time.sleep(wait / 1e3)
            h0, h1, d0, d1 = inputs[i]
            if resident:
                srv.submit_device(i, job_of(stwo, t), d0.data_ptr(), d1.data_ptr())
            else:
                srv.submit(i, job_of(stwo, t), h0, h1)
        if hold:
            if device_time:
                srv.mark_epoch()
            t0 = srv.now_ms()
            srv.resume()
        done.wait()
        th.join()
        bad = [r for r in results.values() if r["status"] != 0]
        if bad:
            raise RuntimeError(f"proof failed: {bad[0]['error']}")
        self.last_wall_ms = max(r["done_ms"] for r in results.values()) - t0
        if device_time:
            dev = [r["device_done_ms"] for r in results.values()]
            if min(dev) < 0:
                raise RuntimeError("a job has no device completion time")
            return results, max(dev)
        return results, self.last_wall_ms

    def close(self):
        self.srv.close()


def percentiles(xs):
    import numpy as np
    a = np.array(xs)
    return {"p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99)),
            "p999_ms": float(np.percentile(a, 99.9)), "mean_ms": float(a.mean())}


def batch48(stwo, dev, args, O=None):
    """The batched-uneven-sizes case: 48 seeded jobs, log_n_rows uniform in {10..20},
    columns uniform in {16, 32, 64, 128}, admitted at once to the proof server, each
    proof compared with the same job proved alone; and one Merkle tree mixing
    columns of log sizes 12..22 (4 per size), its root compared with the oracle's."""
    import numpy as np
    import torch
    rng = np.random.default_rng(4848)
    jobs = [(int(rng.integers(10, 21)), int(rng.choice([16, 32, 64, 128])), int(rng.integers(0, 1 << 62)))
            for _ in range(48)]
    ins = []
    for t in jobs:
        a0, a1 = stwo.wide_fib_inputs(t[0], t[2])
        ins.append((a0, a1, torch.from_numpy(a0.view(np.int32)).to(dev), torch.from_numpy(a1.view(np.int32)).to(dev)))
    batched, single = StreamRunner(stwo, args.workers), StreamRunner(stwo, 1)
    batched.run(jobs[:8], ins[:8], resident=True)
    single.run(jobs[:2], ins[:2], resident=True)
    res_b, ms_b = batched.run(jobs, ins, resident=True, device_time=True)
    res_s, ms_s = single.run(jobs, ins, resident=True, device_time=True)
    b48_batches = batched.srv.batch_stats()
    batched.close()
    single.close()
    identical = all(res_b[i]["proof"] == res_s[i]["proof"] for i in range(len(jobs)))
    # mixed-size tree: layer l hashes its children and the 4 columns of size 2^l (12 <= l <= 22)
    L = stwo._lib
    lib = L.lib()
    sptr = torch.cuda.current_stream(dev).cuda_stream
    top = 22
    cols = {l: [torch.randint(0, P, (1 << l,), dtype=torch.int64, device=dev).to(torch.int32) for _ in range(4)]
            for l in range(12, top + 1)}
    layers = [torch.empty(8 << l, dtype=torch.int32, device=dev) for l in range(top + 1)]

    def tree():
        for l in range(top, -1, -1):
            cs = cols.get(l, [])
            L.check(lib.stwo_merkle_commit_layer(l, layers[l + 1].data_ptr() if l < top else None,
                                                 L.ptr_array([c.data_ptr() for c in cs]), len(cs),
                                                 layers[l].data_ptr(), sptr))
    # the same tree through stwo_merkle_commit_tree: one launch for all 23 layers
    all_cols = [c for l in range(top, 11, -1) for c in cols[l]]
    all_logs = [l for l in range(top, 11, -1) for _ in cols[l]]
    layers_t = [torch.empty(8 << l, dtype=torch.int32, device=dev) for l in range(top + 1)]
    col_p, log_a = L.ptr_array([c.data_ptr() for c in all_cols]), L.u32_array(all_logs)
    lay_p = L.ptr_array([x.data_ptr() for x in layers_t])

    def tree_one_call():
        L.check(lib.stwo_merkle_commit_tree(col_p, log_a, len(all_cols), top, lay_p, sptr))

    def timed3(fn):
        fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(torch.cuda.current_stream(dev))
        for _ in range(3):
            fn()
        e.record(torch.cuda.current_stream(dev))
        torch.cuda.synchronize()
        return s.elapsed_time(e) / 3

    tree_ms = timed3(tree)
    n0 = lib.stwo_kernel_launches()
    tree_one_call()
    torch.cuda.synchronize()
    tree_call_launches = lib.stwo_kernel_launches() - n0
    tree_call_ms = timed3(tree_one_call)
    tree_call_equal = all(torch.equal(a, b) for a, b in zip(layers, layers_t))
    root_equal = None
    if O is not None:
        O.set_threads(os.cpu_count() or 1)
        prev = None
        for l in range(top, -1, -1):
            prev = O.merkle_commit_on_layer(l, prev, [c.cpu().numpy().view(np.uint32) for c in cols.get(l, [])])
        O.set_threads(1)
        root_equal = bool((prev.reshape(-1) == layers[0].cpu().numpy().view(np.uint32)).all())
    return {"jobs": 48, "workload": "log_n_rows U{10..20}, columns U{16,32,64,128}, log_blowup 1, 3 queries, "
                                    "pow_bits 5, all 48 admitted at once",
            "proofs_per_s": len(jobs) / (ms_b / 1e3), "per_job_proofs_per_s": len(jobs) / (ms_s / 1e3),
            "batched_vs_per_job": ms_s / ms_b, "bit_identical": identical, "launch_sequence_batches": b48_batches,
            "mixed_tree": {"columns": "4 per log size 12..22", "ms": tree_ms, "root_equal_to_oracle": root_equal,
                           "one_call_ms": tree_call_ms, "one_call_launches": tree_call_launches,
                           "one_call_equal": tree_call_equal}}


def same_shape(stwo, dev):
    """Repeated-shape serving: 96 jobs of the 64-column x 2^12 proof (each with its own
    inputs) through the server, batched (8 workers) and one at a time. Batched, a worker
    that takes a job also takes the queued jobs of its shape (up to 32) and proves them
    in one launch sequence (stwo_wide_fib_prove_batch); one at a time, the worker reuses
    its slab for consecutive jobs of one shape and replays the proof's CUDA graph. The
    server is paused while the 96 jobs are submitted (stwo_server_pause), so the batches
    do not depend on how the workers' wake-ups interleave with the submissions."""
    import numpy as np
    import torch
    jobs = [(12, 64, 4200 + k) for k in range(96)]
    ins = []
    for t in jobs:
        a0, a1 = stwo.wide_fib_inputs(t[0], t[2])
        ins.append((a0, a1, torch.from_numpy(a0.view(np.int32)).to(dev), torch.from_numpy(a1.view(np.int32)).to(dev)))
    out = {"jobs": len(jobs), "workload": "64 columns x 2^12 rows, log_blowup 1, 3 queries, pow_bits 5, all queued "
                                          "(server paused while submitting), then admitted at once"}
    for name, w in (("batched", 8), ("one_at_a_time", 1)):
        r = StreamRunner(stwo, w)
        r.run(jobs[:16], ins[:16], resident=True, hold=True)
        best = None
        for _ in range(3):
            res, ms = r.run(jobs, ins, resident=True, hold=True)
            if best is None or ms < best[1]:
                best = (res, ms)
        res, ms = best
        per = sorted(v["done_ms"] - v["start_ms"] for v in res.values())
        out[name] = {"proofs_per_s": len(jobs) / (ms / 1e3), "median_job_ms": per[len(per) // 2],
                     **r.srv.graph_stats(), **r.srv.batch_stats()}
        r.close()
    return out


def _sig(x, n=5):
    """x with every float rounded to n significant digits (nested)."""
    if isinstance(x, float):
        return float(f"{x:.{n}g}")
    if isinstance(x, dict):
        return {k: _sig(v, n) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_sig(v, n) for v in x]
    return x


def compact_line(full, detail_path):
    """The printed JSON line: the contract's keys first, then short summaries of each
    record, ending with the serving comparison (batched vs one at a time, latency
    percentiles), so that the end of the line carries the metric. The full record is
    written to detail_path."""
    if detail_path:
        os.makedirs(os.path.dirname(os.path.abspath(detail_path)), exist_ok=True)
        with open(detail_path, "w") as f:
            json.dump(full, f, indent=1)
    keep = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
            "vs_baseline", "dtype", "data", "config", "gpu_launches", "clocks", "cpu_baseline", "e2e")
    line = {k: full[k] for k in keep}
    line["detail"] = detail_path
    k = full.get("kernels")
    if k:
        line["kernels"] = {
            name: {kk: v[kk] for kk in ("ms", "frac_hbm", "frac_alu_bound", "tree_frac_alu_bound", "evaluate_frac_hbm",
                                        "launches_per_step", "speedup_vs_reference", "equal", "root_equal",
                                        "equal_after_one_chain", "equal_sampled_columns") if kk in v}
            for name, v in k.items()}
    sp = full.get("single_proofs")
    if sp:
        line["single_proofs"] = {
            name: dict({kk: v.get(kk) for kk in ("ms_median", "cached_ms_median", "oracle_ms", "equal_to_oracle",
                                                  "simd_cpu_ms", "simd_cpu_equal", "verified")},
                       phases_ms=v.get("phases_ms"))
            for name, v in sp.items()}
    ss = full.get("same_shape")
    if ss:
        line["same_shape"] = {"batched_proofs_per_s": ss["batched"]["proofs_per_s"],
                              "one_at_a_time_proofs_per_s": ss["one_at_a_time"]["proofs_per_s"],
                              "batched_launch_sequences": ss["batched"].get("batches"),
                              "jobs_in_launch_sequences": ss["batched"].get("batched_jobs")}
    b = full.get("batch48")
    if b:
        line["batch48"] = {kk: b[kk] for kk in ("proofs_per_s", "per_job_proofs_per_s", "batched_vs_per_job",
                                                "bit_identical")}
        line["batch48"]["mixed_tree_root_equal_to_oracle"] = b["mixed_tree"]["root_equal_to_oracle"]
        line["batch48"]["mixed_tree_ms_layer_calls_vs_one_call"] = [b["mixed_tree"]["ms"], b["mixed_tree"]["one_call_ms"]]
        line["batch48"]["mixed_tree_one_call_launches"] = b["mixed_tree"]["one_call_launches"]
    fft = full.get("fft")
    if fft:
        rg = fft.get("reference_gpu") or {}
        line["fft"] = {"columns_per_s": fft["columns_per_s"], "reference_gpu_columns_per_s": rg.get("value"),
                       "reference_gpu_equal": rg.get("equal")}
    r = full["roofline"]
    line["roofline"] = {kk: r[kk] for kk in ("bound", "kernel", "achieved", "peak", "unit", "frac", "peak_kind",
                                             "traffic", "interpolate_ms", "evaluate_ms")}
    line["roofline"]["integer_ceiling_frac"] = r["integer_ceiling"]["frac"]
    s = full["serving"]
    line["serving"] = {"batched_proofs_per_s": full["value"], "per_job_proofs_per_s": s["per_job_proofs_per_s"],
                       "bit_identical": s["bit_identical"], "proofs_compared": s["proofs_compared"],
                       "verified_sample": s["verified_sample"],
                       "latency_ms_p50_p99_p999": {
                           load: {mode: [e[mode]["p50_ms"], e[mode]["p99_ms"], e[mode]["p999_ms"]]
                                  for mode in ("batched", "per_job")}
                           for load, e in s["latency"].items()},
                       "batched_vs_per_job": s["batched_vs_per_job"]}
    return _sig(line)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    # Server workers poll the device for up to 2 ms before blocking; with more workers on
    # this node than half its host threads (several replicas), polling would take cores
    # from the workers that launch, so they block at once.
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    if "STWO_SERVER_SPIN_US" not in os.environ and world * args.workers > cores // 2:
        os.environ["STWO_SERVER_SPIN_US"] = "0"
    stwo = load_package()
    import ctypes as C
    tune_buf = C.create_string_buffer(4096)
    stwo._lib.check(stwo._lib.lib().stwo_autotune(tune_buf, 4096))
    autotune = json.loads(tune_buf.value.decode())

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def inputs_for(jobs):
        out = []
        for t in jobs:
            a0, a1 = stwo.wide_fib_inputs(t[0], t[2])
            out.append((a0, a1, torch.from_numpy(a0.view(np.int32)).to(dev), torch.from_numpy(a1.view(np.int32)).to(dev)))
        return out

    # Per-rank streams (weak scaling): rank r proves its own seeded jobs.
    steps = [job_stream(args.jobs, 1000 + s + 7919 * rank) for s in range(args.steps)]
    # Warm-up steps draw full-size steps from the same distribution (other seeds), so
    # the memory pool and per-size state reach their steady state before timing.
    warm = [job_stream(args.jobs, 7000 + w + 7919 * rank) for w in range(args.warmup)]
    step_inputs = [inputs_for(js) for js in steps]
    warm_inputs = [inputs_for(js) for js in warm]
    torch.cuda.synchronize()

    batched = StreamRunner(stwo, args.workers)
    for js, ins in zip(warm, warm_inputs):
        batched.run(js, ins, resident=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    # ---- timed: the batched server, inputs resident in HBM
    launches0 = stwo.kernel_launches()
    step_ms, step_wall_ms, batched_results = [], [], []
    with ClockSampler(local_rank) as clk:
        for js, ins in zip(steps, step_inputs):
            res, ms = batched.run(js, ins, resident=True, device_time=True)
            step_ms.append(ms)
            step_wall_ms.append(batched.last_wall_ms)
            batched_results.append(res)
        torch.cuda.synchronize()
    barrier()
    launches = stwo.kernel_launches() - launches0
    local_ms = sum(step_ms) / len(step_ms)
    ms_step, value = replica_throughput(local_ms, args.jobs, world, dev)

    # ---- end to end: host inputs copied in by the server
    e2e_ms, e2e_wall_ms = [], []
    for js, ins in zip(steps, step_inputs):
        _, ms = batched.run(js, ins, resident=False, device_time=True)
        e2e_ms.append(ms)
        e2e_wall_ms.append(batched.last_wall_ms)
    e2e_step, e2e_value = replica_throughput(sum(e2e_ms) / len(e2e_ms), args.jobs, world, dev)
    h2d = sum(8 << t[0] for t in steps[0])
    d2h = sum(len(r["proof"]) for r in batched_results[0].values())

    # ---- one job at a time on the same jobs (one worker), and byte-for-byte comparison
    single = StreamRunner(stwo, 1)
    single.run(warm[0], warm_inputs[0], resident=True)
    per_ms, identical, compared = [], True, 0
    for js, ins, bres in zip(steps, step_inputs, batched_results):
        res, ms = single.run(js, ins, resident=True, device_time=True)
        per_ms.append(ms)
        for i in res:
            compared += 1
            identical = identical and res[i]["proof"] == bres[i]["proof"]
    per_step, per_value = replica_throughput(sum(per_ms) / len(per_ms), args.jobs, world, dev)

    # ---- Poisson arrivals at three loads (fractions of the one-at-a-time throughput)
    latency = {}
    lat_jobs = job_stream(args.latency_jobs, 4242 + 7919 * rank)
    lat_inputs = inputs_for(lat_jobs)
    rng = np.random.default_rng(99)
    per_rate = per_value / world  # proofs/s of one GPU one at a time
    for load in (0.5, 0.9, 1.5):
        gaps = rng.exponential(1e3 / (load * per_rate), size=len(lat_jobs))
        arrivals = np.cumsum(gaps) - gaps[0]
        entry = {"arrival_rate_per_s": load * per_rate}
        for name, runner in (("batched", batched), ("per_job", single)):
            res, ms = runner.run(lat_jobs, lat_inputs, resident=True, arrivals_ms=list(arrivals))
            lat = [r["done_ms"] - r["submit_ms"] for r in res.values()]
            entry[name] = dict(percentiles(lat), proofs_per_s=len(res) / (ms / 1e3))
        latency[f"load_{load}x"] = entry
    single.close()
    batched.close()
    del step_inputs, warm_inputs, lat_inputs
    torch.cuda.empty_cache()

    # ---- single proofs, FFT roofline, kernel sweep, CPU baseline (rank 0, 1 GPU)
    roof, fft = fft_roofline(stwo, dev, rank, args)
    singles, kernels, cpu, verified, batch, repeated = None, None, None, None, None, None
    if rank == 0:
        O = load_oracle() if not args.no_cpu_baseline else None
        S = load_simd() if not args.no_cpu_baseline else None
        singles = {}
        # The reference CpuBackend's case (64 x 2^12), the large single proof (256 x 2^20,
        # pow_bits 10) and the reference's own end-to-end shape (1024 x 2^16,
        # examples/wide_fibonacci.rs:19-20), each compared byte for byte with the oracle
        # prover (on every host thread), whose time is reported beside the GPU's.
        for name, t in (("cols64_log12", (12, 64, 1, 3, 5)), ("cols256_log20", (20, 256, 1, 3, 10)),
                        ("cols1024_log16", (16, 1024, 1, 3, 5))):
            job = stwo.WideFibJob(*t)
            a0, a1 = stwo.wide_fib_inputs(t[0], 1)
            stwo.prove_wide_fib(job, a0, a1)
            times, stats = [], None
            for _ in range(5):
                t0 = time.perf_counter()
                proof, stats = stwo.prove_wide_fib(job, a0, a1)
                times.append((time.perf_counter() - t0) * 1e3)
            ent = {"job": dict(zip(["log_n_rows", "n_columns", "log_blowup", "n_queries", "pow_bits"], t)),
                   "ms_median": float(np.median(times)), "phases_ms": {k: stats[k] for k in
                   ("trace_ms", "composition_ms", "oods_ms", "fri_ms", "decommit_ms")},
                   "kernel_launches": stats["kernel_launches"], "proof_bytes": len(proof),
                   "verified": bool(stwo.verify(proof, *t))}
            if O is not None:
                O.set_threads(os.cpu_count() or 1)
                t0 = time.perf_counter()
                want, _ = O.wide_fib_prove(t[0], t[1], a0, a1, *t[2:])
                ent["oracle_ms"] = (time.perf_counter() - t0) * 1e3
                ent["oracle_threads"] = os.cpu_count() or 1
                ent["equal_to_oracle"] = want == proof
                O.set_threads(1)
                S.set_threads(os.cpu_count() or 1)
                t0 = time.perf_counter()
                sproof, _ = S.wide_fib_prove(t[0], t[1], a0, a1, *t[2:])
                ent["simd_cpu_ms"] = (time.perf_counter() - t0) * 1e3
                ent["simd_cpu_equal"] = sproof == proof
            # The same proof repeated through a ProveCache (shared tree, own stream):
            # memory reused, launch sequence replayed as a CUDA graph.
            cs = torch.cuda.Stream(dev)
            tree = stwo.CudaBackend.precompute_twiddles(stwo.CanonicCoset(t[0] + 1 + t[2]).half_coset())
            ctimes = []
            with stwo.ProveCache() as cache:
                for k in range(8):
                    t0 = time.perf_counter()
                    cproof, _ = stwo.prove_wide_fib(job, a0, a1, twiddles=tree, stream=cs.cuda_stream, cache=cache)
                    ctimes.append((time.perf_counter() - t0) * 1e3)
                ent["cached_ms_median"] = float(np.median(ctimes[3:]))
                ent["cached_graph_replays"] = cache.stats()["graph_replays"]
                ent["cached_equal"] = cproof == proof
                cache.close(cs.cuda_stream)
            del tree
            singles[name] = ent
        verified = all(stwo.verify(batched_results[0][i]["proof"], *dataclasses.astuple(job_of(stwo, steps[0][i])))
                       for i in range(min(2, args.jobs)))
        if world == 1 and not args.no_suite:
            kernels = kernel_suite(stwo)
            batch = batch48(stwo, dev, args, O)
            repeated = same_shape(stwo, dev)
        if S is not None and world == 1:
            threads = os.cpu_count() or 1
            n, dt, desc = cpu_stream_sample(S, stwo, steps[0], args.cpu_stream_budget, threads)
            cpu = {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}

    if rank == 0:
        full = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "m31 (u32)", "data": "synthetic (seeded SplitMix64 M31 trace inputs)",
            "config": {"workload": job_desc(args.jobs), "jobs_per_step": args.jobs, "workers": args.workers,
                       "worker_poll_us_before_blocking": int(os.environ.get("STWO_SERVER_SPIN_US", "2000")),
                       "device_budget_gb": BUDGET >> 30, "inputs": "resident in HBM before the timed region",
                       "warmup_steps": f"{args.warmup} steps of {args.jobs} jobs from the same distribution, other seeds",
                       "timing": "device: CUDA event on an idle stream just before the first submission to the "
                                 "last job's final GPU operation (its completion event), per step; "
                                 "host wall time alongside as wall_ms_per_step",
                       "wall_ms_per_step": sum(step_wall_ms) / len(step_wall_ms),
                       "l2": "each job's columns and trees are freshly written; the stream's working set "
                             "(GBs) exceeds the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "serving": {"per_job_proofs_per_s": per_value, "batched_vs_per_job": value / per_value,
                        "bit_identical": identical, "proofs_compared": compared, "verified_sample": verified,
                        "latency": latency, "latency_jobs": args.latency_jobs},
            "single_proofs": singles,
            "batch48": batch,
            "same_shape": repeated,
            "roofline": roof,
            "fft": fft,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_step, "wall_ms_per_step": sum(e2e_wall_ms) / len(e2e_wall_ms)},
            "kernels": kernels,
            "autotune": autotune,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(compact_line(full, args.detail_out)), flush=True)


def run_profile(args):
    """One workload between cudaProfilerStart/Stop for ncu (--profile-from-start off),
    after warm-up: `fft[:LOG]` (8 columns at LOG, interpolate + blowup-4 evaluate, two
    steps), `proof:L,N` (one wide-Fibonacci proof, log_blowup 1, 3 queries, pow_bits 5)
    `merkle` (the 64 x 2^22 tree of the kernel sweep), `quotients` (the sweep's 32
    columns x 2^22 with 4 sample points), `fri` (the sweep's fold chain, 2^24 down to
    2^4) or `inverse` (the sweep's batch inverse of 2^24 QM31)."""
    import numpy as np
    import torch
    stwo = load_package()
    L = stwo._lib
    lib = L.lib()
    dev = torch.device("cuda", 0)
    what = args.profile
    if what.startswith("fft"):
        lg = int(what.split(":")[1]) if ":" in what else 24
        ncols, lb = 8, 2
        N = lg + lb
        sptr = torch.cuda.current_stream(dev).cuda_stream
        hc = stwo.CanonicCoset(N).half_coset()
        tsz = 1 << hc.log_size
        tw = torch.empty(tsz, dtype=torch.int32, device=dev)
        itw = torch.empty(tsz, dtype=torch.int32, device=dev)
        L.check(lib.stwo_precompute_twiddles(hc.initial_index, hc.step_size, hc.log_size, tw.data_ptr(),
                                             itw.data_ptr(), sptr))
        evals = [torch.randint(0, P, (1 << lg,), dtype=torch.int64, device=dev).to(torch.int32) for _ in range(ncols)]
        outs = [torch.empty(1 << N, dtype=torch.int32, device=dev) for _ in range(ncols)]
        ev_p, out_p, logs = L.ptr_array([t.data_ptr() for t in evals]), L.ptr_array([t.data_ptr() for t in outs]), \
            L.u32_array([lg] * ncols)

        def work():
            L.check(lib.stwo_interpolate_columns(ev_p, logs, ncols, itw.data_ptr(), tsz, sptr))
            L.check(lib.stwo_extend_evaluate_columns(ev_p, logs, out_p, lb, ncols, tw.data_ptr(), tsz, sptr))
        reps = 2
    elif what.startswith("proof:"):
        lg, nc = (int(x) for x in what.split(":")[1].split(","))
        job = stwo.WideFibJob(lg, nc, 1, 3, 5)
        a0, a1 = stwo.wide_fib_inputs(lg, 7)

        def work():
            stwo.prove_wide_fib(job, a0, a1)
        reps = 1
    elif what == "merkle":
        lg, nc = 22, 64
        sptr = torch.cuda.current_stream(dev).cuda_stream
        cols = [torch.randint(0, P, (1 << lg,), dtype=torch.int64, device=dev).to(torch.int32) for _ in range(nc)]
        layers = [torch.empty(8 << l, dtype=torch.int32, device=dev) for l in range(lg + 1)]
        cptr = L.ptr_array([c.data_ptr() for c in cols])

        def work():
            L.check(lib.stwo_merkle_commit_layer(lg, None, cptr, nc, layers[lg].data_ptr(), sptr))
            for l in range(lg - 1, -1, -1):
                L.check(lib.stwo_merkle_commit_layer(l, layers[l + 1].data_ptr(), None, 0, layers[l].data_ptr(), sptr))
        reps = 1
    elif what.startswith("merkle_tree"):  # merkle_tree[:COLS,LOG]: one stwo_merkle_commit_tree call
        nc, lg = (int(x) for x in what.split(":")[1].split(",")) if ":" in what else (64, 22)
        sptr = torch.cuda.current_stream(dev).cuda_stream
        cols = [torch.randint(0, P, (1 << lg,), dtype=torch.int64, device=dev).to(torch.int32) for _ in range(nc)]
        layers = [torch.empty(8 << l, dtype=torch.int32, device=dev) for l in range(lg + 1)]
        cptr, logs = L.ptr_array([c.data_ptr() for c in cols]), L.u32_array([lg] * nc)
        lay = L.ptr_array([x.data_ptr() for x in layers])

        def work():
            L.check(lib.stwo_merkle_commit_tree(cptr, logs, nc, lg, lay, sptr))
        reps = 1
    elif what == "quotients":
        import ctypes as C
        import random
        lg, nc, nb = 22, 32, 4
        sptr = torch.cuda.current_stream(dev).cuda_stream
        dom = stwo.CanonicCoset(lg).circle_domain()
        cols = [torch.randint(0, P, (1 << lg,), dtype=torch.int64, device=dev).to(torch.int32) for _ in range(nc)]
        outq = [torch.empty(1 << lg, dtype=torch.int32, device=dev) for _ in range(4)]
        rr = random.Random(5)

        def rq():
            return L.QM31(*[rr.randrange(P) for _ in range(4)])
        sp = (L.SPoint * nb)(*[L.SPoint(rq(), rq()) for _ in range(nb)])
        sizes = (C.c_uint32 * nb)(*([nc] * nb))
        idx = (C.c_uint32 * (nc * nb))(*(list(range(nc)) * nb))
        vals = (L.QM31 * (nc * nb))(*[rq() for _ in range(nc * nb)])
        rcoef = rq()
        cp, op = L.ptr_array([c.data_ptr() for c in cols]), L.ptr_array([c.data_ptr() for c in outq])

        def work():
            L.check(lib.stwo_accumulate_quotients(dom.half_coset.initial_index, dom.half_coset.step_size, lg, cp, nc,
                                                  rcoef, sp, sizes, idx, vals, nb, op, sptr))
        reps = 1
    elif what == "fri":
        lg = 24
        sptr = torch.cuda.current_stream(dev).cuda_stream
        hc = stwo.CanonicCoset(lg).half_coset()
        tsz = 1 << hc.log_size
        tree = torch.empty(tsz, dtype=torch.int32, device=dev)
        itree = torch.empty_like(tree)
        L.check(lib.stwo_precompute_twiddles(hc.initial_index, hc.step_size, hc.log_size, tree.data_ptr(),
                                             itree.data_ptr(), sptr))
        src = [torch.randint(0, P, (1 << lg,), dtype=torch.int64, device=dev).to(torch.int32) for _ in range(4)]
        bufs = [[torch.empty(1 << l, dtype=torch.int32, device=dev) for _ in range(4)] for l in range(lg)]
        bp = [L.ptr_array([b.data_ptr() for b in bl]) for bl in bufs]
        sp = L.ptr_array([c.data_ptr() for c in src])
        alpha = L.QM31(12345, 678, 91011, 1213)

        def work():
            L.check(lib.stwo_fold_circle_into_line(sp, 1 << lg, alpha, itree.data_ptr(), 0, bp[lg - 1], sptr))
            for l in range(lg - 1, 4, -1):
                L.check(lib.stwo_fold_line(bp[l], 1 << l, alpha, itree.data_ptr(), tsz - (1 << l), bp[l - 1], sptr))
        reps = 1
    elif what == "inverse":
        n = 1 << 24
        sptr = torch.cuda.current_stream(dev).cuda_stream
        src = torch.randint(1, P, (4 * n,), dtype=torch.int64, device=dev).to(torch.int32)
        dst = torch.empty_like(src)

        def work():
            L.check(lib.stwo_batch_inverse_qm31(src.data_ptr(), dst.data_ptr(), n, sptr))
        reps = 1
    else:
        raise SystemExit(f"unknown --profile {what}")
    for _ in range(3):
        work()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    t0 = time.perf_counter()
    for _ in range(reps):
        work()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile": what, "reps": reps, "wall_ms": (time.perf_counter() - t0) * 1e3}), flush=True)
    del np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--jobs", type=int, default=48, help="jobs per step")
    ap.add_argument("--workers", type=int, default=8, help="proof server jobs in flight")
    ap.add_argument("--cpu-total-budget", type=float, default=120.0,
                    help="--impl reference: stop starting steps after this many seconds of CPU proving")
    ap.add_argument("--latency-jobs", type=int, default=2000, help="jobs per Poisson load level")
    ap.add_argument("--cpu-budget", type=float, default=20.0,
                    help="--impl reference: seconds of CPU proving per step at most (32 jobs otherwise)")
    ap.add_argument("--cpu-stream-budget", type=float, default=45.0,
                    help="seconds of CPU proving for the cpu_baseline leg at most (32 jobs otherwise)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--detail-out", default=os.path.join("bench_out", "bench_detail.json"),
                    help="where the full record goes (the printed line carries summaries)")
    ap.add_argument("--no-suite", action="store_true", help="skip the config-1 per-kernel sweep")
    ap.add_argument("--profile", default=None,
                    help="run one workload for ncu instead: fft[:LOG] | proof:L,N | merkle | merkle_tree[:COLS,LOG] | "
                         "quotients | fri | "
                         "inverse")
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
