"""Benchmark: M31 circle FFT on B200 (the BASELINE metric's "FFT % HBM peak" leg).

Workload (per GPU, weak scaling): 8 M31 columns at log_size 24 — each step
interpolates the 8 evaluations (2^24 each, in place) and evaluates the resulting
coefficients on the blowup-4 domain (2^24 coefficients -> 2^26 evaluations) with
the extension fused into the FFT. One "column" of the metric = one such
interpolate + extend-evaluate. Inputs (512 MB) and outputs (2 GB) exceed the
126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the oracle port of the reference's CPU path (CpuBackend
restated in C, oracle/stwo_oracle.c) on all host cores, one column per step.
Prints one JSON line (rank 0).
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "stwo-gpu_b200")
P = (1 << 31) - 1
METRIC = "circle FFT columns/s at log_size 24 (interpolate + blowup-4 evaluate); FFT % HBM peak in roofline.frac"
UNIT = "columns/s"


def load_package():
    if "stwo_gpu_b200" in sys.modules:
        return sys.modules["stwo_gpu_b200"]
    spec = importlib.util.spec_from_file_location(
        "stwo_gpu_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["stwo_gpu_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    return O


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
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
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
    return {"ms_per_step": ms, "value": ncols / (ms / 1e3), "unit": UNIT,
            "what": "reference CUDA library (oracle/_ref) on this GPU: interpolate_columns + extend + "
                    "evaluate_columns, same 8 x 2^24 step"}


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
    rec = {"ms": t, "gbs": b / t / 1e6, "frac_hbm": b / t / 1e6 / peak, "compressions_per_s": comp / (t / 1e3),
           "workload": "64 cols x 2^22, full tree"}
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
    rec = {"ms": t, "gbs": b / t / 1e6, "frac_hbm": b / t / 1e6 / peak, "workload": "32 cols x 2^22, 4 points"}
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
    for k, v in out.items():
        if "reference_ms" in v:
            v["speedup_vs_reference"] = v["reference_ms"] / v["ms"]
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    O = load_oracle()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline(O, args.log_size, args.log_blowup, threads)
    times = [cpu_baseline(O, args.log_size, args.log_blowup, threads) for _ in range(args.steps)]
    per_col = sum(times) / len(times)
    value = 1.0 / per_col
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_col * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "m31 (u32)", "data": "synthetic (seeded uniform M31)",
        "config": {"workload": f"1 column at log_size {args.log_size}: interpolate + evaluate blowup "
                               f"{1 << args.log_blowup} (CPU sample of the 8-column GPU step)",
                   "columns": 1, "log_size": args.log_size, "log_blowup": args.log_blowup},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"1 column of 2^{args.log_size} per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stwo = load_package()
    L = stwo._lib
    lib = L.lib()
    ncols, lg, lb = args.cols, args.log_size, args.log_blowup
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

    launches_per_step = 4  # 2 passes interpolate + 2 passes evaluate (log 24, 8 columns)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        interp()
        extend_eval()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        start.record(stream)
        for e0, e1, e2 in ev:
            e0.record(stream)
            interp()
            e1.record(stream)
            extend_eval()
            e2.record(stream)
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    total_ms = start.elapsed_time(end)
    t_interp = sum(a.elapsed_time(b) for a, b, _ in ev) / args.steps
    t_eval = sum(b.elapsed_time(c) for _, b, c in ev) / args.steps
    ms_step, value = replica_throughput(total_ms / args.steps, ncols, world, dev)

    # Roofline of the FFT kernel: algorithmic bytes = one read + one write per
    # element (interpolate: 8 B per element; evaluate: 4 B per coefficient read +
    # 4 B per evaluation written); twiddle reads are not counted.
    b_interp = ncols * (1 << lg) * 8
    b_eval = ncols * ((1 << lg) * 4 + (1 << N) * 4)
    achieved = (b_interp + b_eval) / ((t_interp + t_eval) / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    tf = os.path.join(ROOT, "profiles", "fft_traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get("dram_bytes_per_launch")

    # End to end through the C ABI with host buffers: pinned H2D of the 8 input
    # columns, interpolate, extend-evaluate, D2H of the 8 evaluated columns.
    h_in = [torch.empty(1 << lg, dtype=torch.int32, pin_memory=True) for _ in range(ncols)]
    h_out = [torch.empty(1 << N, dtype=torch.int32, pin_memory=True) for _ in range(ncols)]
    for h, d in zip(h_in, evals):
        h.copy_(d)
    e2e_steps = max(2, min(args.steps, 5))

    def e2e_step():
        for h, d in zip(h_in, evals):
            d.copy_(h, non_blocking=True)
        interp()
        extend_eval()
        for h, d in zip(h_out, outs):
            h.copy_(d, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e2.record(stream)
    torch.cuda.synchronize()
    e2e_ms, e2e_value = replica_throughput(s2.elapsed_time(e2) / e2e_steps, ncols, world, dev)

    ref_gpu = reference_gpu_timing(args, evals, lg, lb, ncols, tw, itw, tree_size) if rank == 0 else None
    kernels = None
    if rank == 0 and world == 1 and not args.no_suite:
        del evals, outs, h_in, h_out
        torch.cuda.empty_cache()
        kernels = kernel_suite(stwo)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        O = load_oracle()
        threads = os.cpu_count() or 1
        dt = cpu_baseline(O, lg, lb, threads)
        cpu = {"value": 1.0 / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"1 column of 2^{lg}: interpolate + evaluate blowup {1 << lb} (oracle, {threads} threads)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "m31 (u32)", "data": "synthetic (seeded uniform M31)",
            "config": {"workload": f"{ncols} columns x log_size {lg}: interpolate + extend-evaluate blowup {1 << lb}",
                       "columns_per_gpu": ncols, "log_size": lg, "log_blowup": lb,
                       "l2": "inputs 512 MB + outputs 2 GB > 126 MB L2 (no flush needed)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "kernel": "fft_pass_kernel (interpolate + evaluate transforms)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "interpolate_ms": t_interp, "evaluate_ms": t_eval,
                         "algorithmic_bytes_per_step": b_interp + b_eval},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": ncols * (1 << lg) * 4,
                    "d2h_bytes_per_step": ncols * (1 << N) * 4, "ms_per_step": e2e_ms},
            "reference_gpu": ref_gpu,
            "kernels": kernels,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    del np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cols", type=int, default=8)
    ap.add_argument("--log-size", type=int, default=24)
    ap.add_argument("--log-blowup", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-suite", action="store_true", help="skip the config-1 per-kernel sweep")
    args = ap.parse_args()
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
