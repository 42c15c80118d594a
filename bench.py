"""Benchmark of the H-matrix MVM (y += alpha A x) on B200.

Default workload (one step = one product on one GPU): FP64 H-matrix of the 3D
exponential covariance exp(-r/0.1) + 1e-4 nugget on n = 131072 points
uniform in [0,1]^3 (seed 1), BSP cluster tree leaf 64, eta = 2, ACA + SVD
eps = 1e-6, one right-hand side x ~ N(0,1).  Synthetic inputs, built by the
library's own construction (the leaves on the GPU; --host-build on the host).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2|c1|c3|c2s|c4|c5] [--precision P] [--nrhs K]
                    [--no-cpu-baseline] [--no-autotune] [--no-graph] [--h2] [--shard]
                    [--tune-plan] [--plan k=v,...] [--members N] [--host-build]
                    [--reduced bfp,mixed|none]

Prints one JSON line on rank 0.  Under torchrun (N > 1) every rank runs an
independent replica of the product on its own GPU (weak scaling), time = max
over ranks.  With --shard the ranks share one product instead: each owns a
run of rows of about equal bytes, and every step all-gathers x (strong
scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "H-MVM/s & HBM GB/s vs roofline; FP64 vs mixed-precision at rel.err ≤1e-6"

CONFIGS = {
    # name: (description, problem kwargs, uniform, precision, nrhs)
    "c1": ("FP64 H-MVM, 1D log kernel n=8192, leaf 64, eta 2, eps 1e-6, nrhs 1",
           dict(kind=0, n=8192), False, "f64", 1),
    "c2": ("FP64 H-MVM, 3D exp(-r/0.1)+1e-4 nugget, n=131072 U[0,1]^3, BSP leaf 64, eta 2, eps 1e-6, nrhs 1",
           dict(kind=1, n=131072, ell=0.1, nugget=1e-4), False, "f64", 1),
    "c2s": ("FP64 H-MVM, 3D exp(-r/0.1)+1e-4 nugget, n=32768 (profiling size), leaf 64, eta 2, eps 1e-6, nrhs 1",
            dict(kind=1, n=32768, ell=0.1, nugget=1e-4), False, "f64", 1),
    "c3": ("FP64 uniform-H MVM, 1/(4 pi r)*area on octahedron sphere refined 6x (32768 triangles), leaf 64, "
           "eta 2, eps 1e-6, nrhs 1", dict(kind=2, refine=6, uniform=True), True, "f64", 1),
    "c4": ("FP16-stored H-MVM (per-chunk power-of-two scale), 3D exp(-r/0.1)+1e-4 nugget, n=262144, leaf 64, "
           "eta 2, eps 1e-6, nrhs 64 on tensor cores", dict(kind=1, n=262144, ell=0.1, nugget=1e-4), False, "f16", 64),
}


L2_BYTES = 126 * 1024 * 1024   # B200 L2


def l2_label(stream_bytes: float) -> str:
    """How the L2 relates to the bytes a step streams: products that stream
    less than twice the L2 are labelled L2-resident (no flush between
    products, so part of the matrix may be served from L2)."""
    gb = stream_bytes / 1e9
    if stream_bytes < 2 * L2_BYTES:
        return f"L2-resident: {gb:.3f} GB streamed per step, under 2x the 126 MB L2; no flush between products"
    return f"inputs larger than L2 ({gb:.2f} GB matrix streamed per step)"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_roof(hlr, flops: float, alg_bytes: float, ms_per_product: float, hbm_peak: float, device: int) -> dict:
    """The roof of an FP64 multi-vector product: min(HBM bandwidth x
    intensity, FP64 tensor peak), the peak measured here by a DMMA loop of
    the library (hlrc_fp64_peak).  frac = achieved flop rate / that roof."""
    peak = hlr.fp64_peak(device)
    intensity = flops / alg_bytes
    roof = min(hbm_peak * 1e9 * intensity, peak * 1e12) / 1e12
    achieved = flops / (ms_per_product / 1e3) / 1e12
    return {"fp64_tflops_measured": peak, "flops_per_product": flops, "intensity_flop_per_byte": intensity,
            "roof_tflops": roof, "bound": "hbm" if roof < peak else "fp64", "achieved_tflops": achieved,
            "frac": achieved / roof}


def max_over_ranks(ms: float, world: int, device) -> float:
    """The job's time: the largest of the ranks' times.  Every rank calls it
    at the same point (one all-reduce); with one rank it returns ms."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", self.gpu_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_uuid(dev: int) -> str:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        return str(dev)


def make_problem(cfg, nthreads, h2=False):
    """Problem of a config; with h2 the same problem in H^2 form (nested
    cluster bases built from the H-matrix leaves) instead of H / uniform-H."""
    import hlr_b200 as hlr
    desc, kw, uniform, prec, nrhs = CONFIGS[cfg]
    kw = dict(kw)
    if h2:
        kw["nested"], kw["uniform"], uniform = True, False, False
        desc = desc.replace("uniform-H", "H2 (nested cluster bases)").replace("FP64 H-MVM", "FP64 H2-MVM")
    kw.setdefault("leaf_size", 64)
    kw.setdefault("eta", 2.0)
    kw.setdefault("eps", 1e-6)
    kw["nthreads"] = nthreads
    return hlr.Problem(**kw), desc, uniform, prec, nrhs


def cpu_mvm(hm, uniform, desc_obj, x, y, nthreads):
    import oracle
    from hlr_b200 import _capi
    if isinstance(desc_obj, _capi.hlrc_h2_desc):
        assert oracle.h2_mvm(desc_obj, 1.0, 0, x, y, nthreads) == 0
    elif uniform:
        st = oracle.uniform_mvm(desc_obj, 1.0, 0, x, y, nthreads)
        assert st == 0
    else:
        oracle.hmvm_chunk(desc_obj, 1.0, 0, x, y, nthreads)


def run_reference(args, rank, world):
    """CPU restatement of HLR's TBB MVM (oracle port) on the host cores."""
    if rank != 0:
        return
    import hlr_b200 as hlr
    import oracle
    nthreads = os.cpu_count() or 1
    if args.config == "c5":
        run_reference_batch(args, nthreads)
        return
    prob, desc, uniform, prec, nrhs = make_problem(args.config, nthreads, args.h2)
    hm = hlr.build(prob)
    d = hm.h2_desc() if args.h2 else (hm.uniform_desc() if uniform else hm.h_desc())
    x = np.random.default_rng(2).standard_normal(hm.n)
    y = np.zeros(hm.n)
    t0 = time.perf_counter()
    cpu_mvm(hm, uniform, d, x, y, nthreads)
    t_full = time.perf_counter() - t0
    # bound the run: a step is a sample of the leaves when K full products would exceed ~120 s
    frac = 1.0
    dd = d
    if not uniform and not args.h2 and args.steps * t_full > 120.0:
        stride = int(np.ceil(args.steps * t_full / 120.0))
        sub = [d.blocks[i] for i in range(0, d.nblocks, stride)]
        import ctypes as C
        from hlr_b200 import _capi
        arr = (_capi.hlrc_block * len(sub))(*sub)
        dd = _capi.hlrc_h_desc()
        dd.nrows, dd.ncols, dd.nblocks = d.nrows, d.ncols, len(sub)
        dd.blocks = C.cast(arr, C.POINTER(_capi.hlrc_block))
        dd._keep = (arr, d)
        sub_bytes = sum(8 * (b.nrows * b.ncols if b.kind == 0 else b.rank * (b.nrows + b.ncols)) for b in sub)
        all_bytes = sum(8 * (d.blocks[i].nrows * d.blocks[i].ncols if d.blocks[i].kind == 0 else
                             d.blocks[i].rank * (d.blocks[i].nrows + d.blocks[i].ncols)) for i in range(d.nblocks))
        frac = sub_bytes / all_bytes
    for _ in range(args.warmup):
        cpu_mvm(hm, uniform, dd, x, y, nthreads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_mvm(hm, uniform, dd, x, y, nthreads)
    el = time.perf_counter() - t0
    value = frac * args.steps / el
    sample = ("full product per step" if frac == 1.0 else
              f"every {int(round(1 / frac))}-th leaf per step ({frac * 100:.1f}% of matrix bytes), scaled")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "MVM/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "n": hm.n},
        "cpu_baseline": {"value": value, "unit": "MVM/s", "cores": nthreads, "kind": "port",
                         "sample": sample + ("; oracle/oracle.c oracle_h2_mvm_par (restated TBB hlr::h2::mul_vec, "
                                             "OpenMP tasks over subtrees)"
                                             if args.h2 else "; oracle/oracle.c oracle_hmvm_chunk (restated "
                                             "hlr::tbb::mul_vec, 64-row chunk locks, OpenMP)")},
        "e2e": {"value": value, "unit": "MVM/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_batch(args, nthreads):
    """The batched workload on the host cores: the oracle port multiplies
    each member by one vector per step.  When a full pass over the batch
    would take more than ~120 s for all steps, a step covers every k-th
    member and the rate is scaled by the matrix bytes covered."""
    import hlr_b200 as hlr
    hms = [hlr.build(p) for p in c5_problems(args.members, nthreads=nthreads)]
    rng = np.random.default_rng(9)
    xs = [rng.standard_normal(h.n) for h in hms]
    descs = [h.h_desc() for h in hms]
    nbytes = [hlr.plan_info(h)["matrix_bytes"] for h in hms]

    def step(idx):
        for i in idx:
            cpu_mvm(hms[i], False, descs[i], xs[i], np.zeros(hms[i].n), nthreads)

    t0 = time.perf_counter()
    step(range(len(hms)))
    t_full = time.perf_counter() - t0
    stride = max(1, int(np.ceil(args.steps * t_full / 120.0)))
    idx = list(range(0, len(hms), stride))
    frac = sum(nbytes[i] for i in idx) / sum(nbytes)
    for _ in range(args.warmup):
        step(idx)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(idx)
    el = time.perf_counter() - t0
    value = len(hms) * args.steps * frac / el
    sample = (f"all {len(hms)} members per step" if stride == 1 else
              f"every {stride}-th member per step ({frac * 100:.1f}% of matrix bytes), scaled")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "MVM/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "32 x 3D exp-covariance (C5 batch), one vector per member per step",
                   "members": len(hms), "n_total": sum(h.n for h in hms)},
        "cpu_baseline": {"value": value, "unit": "MVM/s", "cores": nthreads, "kind": "port",
                         "sample": sample + "; oracle/oracle.c oracle_hmvm_chunk (restated hlr::tbb::mul_vec)"},
        "e2e": {"value": value, "unit": "MVM/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def products_per_graph(steps: int) -> int:
    """Products captured in one CUDA graph: the reference times runs of
    nmvm = 50 products; here the K timed products are split into at least
    five equal runs where K allows it (each run one graph replay), so that
    every line carries a min / median / max over runs."""
    want = min(steps, 5)
    return max(d for d in range(1, min(50, steps) + 1) if steps % d == 0 and steps // d >= want)


def time_products(M, step, steps: int, warmup: int, use_graph: bool, world: int, dev, clocks_id=None):
    """Times `steps` products of handle M issued by step() on torch's current
    stream: `warmup` untimed products, then the timed region bracketed by a
    barrier and synchronisations, as replays of one CUDA graph of
    products_per_graph(steps) products (or direct launches).  The timed
    products carry no profiling events.  The per-pass profile comes from one
    more, untimed run with the handle's per-pass CUDA events (recorded as
    graph nodes when graphs are used).  Returns a dict with the region's ms,
    the per-run min / median / max per product, the pass profile, the kernels
    launched per product and the clock samples."""
    import torch
    import torch.distributed as dist
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    l0 = M.launch_count()
    step()                      # one more warm-up product, counting its launches
    torch.cuda.synchronize()
    per_product = M.launch_count() - l0
    M.set_profiling(False)
    graph, per_graph = None, 0
    if use_graph:
        per_graph = products_per_graph(steps)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(per_graph):
                step()
        graph.replay()          # untimed
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = M.launch_count()
    marks = [e0]
    with ClockSampler(clocks_id) if clocks_id is not None else _NoClocks() as clocks:
        e0.record(stream)
        if graph is not None:
            for _ in range(steps // per_graph):
                graph.replay()
                marks.append(torch.cuda.Event(enable_timing=True))
                marks[-1].record(stream)
        else:
            for _ in range(steps):
                step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = per_product * steps if graph is not None else M.launch_count() - launches0
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    runs = None
    if graph is not None:
        rt = [a.elapsed_time(b) / per_graph for a, b in zip(marks[:-1], marks[1:])]
        runs = {"min": min(rt), "median": statistics.median(rt), "max": max(rt), "runs": len(rt)}
    del graph
    # the pass profile: one untimed run with per-pass events
    M.set_profiling(True)
    M.last_profile()  # clear
    if use_graph:
        pgraph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(pgraph):
            for _ in range(per_graph):
                step()
        pgraph.replay()
        torch.cuda.synchronize()
        prof = M.last_profile()
        del pgraph
    else:
        for _ in range(max(1, min(steps, 4))):
            step()
        torch.cuda.synchronize()
        prof = M.last_profile()
    M.set_profiling(False)
    return {"ms": ms, "runs": runs, "prof": prof, "per_product": per_product, "launches": launches,
            "per_graph": per_graph, "clocks": clocks.summary()}


class _NoClocks:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False

    def summary(self):
        return None


def reduced_arms(hlr, hm, x, n, alpha, args, world, dev, y_oracle, v64, peak):
    """The mixed-precision half of the metric on the same matrix and x: the
    block floating point store (24/16-bit, VALR bit rates) and the VALR mixed
    FP32/FP16 store, each timed like the FP64 arm, with its error against
    the oracle's FP64 product and its speed-up over the FP64 GPU product."""
    import torch
    hbm_peak, peak_kind = peak
    out = {}
    for prec in args.reduced:
        plan_times = None
        if args.no_autotune:
            Mr = hlr.upload(hm, precision=prec, max_nrhs=1, plan=args.plan)
        else:   # the near field beside the low-rank passes or fused, as for the FP64 line
            from hlr_b200.tune import autotune_plan
            Mr, pt = autotune_plan(lambda p: hlr.upload(hm, precision=prec, max_nrhs=1, plan=dict(args.plan, **p)),
                                   nrhs=1, knobs=("near_field",), graph=not args.no_graph)
            plan_times = pt["times_ms"]
        tuned = tune_handle(Mr, 1, args)
        if tuned is not None:
            tuned = dict(tuned, plan=Mr.plan or "defaults", plan_times_ms=plan_times)
        yr = torch.zeros(n, dtype=torch.float64, device=dev)
        r = time_products(Mr, lambda: hlr.mul_vec(alpha, hlr.apply_normal, Mr, x, yr), args.steps, args.warmup,
                          not args.no_graph, world, dev, gpu_uuid(dev.index))
        yr.zero_()
        hlr.mul_vec(1.0, hlr.apply_normal, Mr, x, yr)
        torch.cuda.synchronize()
        yh = yr.cpu().numpy()
        ms_max = max_over_ranks(r["ms"], world, dev)
        value = world * args.steps / (ms_max / 1e3)
        info = Mr.info
        arm = {"value": value, "unit": "MVM/s", "ms_per_step": ms_max / args.steps,
               "ms_per_product_of_runs": r["runs"], "speedup_vs_fp64": (value / world) / v64,
               "matrix_bytes": info["matrix_bytes"], "algorithmic_bytes": info["algorithmic_bytes"],
               "hbm_gbs": info["algorithmic_bytes"] / (ms_max / 1e3 / args.steps) / 1e9,
               "roofline": roofline_from_profile(r["prof"], hbm_peak, peak_kind, args.config + "/" + prec),
               "gpu_launches": r["launches"], "tuning": tuned, "clocks": r["clocks"]}
        if y_oracle is not None:
            arm["rel_err_vs_oracle"] = float(np.linalg.norm(yh - y_oracle) / np.linalg.norm(y_oracle))
        out[prec] = arm
        Mr.free()
        del yr
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import hlr_b200 as hlr

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ncpu = os.cpu_count() or 1
    nthreads = max(1, ncpu // max(1, int(os.environ.get("LOCAL_WORLD_SIZE", world))))
    prob, desc, uniform, prec, nrhs = make_problem(args.config, nthreads, args.h2)
    if args.precision:
        prec = args.precision
        desc = desc.replace("FP64 ", f"{prec.upper()}-stored ") if prec != "f64" else desc
    if args.nrhs:
        nrhs = args.nrhs
    # leaves assembled on the GPU (dense evaluation, ACA, QR/SVD) for the H
    # configs unless --host-build; the oracle arms fetch them to the host
    # after the timed products
    prob.on_device = not args.host_build and not uniform and not args.h2
    tb = time.perf_counter()
    hm = hlr.build(prob)
    if hm.leaves_on_device and prec != "f64":
        hm.fetch()   # reduced-precision stores are planned from host leaves: one bulk copy here
    t_build = time.perf_counter() - tb
    tu = time.perf_counter()
    plan_tuned = None
    if args.tune_plan and not args.no_autotune:
        # plan-level choices: the 64-vector T-form's piece length for wide
        # 16-bit products, the finish's two-level threshold otherwise
        from hlr_b200.tune import autotune_plan
        knobs = ("piece_tiles",) if prec in ("f16", "bf16") and nrhs > 8 and not uniform and not args.h2 \
            else (("near_field", "finish_slots") if nrhs == 1 else ("finish_slots",))
        M, plan_tuned = autotune_plan(
            lambda p: hlr.upload(hm, precision=prec, uniform=uniform, max_nrhs=nrhs, h2=args.h2,
                                 plan=dict(args.plan, **p)),
            nrhs=nrhs, knobs=knobs, graph=not args.no_graph)
    else:
        M = hlr.upload(hm, precision=prec, uniform=uniform, max_nrhs=nrhs, h2=args.h2, plan=args.plan)
    t_upload = time.perf_counter() - tu
    tuned = tune_handle(M, nrhs, args)
    if tuned is not None:
        tuned = dict(tuned, plan=M.plan or "defaults",
                     plan_times_ms=plan_tuned["times_ms"] if plan_tuned else None)
    info = M.info
    n = hm.n
    # x ~ N(0,1), one column per right-hand side (column-major (n, nrhs))
    xh = np.random.default_rng(2).standard_normal((nrhs, n))

    def dev_vec(a):
        t_ = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        return t_[0] if nrhs == 1 else t_.T

    x = dev_vec(xh)
    y = dev_vec(np.zeros((nrhs, n)))
    alpha = 2.0

    def step():
        hlr.mul_vec(alpha, hlr.apply_normal, M, x, y)

    # the reference's protocol: runs of products (nmvm = 50 there); here each
    # run is one replay of a CUDA graph of captured products
    tm = time_products(M, step, args.steps, args.warmup, not args.no_graph, world, dev, gpu_uuid(local_rank))
    ms, runs, prof, timed_launches, per_graph = tm["ms"], tm["runs"], tm["prof"], tm["launches"], tm["per_graph"]
    ms_max = max_over_ranks(ms, world, dev)

    t_fetch = None
    if hm.leaves_on_device:
        tf = time.perf_counter()
        hm.fetch()
        t_fetch = time.perf_counter() - tf
    # correctness of the timed path: one product from zero; column 0 is
    # compared with the oracle below
    yc = dev_vec(np.zeros((nrhs, n)))
    hlr.mul_vec(1.0, hlr.apply_normal, M, x, yc)
    torch.cuda.synchronize()
    ygpu_all = (yc if nrhs > 1 else yc[:, None]).cpu().numpy()
    ygpu = ygpu_all[:, 0].copy()
    # the oracle's FP64 product of column 0 (the checker of every arm)
    y_oracle = None
    if world == 1 and not (args.no_cpu_baseline and not args.reduced):
        d_or = hm.h2_desc() if args.h2 else (hm.uniform_desc() if uniform else hm.h_desc())
        y_oracle = np.zeros(n)
        cpu_mvm(hm, uniform, d_or, np.ascontiguousarray(xh[0]), y_oracle, os.cpu_count() or 1)

    # the metric's reduced-precision half, on the same matrix and x: only for
    # the FP64 one-vector H-matrix line (the default)
    reduced = None
    if args.reduced and prec == "f64" and nrhs == 1 and not uniform and not args.h2:
        v64 = args.steps / (ms / 1e3)
        reduced = reduced_arms(hlr, hm, x, n, alpha, args, world, dev, y_oracle, v64, peaks())

    # reduced precision: the FP64 GPU product of the same matrix, timed the
    # same way, is the error reference and the speed-up denominator
    fp64 = None
    if prec != "f64":
        M64 = hlr.upload(hm, precision="f64", uniform=uniform, max_nrhs=nrhs, h2=args.h2)
        tune_handle(M64, nrhs, args)
        y64 = dev_vec(np.zeros((nrhs, n)))
        hlr.mul_vec(1.0, hlr.apply_normal, M64, x, y64)
        yy = dev_vec(np.zeros((nrhs, n)))
        r64 = time_products(M64, lambda: hlr.mul_vec(alpha, hlr.apply_normal, M64, x, yy), args.steps, args.warmup,
                            not args.no_graph, world, dev)
        ms64 = r64["ms"]
        y64h = (y64 if nrhs > 1 else y64[:, None]).cpu().numpy()
        fp64 = {"value": nrhs * args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps,
                "ms_per_product_of_runs": r64["runs"], "matrix_bytes": M64.info["matrix_bytes"],
                "rel_err_vs_fp64": float(np.linalg.norm(ygpu_all - y64h) / np.linalg.norm(y64h))}
        M64.free()
        del yy, y64

    # end to end through the C ABI with pinned host buffers (copies inside)
    xp = torch.from_numpy(xh.copy()).pin_memory()
    yp = torch.zeros((nrhs, n), dtype=torch.float64).pin_memory()
    xpn, ypn = xp.numpy(), yp.numpy()
    if nrhs == 1:
        xpn, ypn = xpn[0], ypn[0]
    else:  # (n, nrhs) Fortran-ordered views of the pinned (nrhs, n) buffers
        xpn, ypn = xpn.T, ypn.T
    for _ in range(max(1, args.warmup // 2)):
        hlr.mul_vec(alpha, hlr.apply_normal, M, xpn, ypn)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ksteps = args.steps
    h0.record()
    for _ in range(ksteps):
        hlr.mul_vec(alpha, hlr.apply_normal, M, xpn, ypn)
    h1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(h0.elapsed_time(h1), world, dev)
    if world > 1:
        dist.barrier()
    if rank != 0:
        return

    hbm_peak, peak_kind = peaks()
    # every right-hand side counts as one matrix-vector product
    value = world * args.steps * nrhs / (ms_max / 1e3)
    # HLR's mul_vec_datasize for nrhs vectors: the matrix once, the vectors
    # (x read, y read and written) once per right-hand side
    alg = info["algorithmic_bytes"] + (nrhs - 1) * 2 * 8 * (info["n_rows"] + info["n_cols"])
    gbs = alg / (ms_max / 1e3 / args.steps) / 1e9
    # the summaries key a workload as config[/precision][/nrhs]
    wl = (args.config + ("/h2" if args.h2 else "") + ("" if prec == "f64" else "/" + prec)
          + ("" if nrhs == 1 else f"/{nrhs}"))
    roof = roofline_from_profile(prof, hbm_peak, peak_kind, wl)
    line = {
        "metric": METRIC, "value": value, "unit": "MVM/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == "f64" else prec, "data": "synthetic",
        "config": {"workload": desc, "n": n, "nrhs": nrhs, "precision": prec, "parallelism": f"replicas x{world}",
                   "l2": l2_label(info["matrix_bytes"]),
                   "matrix_bytes": info["matrix_bytes"], "algorithmic_bytes": alg, "flops": info["flops"],
                   "leaves": info["n_dense"] + info["n_lowrank"], "max_rank": info["max_rank"],
                   "construction": "device" if prob.on_device else "host",
                   "build_s": round(t_build, 2), "upload_s": round(t_upload, 2),
                   "fetch_s": round(t_fetch, 2) if t_fetch is not None else None, "tuning": tuned,
                   "graph": {"products_per_graph": per_graph, "replays": args.steps // per_graph,
                             "ms_per_product_of_runs": runs} if per_graph else None},
        "hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak, "peak_kind": peak_kind,
        "roofline": roof,
        "compute_roof": fp64_roof(hlr, info["flops"] * nrhs, alg, ms_max / args.steps, hbm_peak, local_rank)
        if prec == "f64" and nrhs > 1 else None,
        "passes": {k: {"launches": v[0], "avg_ms": v[1] / max(1, v[0]), "bytes_per_launch": v[2]}
                   for k, v in prof.items()},
        "gpu_launches": timed_launches,
        "e2e": {"value": world * ksteps * nrhs / (e2e_ms / 1e3), "unit": "MVM/s",
                "h2d_bytes_per_step": 2 * 8 * n * nrhs, "d2h_bytes_per_step": 8 * n * nrhs},
        "clocks": tm["clocks"],
    }
    if reduced is not None:
        line["reduced"] = reduced
    if fp64 is not None:
        fp64["speedup"] = (value / world) / fp64["value"]
        line["fp64_gpu"] = fp64
    # CPU baseline (oracle port on the host cores, bounded sample) and error
    if not args.no_cpu_baseline and world == 1:
        d = hm.h2_desc() if args.h2 else (hm.uniform_desc() if uniform else hm.h_desc())
        ncores = os.cpu_count() or 1
        line["rel_err_vs_oracle"] = float(np.linalg.norm(ygpu - y_oracle) / np.linalg.norm(y_oracle))
        reps, el = 0, 0.0
        budget = 15.0
        while el < budget and reps < 50:
            yy = np.zeros(n)
            t0 = time.perf_counter()
            cpu_mvm(hm, uniform, d, np.ascontiguousarray(xh[0]), yy, ncores)
            el += time.perf_counter() - t0
            reps += 1
        line["cpu_baseline"] = {"value": reps / el, "unit": "MVM/s", "cores": ncores, "kind": "port",
                                "sample": f"{reps} full products of the same matrix and x after 1 warm-up "
                                          f"({el:.1f} s); oracle/oracle.c restatement of "
                                          + ("the TBB hlr::h2::mul_vec (OpenMP tasks)" if args.h2
                                             else "hlr::tbb::mul_vec")}
    print(json.dumps(line), flush=True)


def c5_problems(count=32, seed=5, nthreads=0):
    """The batched workload: count 3D exponential-covariance matrices with
    ell ~ U[0.05, 0.2], n log-uniform in [4096, 65536] (numpy default_rng(seed),
    ell drawn before n for each member), U[0,1]^3 points with seed 1000 + i,
    nugget 1e-4, leaf 64, eta 2, eps 1e-6."""
    import hlr_b200 as hlr
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(count):
        ell = float(rng.uniform(0.05, 0.2))
        n = int(round(np.exp(rng.uniform(np.log(4096), np.log(65536)))))
        probs.append(hlr.Problem.exp3d(n, ell=ell, nugget=1e-4, seed=1000 + i, nthreads=nthreads))
    return probs


def run_batch(args, rank, world, local_rank):
    """C5: all members in one batched handle.  Timed: batched products with
    8 right-hand sides in the inner precision (the headline), the same in
    FP64, and the FP64 single-vector drop-in product; then the error of the
    inner product against FP64, an end-to-end run from pinned host buffers,
    and one CG solve with FP64 iterative refinement to 1e-10."""
    import torch

    import hlr_b200 as hlr
    from hlr_b200.solve import cg_refine

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nrhs = args.nrhs or 8
    inner = args.precision or "mixed"
    count = args.members
    tb = time.perf_counter()
    probs = c5_problems(count, nthreads=os.cpu_count() or 0)
    for p in probs:
        p.on_device = not args.host_build
    # the FP64 store is gathered on the device; the leaves are then fetched
    # to the host (one bulk copy per member) for the reduced-precision store
    hms = [hlr.build(p) for p in probs]
    t_build = time.perf_counter() - tb
    pad = (max(h.n for h in hms) + 63) // 64 * 64
    plan64 = planlow = None
    if args.tune_plan and not args.no_autotune:
        # the two-level finish threshold, per store (many small multi-tile outputs)
        from hlr_b200.tune import autotune_plan
        A64, plan64 = autotune_plan(lambda p: hlr.upload_batch(hms, precision="f64", max_nrhs=nrhs, pad_to=pad,
                                                               plan=dict(args.plan, **p)),
                                    nrhs=nrhs, knobs=("near_field", "finish_slots"))
        if inner == "f64":
            Alow = A64
        else:
            for h in hms:
                h.fetch()
            Alow, planlow = autotune_plan(
                lambda p: hlr.upload_batch(hms, precision=inner, max_nrhs=nrhs, pad_to=pad, plan=dict(args.plan, **p)),
                nrhs=nrhs, knobs=("near_field", "finish_slots"))
    else:
        A64 = hlr.upload_batch(hms, precision="f64", max_nrhs=nrhs, pad_to=pad, plan=args.plan)
        if inner != "f64":
            for h in hms:
                h.fetch()
        Alow = A64 if inner == "f64" else hlr.upload_batch(hms, precision=inner, max_nrhs=nrhs, pad_to=pad,
                                                           plan=args.plan)
    tuned64 = tune_handle(A64, nrhs, args)
    tuned = tune_handle(Alow, nrhs, args) if Alow is not A64 else tuned64
    if tuned is not None:
        tuned = dict(tuned, plan=Alow.plan or "defaults", plan_times_ms=planlow["times_ms"] if planlow else None)
    if tuned64 is not None:
        tuned64 = dict(tuned64, plan=A64.plan or "defaults", plan_times_ms=plan64["times_ms"] if plan64 else None)
    N = count * pad
    rng = np.random.default_rng(9)
    b = np.zeros((nrhs, N))
    for i, h in enumerate(hms):
        b[:, i * pad:i * pad + h.n] = rng.standard_normal((nrhs, h.n))
    bt = torch.from_numpy(b).to(dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(M, x, y, steps):
        for _ in range(args.warmup):
            hlr.mul_vec(1.0, hlr.apply_normal, M, x, y)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = M.launch_count()
        e0.record(stream)
        for _ in range(steps):
            hlr.mul_vec(1.0, hlr.apply_normal, M, x, y)
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), world, dev), M.launch_count() - l0

    y = torch.zeros_like(bt)
    with ClockSampler(gpu_uuid(local_rank)) as clocks:
        ms, launches = timed(Alow, bt.T, y.T, args.steps)
    # the pass profile: a few more products with per-pass events, untimed
    Alow.set_profiling(True)
    Alow.last_profile()  # clear
    timed(Alow, bt.T, y.T, min(args.steps, 4))
    prof = Alow.last_profile()
    Alow.set_profiling(False)
    y64 = torch.zeros_like(bt)
    ms64, _ = timed(A64, bt.T, y64.T, args.steps)
    y1 = torch.zeros(N, dtype=torch.float64, device=dev)
    ms64_1, _ = timed(A64, bt[0], y1, args.steps)
    # error of the inner product against FP64, per member and right-hand side
    y.zero_()
    y64.zero_()
    hlr.mul_vec(1.0, hlr.apply_normal, Alow, bt.T, y.T)
    hlr.mul_vec(1.0, hlr.apply_normal, A64, bt.T, y64.T)
    torch.cuda.synchronize()
    d = (y - y64).view(nrhs, count, pad).norm(dim=2)
    r = y64.view(nrhs, count, pad).norm(dim=2)
    rel_err = float((d / r).max())
    # end to end from pinned host buffers (copies inside the timed region)
    xp = torch.from_numpy(b.copy()).pin_memory()
    yp = torch.zeros((nrhs, N), dtype=torch.float64).pin_memory()
    xpn, ypn = xp.numpy().T, yp.numpy().T
    for _ in range(max(1, args.warmup // 2)):
        hlr.mul_vec(1.0, hlr.apply_normal, Alow, xpn, ypn)
    torch.cuda.synchronize()
    barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record()
    for _ in range(args.steps):
        hlr.mul_vec(1.0, hlr.apply_normal, Alow, xpn, ypn)
    h1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(h0.elapsed_time(h1), world, dev)
    # one full solve
    torch.cuda.synchronize()
    ts = time.perf_counter()
    res = cg_refine(A64, Alow, bt, count, pad, tol=1e-10, inner_rtol=1e-7 if inner != "f64" else 1e-11,
                    max_outer=12, max_inner=20000, check_every=25)
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - ts
    if rank != 0:
        return
    hbm_peak, peak_kind = peaks()
    per_step = ms / 1e3 / args.steps
    value = world * nrhs * count / per_step
    v64 = nrhs * count / (ms64 / 1e3 / args.steps)
    v64_1 = count / (ms64_1 / 1e3 / args.steps)
    # mul_vec_datasize for nrhs vectors: the matrix once, x and y per vector
    gbs = (Alow.info["matrix_bytes"] + nrhs * 2 * 8 * 2 * N) / per_step / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "MVM/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": inner, "data": "synthetic",
        "config": {"workload": f"{count} x 3D exp-covariance (ell~U[0.05,0.2], n log-uniform [4096,65536], "
                               f"nugget 1e-4, eps 1e-6) batched in one handle, {nrhs} RHS each, inner storage "
                               f"{inner}, CG + FP64 refinement to 1e-10",
                   "members": count, "n_total": sum(h.n for h in hms), "pad": pad, "nrhs": nrhs,
                   "matrix_bytes_inner": Alow.info["matrix_bytes"], "matrix_bytes_f64": A64.info["matrix_bytes"],
                   "construction": "host" if args.host_build else "device",
                   "build_s": round(t_build, 1), "l2": l2_label(Alow.info["matrix_bytes"]),
                   "tuning": tuned, "tuning_f64": tuned64},
        "hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak, "peak_kind": peak_kind,
        "roofline": roofline_from_profile(prof, hbm_peak, peak_kind,
                                          "c5" + ("" if inner == "f64" else "/" + inner) + f"/{nrhs}"),
        "passes": {k: {"launches": v[0], "avg_ms": v[1] / max(1, v[0]), "bytes_per_launch": v[2]}
                   for k, v in prof.items()},
        "rel_err_vs_fp64": rel_err,
        "fp64_gpu": {"value": v64, "ms_per_step": ms64 / args.steps, "speedup": value / world / v64,
                     "note": "same batch, same right-hand sides, FP64 store"},
        "fp64_dropin": {"value": v64_1, "ms_per_step": ms64_1 / args.steps, "speedup": value / world / v64_1,
                        "note": "FP64 store, one right-hand side per product (the hlr::cuda::mvm drop-in)"},
        "solve": {"seconds": t_solve, "outer_iterations": res.outer_iterations,
                  "inner_iterations": res.inner_iterations, "history": res.history,
                  "systems": int(res.converged.numel()), "converged": int(res.converged.sum()),
                  "max_rel_residual": float(res.rel_residual.max())},
        "gpu_launches": launches,
        "e2e": {"value": world * args.steps * nrhs * count / (e2e_ms / 1e3), "unit": "MVM/s",
                "h2d_bytes_per_step": 2 * 8 * N * nrhs, "d2h_bytes_per_step": 8 * N * nrhs},
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


SIDE_PASSES = {"nform_Dx", "h2_Dx"}   # passes launched on the side stream (hlrc_options.near_field)


def roofline_from_profile(prof: dict, hbm_peak: float, peak_kind: str, workload: str):
    """Roofline object of the dominant pass of a per-pass CUDA-event profile
    {name: (launches, total ms, bytes/launch)}: the pass that moves the most
    bytes (for the H and uniform-H products also the one with the largest
    time; for H^2 the leaf pass rather than a level of small transfers).
    achieved = algorithmic bytes per launch / average launch time."""
    if not prof:
        return None
    name, (cnt, tot_ms, by) = max(prof.items(), key=lambda kv: kv[1][0] * kv[1][2])
    avg_ms = tot_ms / max(1, cnt)
    achieved = by / (avg_ms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "traffic": traffic_from_profiles(name, workload), "peak_kind": peak_kind,
            "bytes_per_launch": by, "avg_ms": avg_ms, "share_of_step": tot_ms / sum(v[1] for v in prof.values()),
            # the near field on the side stream shares HBM with the low-rank
            # passes while its events run: its fraction is a lower bound
            "beside_other_passes": name in SIDE_PASSES}


def run_shard(args, rank, world, local_rank):
    """--shard: one product over all ranks.  The rows are cut into runs of
    about equal stored bytes (hlr_b200.dist.row_cuts); each rank uploads its
    shard and owns the matching slices of x and y.  A step all-gathers x and
    multiplies the shard, so the exchange is inside the timed region; value
    is whole products per second (strong scaling).  The check compares the
    sharded product with the whole matrix's product on the same GPU."""
    import torch
    import torch.distributed as dist

    import hlr_b200 as hlr
    from hlr_b200 import dist as hdist

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ncpu = os.cpu_count() or 1
    nthreads = max(1, ncpu // max(1, int(os.environ.get("LOCAL_WORLD_SIZE", world))))
    prob, desc, uniform, prec, _ = make_problem(args.config, nthreads)
    if uniform or args.h2 or args.config == "c5":
        raise SystemExit("--shard takes the H-matrix configs (c1, c2, c2s, c4)")
    if args.precision:
        prec = args.precision
    tb = time.perf_counter()
    hm = hlr.build(prob)
    t_build = time.perf_counter() - tb
    n = hm.n
    cuts = hdist.row_cuts(hm, world)
    sh = hdist.RowShards(cuts, rank, world)
    M = hdist.upload_shard(hm, cuts, rank, precision=prec)
    tuned = tune_handle(M, 1, args)
    xh = np.random.default_rng(2).standard_normal(n)
    x_local = torch.from_numpy(xh[sh.r0:sh.r1].copy()).to(dev)
    y_local = torch.zeros(sh.r1 - sh.r0, dtype=torch.float64, device=dev)

    def local(a, op, xx, yy):
        hlr.mul_vec(a, op, M, xx, yy)

    def step():
        sh.mul_vec(2.0, hlr.apply_normal, local, x_local, y_local)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = M.launch_count()
    with ClockSampler(gpu_uuid(local_rank)) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    launches = M.launch_count() - launches0
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, dev)

    # check: the sharded product against the whole matrix's product
    Mf = hlr.upload(hm, precision=prec)
    yfull = torch.zeros(n, dtype=torch.float64, device=dev)
    hlr.mul_vec(1.0, hlr.apply_normal, Mf, torch.from_numpy(xh).to(dev), yfull)
    y1 = torch.zeros_like(y_local)
    sh.mul_vec(1.0, hlr.apply_normal, local, x_local, y1)
    torch.cuda.synchronize()
    ref = yfull[sh.r0:sh.r1]
    err_num = torch.tensor([float(torch.linalg.norm(y1 - ref)) ** 2, float(torch.linalg.norm(ref)) ** 2],
                           dtype=torch.float64, device=dev)
    Mf.free()
    del yfull
    if world > 1:
        dist.all_reduce(err_num)
    err = float(err_num[0].sqrt() / err_num[1].sqrt()) if float(err_num[1]) > 0 else 0.0

    # e2e: this rank's x slice from pinned host memory, the product, y slice back
    xp = torch.from_numpy(xh[sh.r0:sh.r1].copy()).pin_memory()
    yp = torch.empty(sh.r1 - sh.r0, dtype=torch.float64).pin_memory()

    def e2e_step():
        x_local.copy_(xp, non_blocking=True)
        y_local.zero_()
        step()
        yp.copy_(y_local, non_blocking=True)

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    h1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(h0.elapsed_time(h1), world, dev)
    info = M.info
    sizes = torch.tensor([info["algorithmic_bytes"], sh.r1 - sh.r0], dtype=torch.float64, device=dev)
    all_sizes = [torch.zeros_like(sizes) for _ in range(world)]
    if world > 1:
        dist.all_gather(all_sizes, sizes)
    else:
        all_sizes = [sizes]
    if world > 1:
        dist.barrier()
    if rank != 0:
        return
    hbm_peak, peak_kind = peaks()
    alg0 = info["algorithmic_bytes"]
    achieved = alg0 / (ms / args.steps / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": args.steps / (ms_max / 1e3), "unit": "MVM/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64" if prec == "f64" else prec, "data": "synthetic",
        "config": {"workload": desc + ", rows sharded over the ranks", "n": n, "nrhs": 1, "precision": prec,
                   "parallelism": f"row shards x{world}", "cuts": cuts,
                   "shard_algorithmic_bytes": [int(t[0]) for t in all_sizes],
                   "l2": l2_label(min(int(t[0]) for t in all_sizes)) + " (smallest shard)",
                   "exchange": {"op": "all_gather of x" if world > 1 else "none", "bytes_per_step": 8 * n},
                   "build_s": round(t_build, 2), "tuning": tuned},
        "roofline": {"bound": "hbm", "kernel": "rank 0 shard, whole step (exchange included)",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": None, "peak_kind": peak_kind, "bytes_per_launch": alg0,
                     "avg_ms": ms / args.steps},
        "gpu_launches": launches,
        "e2e": {"value": args.steps / (e2e_ms / 1e3), "unit": "MVM/s",
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "rel_err_vs_unsharded": err,
        "cpu_baseline": None,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


def tune_handle(M, nrhs: int, args):
    """Launch shapes from the autotuner, before any timed region: warps per
    CTA for one vector, then (nrhs > 1) the 8-vector kernels against a loop
    of one-vector products.  No cache file: each run times its own device,
    in CUDA graph replays unless the products are timed without graphs."""
    if args.no_autotune:
        return None
    from hlr_b200.tune import autotune
    autotune(M, nrhs=1, cache=None, graph=not args.no_graph)
    if nrhs > 1:
        autotune(M, nrhs=nrhs, cache=None, graph=not args.no_graph)
    return M.tuning


def traffic_from_profiles(kernel: str, config: str):
    """DRAM bytes per launch of `kernel` from a committed ncu summary table
    row `| kernel | workload | bytes |` in profiles/*.md, if any; the
    workload is the config, then /h2 for the H^2 form, then /precision unless
    FP64, then /nrhs unless 1 (e.g. c2, c2/mixed, c2/mixed/8, c3/h2)."""
    for p in sorted((ROOT / "profiles").glob("*.md")):
        for ln in p.read_text().splitlines():
            parts = [s.strip() for s in ln.strip().strip("|").split("|")]
            if len(parts) == 3 and parts[0] == kernel and parts[1] == config:
                try:
                    return float(parts[2])
                except ValueError:
                    return None
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS) + ["c5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--no-graph", action="store_true", help="launch every product directly (no CUDA graph)")
    ap.add_argument("--h2", action="store_true", help="the config's problem in H2 form (nested cluster bases)")
    ap.add_argument("--precision", default=None, choices=["f64", "f32", "bf16", "f16", "mixed", "bfp"],
                    help="storage precision (default: the config's)")
    ap.add_argument("--nrhs", type=int, default=None, help="right-hand sides per product (default: the config's)")
    ap.add_argument("--shard", action="store_true",
                    help="one product over all ranks: rows sharded, x all-gathered per step (strong scaling)")
    ap.add_argument("--tune-plan", action="store_true", default=None,
                    help="also tune plan-level choices by re-uploading (default: on for c1, c4 and c5)")
    ap.add_argument("--members", type=int, default=32,
                    help="c5: the first N members of the batch (32, the workload; fewer for profiling)")
    ap.add_argument("--plan", default="", help="plan-level choices k=v[,k=v] (finish_slots, piece_tiles, "
                    "near_field), before any plan tuning")
    ap.add_argument("--host-build", action="store_true",
                    help="assemble the leaves on the host (default: on the GPU for the H-matrix configs)")
    ap.add_argument("--reduced", default="bfp,mixed",
                    help="reduced-precision stores timed beside the FP64 one-vector H-matrix line "
                         "(comma list of bfp, mixed, f32, f16, bf16; 'none' for none)")
    args = ap.parse_args()
    args.reduced = [] if args.reduced in ("", "none") else args.reduced.split(",")
    args.plan = {k: int(v) for k, v in (kv.split("=") for kv in args.plan.split(",") if kv)}
    if args.tune_plan is None:
        args.tune_plan = args.config in ("c1", "c4", "c5")
    args.warmup = max(3, args.warmup)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.shard:
            run_shard(args, rank, world, local_rank)
        elif args.config == "c5":
            run_batch(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
