"""Autotuner for the launch shapes of a device matrix's products.

For one matrix, right-hand-side count and operation, ``autotune`` times the
candidate settings of ``hlrc_tuning`` on the current device and keeps the
fastest:

* one vector: warps per CTA (4, 8 or 16) of the N-form and of the tile
  T-form kernels, nine combinations;
* several vectors: the 8-vector tensor-core kernels against a loop of
  one-vector products (``mr_min_nrhs`` 2 or ``HLRC_MR_NEVER``); with more
  than 8 vectors also the one-pass 64-vector kernels of 16-bit stores
  (``wide_min_nrhs`` 9 or ``HLRC_MR_NEVER``).

Each candidate runs ``warmup`` untimed products and then at least ``reps``
products (enough to last 20 ms) timed with CUDA events on the launching
stream, on private random vectors (the caller's vectors are not touched).
The candidates are swept twice, interleaved, and each keeps its best time.
The default setting is kept unless another one is faster by more than
``keep_default_within`` (2 %), so timing noise does not flip the choice.
Winners are cached in a JSON file keyed by the device name and the matrix's
signature (kind, precision, shape, stored bytes, leaf counts, vector count,
operation); a later call for the same signature takes the cached setting
without timing anything.

The reference has no counterpart: its TBB products have no launch shapes.
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Callable, Optional

from ._capi import HLRC_MR_NEVER

DEFAULT = {"nform_warps": 8, "ttform_warps": 8, "mr_min_nrhs": 2, "wide_min_nrhs": 9, "overlap": 1, "side_at": 0}
# one vector, second phase at the chosen launch shapes: where the near
# field's side pass is forked (a handle without one times the same for all)
SIDE_AT = (0, 1, 2, 3)


def default_cache_path() -> Path:
    """``$HLRC_TUNING_CACHE``, else ``~/.cache/hlr_b200/tuning.json``."""
    env = os.environ.get("HLRC_TUNING_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "hlr_b200" / "tuning.json"


def signature(M, nrhs: int, op: int, device_name: str) -> str:
    i = M.info
    kind = ("h", "uniform", "h2")[int(i.get("kind", 1 if M.uniform else 0))]
    return "|".join(str(v) for v in (device_name, kind, i["precision"], i["n_rows"], i["n_cols"], i["matrix_bytes"],
                                      i["n_dense"], i["n_lowrank"], nrhs, op))


def candidates(current: dict, nrhs: int) -> list:
    """Settings to time; the first is the default for this vector count."""
    if nrhs <= 1:
        return [dict(current, nform_warps=a, ttform_warps=b) for a in (8, 4, 16) for b in (8, 4, 16)]
    if nrhs <= 8:
        return [dict(current, mr_min_nrhs=2), dict(current, mr_min_nrhs=HLRC_MR_NEVER)]
    return [dict(current, wide_min_nrhs=9, mr_min_nrhs=2), dict(current, wide_min_nrhs=HLRC_MR_NEVER, mr_min_nrhs=2),
            dict(current, wide_min_nrhs=HLRC_MR_NEVER, mr_min_nrhs=HLRC_MR_NEVER)]


def _load(path: Path) -> dict:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(path: Path, key: str, entry: dict) -> None:
    d = _load(path)
    d[key] = entry
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(path.name + f".tmp{os.getpid()}")
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def event_timer(M, nrhs: int, op: int, reps: int = 5, warmup: int = 2, min_ms: float = 20.0,
                graph: bool = False) -> Callable[[], float]:
    """Returns a function timing one product of M (ms per product) with the
    handle's current setting, on private random device vectors.  A timed run
    covers ``reps`` products, or more if needed to last ``min_ms``.  With
    ``graph`` the products are captured into a CUDA graph and its replay is
    timed: the launch cost the caller pays when it replays graphs (small
    products are otherwise bound by the host's launch rate)."""
    import torch

    from . import apply_normal, mul_vec

    dev = torch.device("cuda", torch.cuda.current_device())
    nx = M.ncols if op == apply_normal else M.nrows
    ny = M.nrows if op == apply_normal else M.ncols
    g = torch.Generator(device=dev).manual_seed(12345)
    if nrhs == 1:
        x = torch.randn(nx, dtype=torch.float64, device=dev, generator=g)
        y = torch.zeros(ny, dtype=torch.float64, device=dev)
    else:  # column-major (n, nrhs) views
        x = torch.randn((nrhs, nx), dtype=torch.float64, device=dev, generator=g).T
        y = torch.zeros((nrhs, ny), dtype=torch.float64, device=dev).T
    stream = torch.cuda.current_stream(dev)

    def timed(n: int) -> float:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if graph:
            n = min(n, 2000)
            torch.cuda.synchronize(dev)
            gr = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gr):
                for _ in range(n):
                    mul_vec(1.0, op, M, x, y)
            gr.replay()   # first replay uploads the graph
            e0.record(stream)
            gr.replay()
            e1.record(stream)
            e1.synchronize()
            del gr
            return e0.elapsed_time(e1) / n
        e0.record(stream)
        for _ in range(n):
            mul_vec(1.0, op, M, x, y)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / n

    def run() -> float:
        for _ in range(warmup):
            mul_vec(1.0, op, M, x, y)
        t = timed(reps)
        if t * reps < min_ms:
            t = timed(min(10000, int(min_ms / max(t, 1e-3)) + 1))
        return t

    return run


def autotune(M, nrhs: int = 1, op: int = 0, cache: Optional[os.PathLike] = "default", reps: int = 5,
             warmup: int = 2, keep_default_within: float = 0.02, timer: Optional[Callable[[], float]] = None,
             device_name: Optional[str] = None, sweeps: int = 2, graph: bool = False) -> dict:
    """Picks and sets the fastest launch shapes of M for ``nrhs`` vectors and
    operation ``op``.  ``cache`` is a JSON path, "default" for
    ``default_cache_path()``, or None for no cache.  ``timer`` (tests) times
    one product with the handle's current setting; by default CUDA events
    (around a CUDA graph replay with ``graph``, which is part of the key).

    Returns {"tuning": chosen setting, "times_ms": [(setting, ms), ...],
    "cached": whether the setting came from the cache, "key": cache key}."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(torch.cuda.current_device())
    path = default_cache_path() if cache == "default" else (Path(cache) if cache is not None else None)
    key = signature(M, nrhs, op, device_name) + ("|graph" if graph else "")
    if path is not None:
        hit = _load(path).get(key)
        if isinstance(hit, dict) and isinstance(hit.get("tuning"), dict):
            try:
                M.set_tuning(**hit["tuning"])
                return {"tuning": M.tuning, "times_ms": hit.get("times_ms", []), "cached": True, "key": key}
            except Exception:
                pass  # stale or foreign entry: tune afresh
    if timer is None:
        timer = event_timer(M, nrhs, op, reps=reps, warmup=warmup, graph=graph)
    start = M.tuning

    def pick(cands):
        best = [float("inf")] * len(cands)
        try:
            for _ in range(sweeps):   # interleaved sweeps; a candidate keeps its best time
                for i, c in enumerate(cands):
                    M.set_tuning(**c)
                    best[i] = min(best[i], float(timer()))
        except BaseException:
            M.set_tuning(**start)
            raise
        tm = [(dict(c), t) for c, t in zip(cands, best)]
        best_c, best_t = min(tm, key=lambda ct: ct[1])
        if tm[0][1] <= best_t * (1.0 + keep_default_within):
            best_c = tm[0][0]
        return best_c, tm

    best_c, times = pick(candidates(start, nrhs))
    if nrhs <= 1:
        best_c, t2 = pick([dict(best_c, side_at=k) for k in SIDE_AT])
        times += t2[1:]
    M.set_tuning(**best_c)
    out = {"tuning": M.tuning, "times_ms": times, "cached": False, "key": key}
    if path is not None:
        _store(path, key, {"tuning": out["tuning"], "times_ms": times})
    return out


# ------------------------------------------------------------ plan level
PLAN_CANDIDATES = {
    # tile T-form outputs with more partials than this are summed in two levels
    "finish_slots": (16, 8, 32, 64),
    # 64-vector T-form: tiles per piece of a long column cluster
    "piece_tiles": (32, 16, 8),
    # one-vector products: the near field on a side stream (0, the default)
    # or fused into the last pass (1)
    "near_field": (0, 1),
}


def autotune_plan(upload_fn: Callable[[dict], object], nrhs: int = 1, op: int = 0, knobs=("finish_slots",),
                  keep_default_within: float = 0.02, timer_for: Optional[Callable] = None, sweeps: int = 2,
                  graph: bool = False):
    """Plan-level choices, timed by uploading the matrix once per candidate.

    ``upload_fn(plan)`` uploads the matrix with hlrc_options plan choices
    ``plan`` (e.g. ``lambda p: upload(hm, precision="f16", max_nrhs=64,
    plan=p)``); each knob in ``knobs`` is tried over PLAN_CANDIDATES (the
    first value is the default), one knob at a time, the others at their
    current choice, and products are timed with CUDA events as in
    ``autotune``.  The default is kept unless another value is faster by more
    than ``keep_default_within``.  Candidates are uploaded and timed one after
    another, so that at most two handles (the best so far and the newest)
    hold device memory at once.  Returns (handle of the chosen plan,
    {"plan": choice, "times_ms": [(plan, ms), ...]}); the other handles are
    freed.  ``timer_for(M)`` (tests) replaces the event timer; ``graph``
    times CUDA graph replays, as ``event_timer``."""
    choice, times = {}, []
    best_M = None   # the handle of `choice`

    def timed(M):
        timer = timer_for(M) if timer_for is not None else event_timer(M, nrhs, op, graph=graph)
        return min(float(timer()) for _ in range(sweeps))

    for knob in knobs:
        vals = PLAN_CANDIDATES[knob]
        # the incumbent: the choice so far with the knob at its default
        # (the handle of the previous knob's choice is that plan)
        plan0 = dict(choice, **{knob: vals[0]})
        if best_M is None:
            best_M = upload_fn(plan0)
        t0 = timed(best_M)
        times.append((plan0, t0))
        best_plan, best_t, best_is_default = plan0, t0, True
        # one candidate at a time: at most two handles exist at once
        for v in vals[1:]:
            plan = dict(choice, **{knob: v})
            M = upload_fn(plan)
            t = timed(M)
            times.append((plan, t))
            if t * (1.0 + keep_default_within if best_is_default else 1.0) < best_t:
                best_M.free()
                best_M, best_plan, best_t, best_is_default = M, plan, t, False
            else:
                M.free()
        choice = dict(best_plan)
    return best_M, {"plan": choice, "times_ms": times}
