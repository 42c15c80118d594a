"""Autotuner host logic (no GPU): candidate sets, choice of the fastest
setting with the default kept inside the noise band, the JSON cache and its
reuse, and rejection of unknown settings.  A fake handle stands in for an
uploaded matrix and a fake timer for the CUDA-event timing."""
import json

import pytest

from hlr_b200 import tune
from hlr_b200._capi import HLRC_MR_NEVER


class FakeMatrix:
    uniform = False
    info = {"precision": 0, "n_rows": 4096, "n_cols": 4096, "matrix_bytes": 123456, "n_dense": 10,
            "n_lowrank": 20}

    def __init__(self):
        self._t = dict(tune.DEFAULT)
        self.sets = 0

    @property
    def tuning(self):
        return dict(self._t)

    def set_tuning(self, **kw):
        if set(kw) - set(self._t):
            raise ValueError("unknown key")
        if kw.get("nform_warps", 8) not in (4, 8, 16) or kw.get("ttform_warps", 8) not in (4, 8, 16):
            raise ValueError("bad warps")
        self._t.update(kw)
        self.sets += 1


def timer_for(M, table):
    """Time of the handle's current setting, looked up in `table`."""
    calls = []

    def t():
        s = M.tuning
        calls.append(s)
        return table(s)
    return t, calls


def test_candidates():
    one = tune.candidates(dict(tune.DEFAULT), 1)
    assert one[0] == tune.DEFAULT and len(one) == 9
    assert {(c["nform_warps"], c["ttform_warps"]) for c in one} == {(a, b) for a in (4, 8, 16) for b in (4, 8, 16)}
    many = tune.candidates(dict(tune.DEFAULT), 8)
    assert [c["mr_min_nrhs"] for c in many] == [2, HLRC_MR_NEVER]


def test_picks_fastest_and_caches(tmp_path):
    M = FakeMatrix()
    t, calls = timer_for(M, lambda s: 1.0 if s["nform_warps"] == 4 and s["ttform_warps"] == 8 else 2.0)
    path = tmp_path / "tuning.json"
    r = tune.autotune(M, nrhs=1, cache=path, timer=t, device_name="GPU-X")
    assert not r["cached"] and len(calls) == 18 + 8   # two sweeps of nine, then of the four fork points
    assert M.tuning == {"nform_warps": 4, "ttform_warps": 8, "mr_min_nrhs": 2, "wide_min_nrhs": 9, "overlap": 1,
                        "side_at": 0}
    d = json.loads(path.read_text())
    assert d[r["key"]]["tuning"] == M.tuning
    # a fresh handle of the same signature takes the cached setting untimed
    M2 = FakeMatrix()
    t2, calls2 = timer_for(M2, lambda s: 1.0)
    r2 = tune.autotune(M2, nrhs=1, cache=path, timer=t2, device_name="GPU-X")
    assert r2["cached"] and calls2 == [] and M2.tuning == M.tuning
    # another device or vector count is another key
    M3 = FakeMatrix()
    t3, calls3 = timer_for(M3, lambda s: 1.0)
    assert not tune.autotune(M3, nrhs=1, cache=path, timer=t3, device_name="GPU-Y")["cached"]
    assert not tune.autotune(M3, nrhs=8, cache=path, timer=t3, device_name="GPU-X")["cached"]
    assert len(json.loads(path.read_text())) == 3


def test_default_kept_within_noise():
    M = FakeMatrix()
    t, _ = timer_for(M, lambda s: 1.00 if s == tune.DEFAULT else 0.99)
    assert tune.autotune(M, nrhs=1, cache=None, timer=t, device_name="G")["tuning"] == tune.DEFAULT
    M = FakeMatrix()
    t, _ = timer_for(M, lambda s: 1.00 if s == tune.DEFAULT else 0.90)
    assert tune.autotune(M, nrhs=1, cache=None, timer=t, device_name="G")["tuning"] != tune.DEFAULT


def test_side_fork_point_tuned_at_the_chosen_warps():
    """One vector: the fork point of the near field's side pass is timed in
    a second phase, at the launch shapes the first phase picked."""
    M = FakeMatrix()
    t, calls = timer_for(M, lambda s: (1.0 if s["nform_warps"] == 16 else 2.0) - (0.5 if s["side_at"] == 2 else 0.0))
    r = tune.autotune(M, nrhs=1, cache=None, timer=t, device_name="G")
    assert r["tuning"]["nform_warps"] == 16 and r["tuning"]["side_at"] == 2
    assert all(c["nform_warps"] == 16 for c in calls[18:])
    assert [c["side_at"] for c in calls[18:22]] == list(tune.SIDE_AT)
    assert len(r["times_ms"]) == 9 + 3


def test_multi_vector_choice():
    M = FakeMatrix()
    t, calls = timer_for(M, lambda s: 5.0 if s["mr_min_nrhs"] == 2 else 9.0)
    r = tune.autotune(M, nrhs=8, cache=None, timer=t, device_name="G")
    assert r["tuning"]["mr_min_nrhs"] == 2 and len(calls) == 4
    M = FakeMatrix()
    t, _ = timer_for(M, lambda s: 9.0 if s["mr_min_nrhs"] == 2 else 5.0)
    assert tune.autotune(M, nrhs=3, cache=None, timer=t, device_name="G")["tuning"]["mr_min_nrhs"] == HLRC_MR_NEVER


def test_bad_cache_entries_are_retuned(tmp_path):
    path = tmp_path / "tuning.json"
    path.write_text("not json")
    M = FakeMatrix()
    t, calls = timer_for(M, lambda s: 1.0)
    r = tune.autotune(M, nrhs=1, cache=path, timer=t, device_name="G")
    assert not r["cached"] and len(calls) == 26
    d = json.loads(path.read_text())
    d[r["key"]]["tuning"] = {"nform_warps": 5, "ttform_warps": 8, "mr_min_nrhs": 2}   # rejected by the handle
    path.write_text(json.dumps(d))
    M2 = FakeMatrix()
    t2, calls2 = timer_for(M2, lambda s: 1.0)
    assert not tune.autotune(M2, nrhs=1, cache=path, timer=t2, device_name="G")["cached"] and len(calls2) == 26


def test_timer_failure_restores_setting():
    M = FakeMatrix()
    M.set_tuning(nform_warps=4)

    def boom():
        raise RuntimeError("timing failed")
    with pytest.raises(RuntimeError):
        tune.autotune(M, nrhs=1, cache=None, timer=boom, device_name="G")
    assert M.tuning["nform_warps"] == 4


def test_wide_candidates_above_eight_vectors():
    """More than 8 vectors: the 64-vector kernels, the 8-vector kernels, and
    the loop of one-vector products; the fastest wins."""
    M = FakeMatrix()
    c = tune.candidates(M.tuning, 64)
    assert [(x["wide_min_nrhs"], x["mr_min_nrhs"]) for x in c] == [(9, 2), (HLRC_MR_NEVER, 2),
                                                                   (HLRC_MR_NEVER, HLRC_MR_NEVER)]
    t, calls = timer_for(M, lambda s: 3.0 if s["wide_min_nrhs"] == HLRC_MR_NEVER and s["mr_min_nrhs"] == 2 else 6.0)
    r = tune.autotune(M, nrhs=64, cache=None, timer=t, device_name="G")
    assert r["tuning"]["wide_min_nrhs"] == HLRC_MR_NEVER and r["tuning"]["mr_min_nrhs"] == 2 and len(calls) == 6


class FakePlanned:
    """An uploaded handle whose speed depends on its plan choices."""
    def __init__(self, plan):
        self.plan = dict(plan)
        self.freed = False

    def free(self):
        self.freed = True


def test_autotune_plan_times_each_knob_and_frees_the_losers():
    made = []

    def upload_fn(plan):
        M = FakePlanned(plan)
        made.append(M)
        return M

    def ms(M):
        p = M.plan
        return 1.0 + (0.0 if p.get("finish_slots") == 8 else 0.5) + (0.0 if p.get("piece_tiles", 32) == 16 else 0.25)

    M, out = tune.autotune_plan(upload_fn, nrhs=64, knobs=("finish_slots", "piece_tiles"),
                                timer_for=lambda M: (lambda: ms(M)))
    assert out["plan"] == {"finish_slots": 8, "piece_tiles": 16}
    assert M.plan == out["plan"] and not M.freed
    assert all(m.freed for m in made if m is not M)
    assert len(out["times_ms"]) == len(tune.PLAN_CANDIDATES["finish_slots"]) + len(tune.PLAN_CANDIDATES["piece_tiles"])


def test_autotune_plan_holds_at_most_two_handles():
    """Candidates are uploaded one at a time; a loser is freed before the
    next upload, so a plan whose store takes most of the device still
    tunes."""
    live, peak = [], [0]

    class Tracked(FakePlanned):
        def __init__(self, plan):
            super().__init__(plan)
            live.append(self)
            peak[0] = max(peak[0], len(live))

        def free(self):
            super().free()
            live.remove(self)

    M, out = tune.autotune_plan(Tracked, knobs=("finish_slots", "near_field"),
                                timer_for=lambda M: (lambda: 1.0 - 0.1 * (M.plan.get("finish_slots") == 64)))
    assert out["plan"]["finish_slots"] == 64 and out["plan"]["near_field"] == 0
    assert peak[0] == 2 and live == [M]
    assert len(out["times_ms"]) == len(tune.PLAN_CANDIDATES["finish_slots"]) + len(tune.PLAN_CANDIDATES["near_field"])


def test_autotune_plan_keeps_default_within_noise():
    def upload_fn(plan):
        return FakePlanned(plan)
    M, out = tune.autotune_plan(upload_fn, knobs=("finish_slots",),
                                timer_for=lambda M: (lambda: 1.0 if M.plan["finish_slots"] == 16 else 0.995))
    assert out["plan"] == {"finish_slots": 16}
