"""Every launch shape the autotuner may pick computes the same product:
FP64 and mixed stores, one and eight vectors, against the default setting
(FP64 to 1e-13, mixed to 1e-6 relative); invalid settings are rejected; and
autotune() on a device sets a valid setting and fills its cache."""
import json

import numpy as np
import pytest

import hlr_b200 as hlr
from hlr_b200 import tune
from hlr_b200._capi import HLRC_MR_NEVER

from conftest import relerr

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-13, "mixed": 1e-6}


def run(M, X, nrhs):
    if nrhs == 1:
        x = torch.from_numpy(X[:, 0].copy()).cuda()
        y = torch.zeros(M.nrows, dtype=torch.float64, device="cuda")
    else:
        x = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().T
        y = torch.zeros((nrhs, M.nrows), dtype=torch.float64, device="cuda").T
    hlr.mul_vec(1.0, hlr.apply_normal, M, x, y)
    torch.cuda.synchronize()
    return y.cpu().numpy().reshape(M.nrows, -1)


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_all_settings_agree(c2_small, prec):
    M = hlr.upload(c2_small, precision=prec, max_nrhs=8)
    X = np.random.default_rng(5).standard_normal((c2_small.n, 8))
    ref1 = run(M, X, 1)
    ref8 = run(M, X, 8)
    for c in tune.candidates(M.tuning, 1) + [dict(tune.DEFAULT, side_at=k) for k in tune.SIDE_AT]:
        M.set_tuning(**c)
        assert M.tuning == c
        assert relerr(run(M, X, 1), ref1) <= TOL[prec], c
    M.set_tuning(**tune.DEFAULT)
    M.set_tuning(mr_min_nrhs=HLRC_MR_NEVER)      # eight vectors as eight one-vector products
    assert relerr(run(M, X, 8), ref8) <= TOL[prec]
    M.set_tuning(mr_min_nrhs=9)                   # 8 < 9: also the loop
    assert relerr(run(M, X, 8), ref8) <= TOL[prec]
    assert M.device_error() == 0
    M.free()


def test_invalid_settings_rejected(c2_small):
    M = hlr.upload(c2_small, precision="f64")
    for bad in ({"nform_warps": 6}, {"ttform_warps": 32}, {"mr_min_nrhs": 1}, {"mr_min_nrhs": HLRC_MR_NEVER + 1},
                {"overlap": 2}, {"side_at": -1}, {"side_at": 17}, {"nform_warps": 4, "side_at": 99}):
        with pytest.raises(hlr.HLRCError):
            M.set_tuning(**bad)
        assert M.tuning == tune.DEFAULT
    M.free()


def test_autotune_on_device(c2_small, tmp_path):
    M = hlr.upload(c2_small, precision="mixed", max_nrhs=8)
    path = tmp_path / "tuning.json"
    r1 = tune.autotune(M, nrhs=1, cache=path, reps=2, warmup=1)
    r8 = tune.autotune(M, nrhs=8, cache=path, reps=2, warmup=1)
    assert not r1["cached"] and not r8["cached"]
    assert len(r1["times_ms"]) == len(tune.candidates(tune.DEFAULT, 1)) + len(tune.SIDE_AT) - 1
    assert len(r8["times_ms"]) == 2
    assert all(t > 0 for _, t in r1["times_ms"] + r8["times_ms"])
    assert M.tuning["nform_warps"] in (4, 8, 16) and M.tuning["mr_min_nrhs"] in (2, HLRC_MR_NEVER)
    assert len(json.loads(path.read_text())) == 2
    M2 = hlr.upload(c2_small, precision="mixed", max_nrhs=8)
    assert tune.autotune(M2, nrhs=1, cache=path)["cached"]
    M.free()
    M2.free()
