"""Generates the golden vectors in this folder.

The reference ships no fixture for its MVM, so these pin this project's own
host construction + CPU oracle: for each small problem they store the
permutation, a seeded x, the oracle product y = op(M) x and the dense
kernel product op(A) x.  Run from the repository root:

    python tests/golden/make_golden.py [case ...]
"""
import json
import sys
from dataclasses import asdict
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import hlr_b200 as hlr  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "log1d_n1024": (hlr.Problem.log1d(1024), [0, 1], 1e-6),
    "exp3d_n2048": (hlr.Problem.exp3d(2048), [0, 1], 1e-6),
    "sphere_r3_uniform": (hlr.Problem.laplace_sphere(refine=3, uniform=True), [0, 2], 1e-6),
    "sphere_r4_h2": (hlr.Problem.laplace_sphere(refine=4, nested=True), [0, 2], 2e-6),
}


def main(names=None):
    for name, (prob, ops, tol) in CASES.items():
        if names and name not in names:
            continue
        hm = hlr.build(prob)
        x = np.random.default_rng(7).standard_normal(hm.n)
        out = {"perm": hm.perm_i2e, "x": x}
        for op in ops:
            y = np.zeros(hm.n)
            if prob.nested:
                assert oracle.h2_mvm(hm.h2_desc(), 1.0, op, x, y) == 0
            elif prob.uniform:
                assert oracle.uniform_mvm(hm.uniform_desc(), 1.0, op, x, y) == 0
            else:
                oracle.hmvm_seq(hm.h_desc(), 1.0, op, x, y)
            yd = np.zeros(hm.n)
            oracle.dense_matvec(hm, 1.0, op, x, yd)
            out[f"y_op{op}"] = y
            out[f"ydense_op{op}"] = yd
        np.savez_compressed(HERE / f"{name}.npz", **out)
        meta = {"problem": asdict(prob), "ops": ops, "nleaves": hm.nleaves, "dense_tol": tol}
        (HERE / f"{name}.json").write_text(json.dumps(meta, indent=1) + "\n")
        print(name, hm.n, hm.nleaves)


if __name__ == "__main__":
    main(sys.argv[1:])    # optional case names: regenerate only those
