"""Writes tests/golden/ensemble_iterations.json: the outer iterations and verdict of
every draw of the 256-draw channel ensemble (seed 20261010, Re_tau 182/550/1000 on
3 x 128/256/512 cells, alpha_U 0.8, tol 1e-8, cap 300000) as the FP64 GPU path
counts them. bench.py --impl reference multiplies these by the reference solver's
measured per-iteration times to extrapolate its whole-ensemble figure (a converged
Re_tau 1000 draw takes about ten CPU minutes, so the reference is not run to the end
on every draw). Needs a GPU; about 150 s.

    python tests/golden/make_ensemble_iterations.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def main():
    import rans_uq_b200 as rq
    import rans_uq_b200.workloads as wl

    ens = wl.channel_ensemble(256)
    res = rq.evaluate_multi(ens.batches, ens.cls, ens.theta)
    out = {"what": "outer iterations per draw of the 256-draw channel ensemble, FP64 GPU path",
           "seed": wl.SEED, "alpha_u": wl.ALPHA_U, "tol": wl.TOL, "max_iter": wl.MAX_ITER,
           "iterations": [int(r.result.simple_iters) for r in res.rows],
           "status": [r.result.status.name for r in res.rows]}
    path = Path(__file__).with_name("ensemble_iterations.json")
    path.write_text(json.dumps(out, indent=0) + "\n")
    print(f"wrote {path}: {np.bincount(ens.cls)} draws per class")


if __name__ == "__main__":
    main()
