"""Writes bayesian-rans-uq_b200/data/channel_truth.json: the noise-free synthetic observed profile of each
Re_tau class of the channel ensemble -- the reference's own FP64 ForwardModel
solve at (a1, beta*) = (0.31, 0.09) on that class's mesh, sampled at the 30
stations (the stand-in for the Lee-Moser DNS profile, which is not shipped). Run where oracle/_ref is built:  python tests/golden/make_channel_truth.py
"""
import json
import multiprocessing
import sys
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import checker as ck  # noqa: E402
import rans_uq_b200.workloads as wl  # noqa: E402

def run(c):
    re_tau, ny = wl.CLASSES[c]
    x, y = wl.channel_probes(re_tau)
    case = ck.Case(ny=ny, re_tau=re_tau, nu=1 / re_tau, yplus=0.5, alpha_u=wl.ALPHA_U, tol=wl.TOL,
                   max_iter=wl.MAX_ITER, obs_x=x, obs_y=y, obs_value=np.zeros(30),
                   obs_sigma=np.ones(30)).with_theta(0.31, 0.09)
    o = ck.solve(case, "ref")
    print(c, o.status, o.iterations, flush=True)
    return {"re_tau": re_tau, "ny": ny, "status": o.status, "iterations": o.iterations,
            "profile": [float(v) for v in o.predictions]}


if __name__ == "__main__":
    # one process per class: the reference solver is not safe to run from several
    # threads of one process
    with ProcessPoolExecutor(3, mp_context=multiprocessing.get_context("spawn")) as ex:
        recs = list(ex.map(run, range(3)))
    out = {str(c): r for c, r in enumerate(recs)}
    (ROOT / "bayesian-rans-uq_b200" / "data" / "channel_truth.json").write_text(
        json.dumps(out, indent=1))
