"""Writes tests/golden/ensemble_subset_ref.npz: a seeded subset of the benchmark's own
256-draw channel ensemble (the prior-design draws of seed 20261010, draw i on Re_tau
class i mod 3) solved to its verdict by the compiled reference (oracle/_ref, the
reference's own ForwardModel) with the ensemble's settings (alpha_U 0.8, tol 1e-8,
cap 300000, the class's synthetic observation). Draws: the first 8 of Re_tau 182,
the first 4 of Re_tau 550 and the first 2 of Re_tau 1000. Stored per draw: verdict,
outer iterations, log-likelihood, the 30 probe predictions and the Ux, k, omega
fields. One process per draw; the Re_tau 1000 draws take about ten minutes each.

    python tests/golden/make_ensemble_subset.py
"""
import multiprocessing
import sys
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

SUBSET = {0: 8, 1: 4, 2: 2}


def draws():
    ids = []
    for c, count in SUBSET.items():
        ids += [i for i in range(256) if i % 3 == c][:count]
    return sorted(ids)


def solve(i):
    from oracle import checker as ck
    import rans_uq_b200.workloads as wl

    c = i % 3
    re_tau, ny = wl.CLASSES[c]
    a1, bs = wl.uniform_design([i])[0]
    x, y = wl.channel_probes(re_tau)
    observed, sigma = wl.class_observation(c)
    case = ck.Case(ny=ny, re_tau=re_tau, nu=1 / re_tau, yplus=0.5, alpha_u=wl.ALPHA_U,
                   tol=wl.TOL, max_iter=wl.MAX_ITER, obs_x=x, obs_y=y, obs_value=observed,
                   obs_sigma=sigma).with_theta(a1, bs)
    o = ck.solve(case, "ref")
    print(i, c, o.status, o.iterations, flush=True)
    return (i, c, a1, bs, o.status, o.iterations, o.loglik, o.predictions, o.field("Ux"),
            o.field("k"), o.field("omega"))


def main():
    ids = draws()
    # longest first, so the two Re_tau 1000 draws start at once
    order = sorted(ids, key=lambda i: -(i % 3))
    with ProcessPoolExecutor(max_workers=min(len(ids), multiprocessing.cpu_count()),
                             mp_context=multiprocessing.get_context("spawn")) as ex:
        res = {r[0]: r for r in ex.map(solve, order)}
    out = {"ids": np.array(ids), "cls": np.array([res[i][1] for i in ids]),
           "theta": np.array([[res[i][2], res[i][3]] for i in ids]),
           "status": np.array([res[i][4] for i in ids]),
           "iterations": np.array([res[i][5] for i in ids]),
           "loglik": np.array([res[i][6] for i in ids]),
           "predictions": np.array([res[i][7] for i in ids])}
    for c in SUBSET:
        sel = [i for i in ids if i % 3 == c]
        out[f"Ux_c{c}"] = np.array([res[i][8] for i in sel])
        out[f"k_c{c}"] = np.array([res[i][9] for i in sel])
        out[f"omega_c{c}"] = np.array([res[i][10] for i in sel])
    np.savez_compressed(Path(__file__).with_name("ensemble_subset_ref.npz"), **out)
    print("wrote ensemble_subset_ref.npz")


if __name__ == "__main__":
    main()
