"""Writes tests/golden/bump_100x50_ref.npz: converged solves of the bump-wall channel
(the benchmark's geometry -- bump of height h = 1, L = 9h, W = 4h, top 3.04h, Re 5600,
y+ 1 -- on 100 x 50 cells, tol 1e-8, cap 30000) by the compiled reference
(oracle/_ref, the reference's own ForwardModel) at (a1, beta*) = (0.31, 0.09), once
with its AMG pressure solver and once with BiCGSTAB. Stored: verdict, outer
iterations, predictions at the 6 probes and the Ux, Uy, p, k, omega fields. About six
CPU minutes per solve (the two run concurrently).

    python tests/golden/make_bump_golden.py
"""
import multiprocessing
import sys
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def solve(psolver):
    from oracle import checker as ck
    import cases

    case = cases.bump_case(100, 50, tol=1e-8, max_iter=30000,
                           pressure_solver=psolver).with_theta(0.31, 0.09)
    o = ck.solve(case, "ref")
    print(psolver, o.status, o.iterations, flush=True)
    return psolver, o


def main():
    from oracle import checker as ck

    with ProcessPoolExecutor(max_workers=2, mp_context=multiprocessing.get_context("spawn")) as ex:
        res = dict(ex.map(solve, [ck.P_AMG, ck.P_BICGSTAB]))
    out = {}
    for name, k in (("amg", ck.P_AMG), ("bicgstab", ck.P_BICGSTAB)):
        o = res[k]
        out.update({f"{name}_status": o.status, f"{name}_iterations": o.iterations,
                    f"{name}_loglik": o.loglik, f"{name}_predictions": o.predictions,
                    f"{name}_Ux": o.field("Ux"), f"{name}_Uy": o.field("Uy"),
                    f"{name}_p": o.field("p"), f"{name}_k": o.field("k"),
                    f"{name}_omega": o.field("omega")})
    np.savez_compressed(Path(__file__).with_name("bump_100x50_ref.npz"), **out)
    print("wrote bump_100x50_ref.npz")


if __name__ == "__main__":
    main()
