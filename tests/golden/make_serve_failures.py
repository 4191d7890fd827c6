"""Writes tests/golden/serve_failures_ref.json: the compiled reference's verdicts
(oracle/_ref, the reference's own ForwardModel) on the 3 x 24 test channel capped at
9000 outer iterations, for in-bounds coefficient draws far from the calibration box
(a1 or beta* at the edges of their admissible ranges) that do not converge, beside
in-box draws that do. The serving test submits the same draws to the serving loop
and requires these verdicts.

    python tests/golden/make_serve_failures.py
"""
import json
import multiprocessing
import sys
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

CAP = 9000
THETAS = [(0.31, 0.09), (0.1, 0.2), (0.8, 0.2), (0.5, 0.2), (0.1, 0.1), (0.8, 0.01),
          (0.30, 0.088)]


def run(theta):
    import cases
    from oracle import checker as ck

    o = ck.solve(cases.small_channel(max_iter=CAP).with_theta(*theta), "ref")
    return {"theta": list(theta), "status": o.status, "iterations": int(o.iterations)}


def main():
    with ProcessPoolExecutor(len(THETAS), mp_context=multiprocessing.get_context("spawn")) as ex:
        rows = list(ex.map(run, THETAS))
    for r in rows:
        print(r)
    Path(__file__).with_name("serve_failures_ref.json").write_text(
        json.dumps({"cap": CAP, "rows": rows}, indent=1) + "\n")


if __name__ == "__main__":
    main()
