"""Regenerates the golden fixtures of tests/golden/ from the reference itself.

Run in a container where the reference sources are mounted and oracle/_ref is
built (``make -C oracle ref``):  python tests/golden/make_golden.py
Every number written here was computed by the compiled reference
(oracle/_ref/libcfdr_ref.so, the reference's own ForwardModel), or read from
the reference's committed golden JSON.
"""
import os
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
from oracle import checker as ck  # noqa: E402
import cases  # noqa: E402

OUT = Path(__file__).resolve().parent
REF = Path(os.environ.get("RQ_REFERENCE_DIR", "/root/reference"))


def solve_npz(name, case, hist=0):
    o = ck.solve(case, "ref", hist_cap=hist)
    np.savez_compressed(OUT / f"{name}.npz", status=o.status, iterations=o.iterations,
                        loglik=o.loglik, final_worst=o.final_worst, predictions=o.predictions,
                        Ux=o.field("Ux"), k=o.field("k"), omega=o.field("omega"),
                        nuT=o.field("nuT"), p=o.field("p"))
    print(name, o.status, o.iterations, flush=True)


def sequence_npz(name, case, thetas, byte_budget=64 * 1024 * 1024):
    """One reference ForwardModel evaluating thetas in order with its warm-start cache."""
    o = ck.solve_sequence(case, thetas, "ref", byte_budget=byte_budget)
    np.savez_compressed(OUT / f"{name}.npz", thetas=np.asarray(thetas, float),
                        status=np.array(o.status), iterations=o.iterations, loglik=o.loglik,
                        predictions=o.predictions, used_warm=o.used_warm, retained=o.retained,
                        byte_budget=byte_budget)
    print(name, o.status, o.iterations, o.used_warm, flush=True)


def main():
    which = set(sys.argv[1:]) or {"small", "config1", "goldens", "warm", "snapshot", "meshbin"}
    if "meshbin" in which:
        import hashlib
        import tempfile
        digests = {}
        for name, case in cases.MESH_BINARY_CASES.items():
            with tempfile.TemporaryDirectory() as d:
                path = Path(d) / "mesh.bin"
                ck.mesh_save_binary(case, path)
                data = path.read_bytes()
            digests[name] = {"bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
            print(name, len(data), flush=True)
        (OUT / "mesh_binary_sha256.json").write_text(json.dumps(digests, indent=1))
    if "snapshot" in which:
        for name, case in (("snapshot_small_channel_ref", cases.small_channel()),
                           ("snapshot_small_channel_capped_ref", cases.small_channel(max_iter=300))):
            o = ck.solve_snapshot(case)
            np.savez_compressed(OUT / f"{name}.npz", status=o["status"],
                                iterations=o["iterations"], cells=o["cells"],
                                boundary=o["boundary"], face_fluxes=o["face_fluxes"],
                                turb_established=o["turb_established"])
            print(name, o["status"], o["iterations"], o["turb_established"], flush=True)
    if "warm" in which:
        sequence_npz("warm_sequence_ref", cases.small_channel(), cases.WARM_SEQUENCE)
        sequence_npz("warm_budget_ref", cases.small_channel(), cases.WARM_BUDGET_SEQUENCE,
                     byte_budget=cases.WARM_BUDGET_BYTES)
    if "small" in which:
        solve_npz("small_channel_ref", cases.small_channel())
        solve_npz("small_channel_pcg_ref", cases.small_channel(pressure_solver=ck.P_PCG))
    if "config1" in which:
        solve_npz("config1_ref", ck.config1_case())
    if "goldens" in which:
        g = json.loads((REF / "tests/golden/constrained_omega/periodic_channel_re180.json").read_text())
        keep = {"nu": g["nu"], "mesh": g["mesh"], "settings": g["settings"],
                "result": {k: g["result"][k] for k in ("status", "final_iter", "final_worst_measure",
                                                        "contraction_rate_u")},
                "field_norms": g["result"]["field_norms"],
                "probe_y_over_delta": g["qoi"]["probe_y_over_delta"],
                "u_plus_probes": g["qoi"]["u_plus_probes"]}
        src = (REF / "rans-uq/tests/test_sst_channel_grid_convergence.cpp").read_text()
        keep["grid_convergence_note"] = "stations and U+ of test_sst_channel_grid_convergence.cpp:14-17"
        keep["grid_convergence_stations"] = [0.01, 0.03, 0.1, 0.2, 0.4, 0.7, 0.95]
        import re
        block = src[src.index("reference{"):src.index("};", src.index("reference{"))]
        keep["grid_convergence_uplus"] = [float(v) for v in re.findall(r"[0-9]+\.[0-9]+", block)]
        (OUT / "reference_goldens.json").write_text(json.dumps(keep, indent=1))
        print("goldens", len(keep["grid_convergence_uplus"]))


if __name__ == "__main__":
    main()
