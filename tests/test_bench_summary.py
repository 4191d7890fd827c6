"""bench.py's JSON line from host copies of a step, on synthetic records (no GPU):
the row decoding of the 40-byte rq_row_out, the contract's keys, and the
roofline / latency arithmetic."""
import argparse
import json

import numpy as np

import bench
import rans_uq_b200 as rq


def fake_step(n=12):
    cls = np.arange(n) % 3
    rec = np.zeros(n, dtype=np.dtype([("status", "<i4"), ("iterations", "<i4"),
                                      ("stalled", "<i4"), ("converged", "<i4"),
                                      ("loglik", "<f8"), ("final_worst", "<f8"),
                                      ("contraction_rate", "<f8")]))
    rec["iterations"] = np.array([100, 200, 400])[cls]
    rec["status"][-1] = 1
    raw = np.frombuffer(rec.tobytes(), dtype=np.uint8)  # as copied from the device
    clock = np.zeros((n, 12), dtype=np.int64)
    clock[:, 0] = 1_000_000
    clock[:, 1] = 1_000_000 + np.array([1, 2, 4])[cls] * 1_000_000
    clock[:, 2] = 10 * rec["iterations"]
    clock[:, 3] = 5 * rec["iterations"]
    cells = np.array([384, 768, 1536])[cls]
    return raw, clock, cls, cells


def test_rows_decode_40_byte_records():
    raw, _, _, _ = fake_step()
    assert raw.size == 12 * 40
    recs = rq.rows_from_device_bytes(raw)
    assert len(recs) == 12 and recs["iterations"][2] == 400 and recs["status"][-1] == 1


def test_summary_has_contract_keys():
    raw, clock, cls, cells = fake_step()
    recs = rq.rows_from_device_bytes(raw)
    args = argparse.Namespace(steps=1, warmup=3, precision="fp64")
    out = bench.summarize(recs, clock, cls, cells, 4.0, 11, 1, args, 300000, 1.5, 100, 200,
                          [1e-4, 2e-4, 4e-4], {"hbm_gbs": 6552.3, "gpu_name": "x"},
                          {"sm_mhz": 1900}, None)
    json.dumps(out)
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e",
                "gpu_launches", "roofline", "clocks", "cpu_baseline"):
        assert key in out, key
    assert out["value"] == 11 / 4e-3 and out["converged"] == 11
    assert out["gpu_launches"] == 3
    # dominant class 2: 4 rows x 1536 cells x (1600*400 + 360*4000 + 400*2000) over 4 ms
    want = 4 * 1536 * (1600 * 400 + 360 * 4000 + 400 * 2000) / 4e-3 / 1e9
    assert abs(out["roofline"]["achieved"] - want) < 1e-9 * want
    assert out["roofline"]["peak"] == 6552.3
    r = out["roofline"]
    assert r["algorithmic_frac"] == r["frac"]
    # DRAM: first touch per 1536-cell draw x 4 draws; L2: bytes per iteration x 4 x 400
    assert r["traffic"] == bench.DRAM_BYTES_PER_DRAW_1536 * 4
    assert abs(r["l2_bytes"] - bench.L2_BYTES_PER_ITER_1536 * 1600) < 1e-6 * r["l2_bytes"]
    assert abs(r["l2_frac"] - r["l2_bytes"] / 4e-3 / 1e9 / bench.L2_PEAK_GBS) < 1e-12
    assert abs(out["latency_ms"]["max"] - 4.0) < 1e-12
    assert out["plain_fp64"]["solves_per_s"] > 0 and out["batched_vs_plain"] > 0


def test_summary_when_nothing_converges():
    raw, clock, cls, cells = fake_step()
    rec = rq.rows_from_device_bytes(raw).copy()
    rec["status"][:] = 1
    args = argparse.Namespace(steps=1, warmup=3, precision="fp64")
    out = bench.summarize(rec, clock, cls, cells, 4.0, 0, 1, args, 2000, 0.0, 100, 200,
                          [1e-4, 2e-4, 4e-4], {"hbm_gbs": 6552.3}, {}, None)
    assert out["value"] == 0.0 and out["batched_vs_plain"] is None
    assert out["roofline"]["peak_source"] == "fallback"


def test_summary_of_two_replicas():
    """At N = 2 the line reports the whole job: n_gpus 2, the converged solves of both
    ranks over the max-over-ranks step time, replicas x2, and no host CPU baseline."""
    raw, clock, cls, cells = fake_step()
    recs = rq.rows_from_device_bytes(raw)
    args = argparse.Namespace(steps=1, warmup=3, precision="fp64")
    out = bench.summarize(recs, clock, cls, cells, 5.0, 22, 2, args, 300000, 3.0, 100, 200,
                          [1e-4, 2e-4, 4e-4], {"hbm_gbs": 6552.3}, {"sm_mhz": 1900}, None)
    assert out["n_gpus"] == 2 and out["config"]["parallelism"] == "replicas x2"
    assert out["value"] == 22 / 5e-3 and out["cpu_baseline"] is None
    assert out["scaling"] == "weak"


def test_timed_steps_fit_the_driver_run():
    """The driver runs `--steps 20 --warmup 5` under an 1800 s limit. With a 148 s
    ensemble step, set-up and untimed legs of 120 s, and 2 full warm-up steps, the
    plan keeps the whole run inside the 1400 s default budget and still times at
    least one step."""
    elapsed = 120.0 + 2 * 148.0
    k = bench.plan_timed_steps(20, elapsed, 148.0, 1400.0)
    assert 1 <= k < 20
    assert elapsed + k * 148.0 + 30.0 <= 1400.0
    assert elapsed + (k + 1) * 148.0 + 30.0 > 1400.0
    # a short step runs every requested step; an over-budget run still times one
    assert bench.plan_timed_steps(20, 100.0, 1.0, 1400.0) == 20
    assert bench.plan_timed_steps(20, 1390.0, 148.0, 1400.0) == 1


def test_summary_reports_requested_and_timed_steps():
    raw, clock, cls, cells = fake_step()
    recs = rq.rows_from_device_bytes(raw)
    args = argparse.Namespace(steps=6, steps_requested=20, warmup=5, warmup_requested=5,
                              precision="fp64")
    out = bench.summarize(recs, clock, cls, cells, 4.0, 11, 1, args, 300000, 1.5, 100, 200,
                          [1e-4, 2e-4, 4e-4], {"hbm_gbs": 6552.3, "gpu_name": "x"},
                          {"sm_mhz": 1900}, None)
    assert out["steps"] == 6 and out["steps_requested"] == 20
    assert out["warmup"] == 5 and out["gpu_launches"] == 3 * 6


def test_cpu_baseline_extrapolates_each_draws_iterations():
    """The CPU line multiplies each draw's own outer iterations by its class's
    contended per-iteration time and divides by the cores; the measured subset's own
    counts replace the table's for the draws it ran."""
    cls = np.arange(6) % 3
    sample = {"cores": 2, "per_iteration_s": [1e-3, 2e-3, 4e-3],
              "subset": {"draws": [0], "iterations": [150], "statuses": ["Converged"],
                         "wall_s": 0.2, "solves_per_s": 5.0},
              "capped": {"draws": [1, 2], "iterations": 1500}}
    iters = np.array([100, 200, 400, 100, 200, 400])
    cb = bench.cpu_baseline(np.zeros((6, 2)), cls, iters, sample, "test")
    total = 150 * 1e-3 + 200 * 2e-3 + 400 * 4e-3 + 100 * 1e-3 + 200 * 2e-3 + 400 * 4e-3
    assert abs(cb["value"] - 6 / (total / 2)) < 1e-12
    assert cb["measured_subset"]["solves_per_s"] == 5.0 and cb["cores"] == 2
