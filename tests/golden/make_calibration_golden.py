"""Writes calibration_stages.json: the reference's own calibration-stage functions
(docs/figures/calibration_coverage.py: pattern_search, laplace_fit,
student_t_draws, importance weighting and resampling; cfdr.statistics) run on an
analytic log-likelihood instead of the SST solve, so that the stage logic of
rans_uq_b200.calibration can be checked against them without a flow solver.
Run in a checkout where the reference sources are present:

    python tests/golden/make_calibration_golden.py /path/to/reference
"""
import os
import dataclasses
import importlib.util
import json
import math
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RQ_REFERENCE_DIR", "/root/reference"))


def analytic_loglik(theta):
    """A smooth, slightly non-quadratic log-likelihood peaked near (0.3137, 0.0912)."""
    d = (np.asarray(theta) - np.array([0.3137, 0.0912])) / np.array([0.002, 0.0007])
    rho = 0.4
    q = (d[0] ** 2 - 2 * rho * d[0] * d[1] + d[1] ** 2) / (1 - rho ** 2)
    return float(-0.5 * q - 0.02 * q * q)


# stand-ins for the compiled module and the plotting library
core = types.ModuleType("cfdr._core")


class _Status:
    name = "Converged"


class _Result:
    def __init__(self, theta):
        self.status = _Status()
        self.log_lik = analytic_loglik(theta)
        self.predictions = [float(theta[0]), float(theta[1])]
        self.simple_iters = 1


class _Row:
    def __init__(self, theta):
        self.result = _Result(theta)
        self.error = ""


class ForwardBatch:
    def evaluate(self, theta, workers=1):
        return types.SimpleNamespace(rows=[_Row(t) for t in np.asarray(theta)])


core.ForwardBatch = ForwardBatch
core.ForwardModel = type("ForwardModel", (), {})
pkg = types.ModuleType("cfdr")
pkg.__path__ = [str(REF / "rans-uq" / "python" / "cfdr")]
sys.modules["cfdr"] = pkg
sys.modules["cfdr._core"] = core
pkg._core = core
for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.patches", "matplotlib.ticker"):
    m = types.ModuleType(name)
    m.FancyBboxPatch = m.FixedLocator = m.NullFormatter = m.NullLocator = object
    sys.modules[name] = m
spec = importlib.util.spec_from_file_location("cfdr.statistics",
                                              REF / "rans-uq/python/cfdr/statistics.py")
stats = importlib.util.module_from_spec(spec)
sys.modules["cfdr.statistics"] = stats
spec.loader.exec_module(stats)
pkg.statistics = stats
spec = importlib.util.spec_from_file_location("calibration_coverage",
                                              REF / "docs/figures/calibration_coverage.py")
cal = importlib.util.module_from_spec(spec)
spec.loader.exec_module(cal)

batch = ForwardBatch()
lower, upper = cal.STAGE1_BOX
stage1 = cal.evaluate(batch, stats.independent_uniform_design(range(24), lower, upper,
                                                              root_seed=cal.SEED), 1)
first = max(stage1.records, key=lambda r: r.log_likelihood)
optimum, step, path = cal.pattern_search(batch, first.theta, first.log_likelihood, 1)
offsets = np.array([(i, j) for i in range(-2, 3) for j in range(-2, 3)], dtype=float)
grid = cal.evaluate(batch, tuple(stats.Sample(200 + k, tuple(optimum + step * o))
                                 for k, o in enumerate(offsets)), 1)
scaled = np.array([(np.asarray(r.theta) - optimum) / step for r in grid.records])
fit = cal.laplace_fit(np.array([r.log_likelihood for r in grid.records]), scaled)
center = optimum + step * fit["peak"]
scale = np.diag(step) @ fit["covariance"] @ np.diag(step)


def importance(ids, seed):
    samples, log_q = cal.student_t_draws(center, scale, ids, seed)
    ev = cal.evaluate(batch, samples, 1)
    ratio = stats.EvaluationSet(tuple(dataclasses.replace(r, log_likelihood=r.log_likelihood
                                                          - log_q[r.sample_id])
                                      for r in ev.records))
    w = stats.posterior_weights(ratio)
    theta = np.array([r.theta for r in ratio.records])
    mean = w @ theta
    draws = stats.resample_posterior(ratio, range(1000, 1400), root_seed=seed + 1)
    return {"theta": theta.tolist(), "log_q": [log_q[i] for i in ids], "weights": w.tolist(),
            "effective_sample_size": float(1 / np.sum(w ** 2)), "max_weight": float(w.max()),
            "distinct_draws": len({d.theta for d in draws}), "theta_mean": mean.tolist(),
            "theta_sd": np.sqrt(w @ (theta - mean) ** 2).tolist(),
            "draws_head": [list(d.theta) for d in draws[:20]]}


out = {"stage1_best": list(first.theta), "stage1_best_ll": first.log_likelihood,
       "optimum": optimum.tolist(), "step": step.tolist(), "path": path,
       "laplace": {"peak": fit["peak"].tolist(), "covariance": fit["covariance"].tolist(),
                   "residual_rms": fit["residual_rms"], "range": fit["range"]},
       "center": center.tolist(), "scale": scale.tolist(),
       "main": importance(range(300, 300 + cal.PROPOSAL_DRAWS), cal.SEED + 1),
       "replicate": importance(range(400, 400 + cal.PROPOSAL_DRAWS), cal.SEED + 11)}


# ---- the reference's whole study, calibrate() (calibration_coverage.py:225-307), on
# the same analytic log-likelihood with 30 analytic station predictions, and a
# synthetic profile written in the simulation files' column layout (y/delta, y+, U+):
# the posterior predictive ranges, the split-conformal recalibration and coverage.
def station_speed(y):
    """A smooth positive stand-in for the mean profile at y (in half heights)."""
    yp = np.asarray(y) * cal.RE_TAU
    return 2.5 * np.log1p(yp) + 5.0 * (1.0 - np.exp(-yp / 11.0))


def analytic_predictions(theta, y):
    return station_speed(y) * (1 + 4 * (theta[0] - 0.3137) - 9 * (theta[1] - 0.0912))


class Vec3:
    def __init__(self, x=0.0, y=0.0, z=0.0):
        self.x, self.y, self.z = x, y, z


class Observations:
    def __init__(self):
        self.y = []

    def add_velocity_profile(self, at, component, value, sigma):
        self.y.append(at.y)


class _StudyResult:
    def __init__(self, theta, y):
        self.status = _Status()
        self.log_lik = analytic_loglik(theta)
        self.predictions = [float(v) for v in analytic_predictions(theta, y)]
        self.simple_iters = 1


class StudyBatch(ForwardBatch):
    def __init__(self, mesh=None, params=None, obs=None, *args):
        self.y = np.asarray(obs.y)

    def evaluate(self, theta, workers=1):
        rows = []
        for t in np.asarray(theta):
            row = _Row(t)
            row.result = _StudyResult(t, self.y)
            rows.append(row)
        return types.SimpleNamespace(rows=rows)


class Mesh:
    @staticmethod
    def make_periodic_channel_2d(*args):
        return types.SimpleNamespace(compute_wall_distance=lambda: None)


core.Vec3 = Vec3
core.ObservationOperator = Observations
core.Mesh = Mesh
core.SolverSettings = types.SimpleNamespace
core.FlowBoundaryConditions = types.SimpleNamespace(channel_defaults=lambda *a: None)
core.InferenceParameterSet = types.SimpleNamespace(a1_betaStar=lambda: None)
core.ForwardBatch = StudyBatch
cal.c = core

import tempfile  # noqa: E402

yp_grid = np.geomspace(0.05, 182.088, 400)
speed = station_speed(yp_grid / cal.RE_TAU)
noise = np.random.default_rng(5).standard_normal(400)
with tempfile.TemporaryDirectory() as d:
    mean_file, stdev_file = Path(d) / "mean.dat", Path(d) / "stdev.dat"
    np.savetxt(mean_file, np.column_stack([yp_grid / cal.RE_TAU, yp_grid,
                                           speed * (1 + 0.01 * noise)]), header="synthetic",
               comments="% ")
    np.savetxt(stdev_file, np.column_stack([yp_grid / cal.RE_TAU, yp_grid, 0.0014 * speed]),
               header="synthetic", comments="% ")
    study = cal.calibrate(mean_file, stdev_file, 1)
keys = ("y_plus", "truth", "sigma", "group", "prediction", "standard_low", "standard_high",
        "recalibrated_low", "recalibrated_high", "latent_variance", "observation_variance",
        "standard_covered", "recalibrated_covered", "held_out", "effective_sample_size",
        "distinct_draws", "solves")
out["study"] = {k: study[k] for k in keys}
out["study"]["replicate"] = {k: study["replicate"][k] for k in
                             ("prediction", "standard_low", "standard_high", "standard_covered")}
out["study"]["predictive_samples_head"] = study["predictive_samples"][:3]
out["study"]["predictive_samples_mean"] = np.mean(study["predictive_samples"], axis=0).tolist()
print("study", study["standard_covered"], study["recalibrated_covered"], study["held_out"])
(HERE / "calibration_stages.json").write_text(json.dumps(out, indent=1))
print("path steps", len(path), "center", center, "ESS", out["main"]["effective_sample_size"])
