"""Writes statistics_ref.npz: the reference's own cfdr.statistics functions
(rans-uq/python/cfdr/statistics.py: resample_posterior :235-259, predictive_summary
:277-339, conformal_quantile :349-355, split_conformal_intervals :358-378) run on
seeded synthetic ensembles, for the device statistics to be checked against. The
compiled cfdr._core is not needed by these functions and is stubbed. Run where the
reference sources are present:

    python tests/golden/make_statistics_golden.py /path/to/reference
"""
import os
import importlib.util
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RQ_REFERENCE_DIR", "/root/reference"))

pkg = types.ModuleType("cfdr")
pkg.__path__ = [str(REF / "rans-uq" / "python" / "cfdr")]
core = types.ModuleType("cfdr._core")
sys.modules["cfdr"] = pkg
sys.modules["cfdr._core"] = core
pkg._core = core
spec = importlib.util.spec_from_file_location("cfdr.statistics",
                                              REF / "rans-uq/python/cfdr/statistics.py")
stats = importlib.util.module_from_spec(spec)
sys.modules["cfdr.statistics"] = stats
spec.loader.exec_module(stats)


def records(n, d, seed):
    """n converged evaluations with shuffled sample ids, 2 parameters, d predictions."""
    rng = np.random.default_rng(seed)
    ids = rng.permutation(np.arange(100, 100 + 3 * n))[:n]
    theta = rng.uniform([0.28, 0.084], [0.34, 0.096], size=(n, 2))
    pred = rng.normal(10.0, 3.0, size=(n, d)) * rng.uniform(0.5, 2.0, size=d)
    ll = -0.5 * rng.chisquare(d, n) * rng.uniform(0.5, 30.0)
    recs = tuple(stats.Evaluation(int(ids[i]), tuple(map(float, theta[i])), "Converged",
                                  tuple(map(float, pred[i])), float(ll[i]), 10, "b200", "")
                 for i in range(n))
    return stats.EvaluationSet(recs), ids, theta, pred, ll


out = {}
for tag, n, d in (("a", 64, 30), ("b", 1000, 1), ("c", 7, 3)):
    ev, ids, theta, pred, ll = records(n, d, seed=len(tag) * 1000 + n + d)
    out[f"{tag}_ids"], out[f"{tag}_theta"], out[f"{tag}_pred"], out[f"{tag}_ll"] = ids, theta, pred, ll
    draws = stats.resample_posterior(ev, range(5000, 5400), root_seed=20261010)
    out[f"{tag}_resample_ids"] = np.arange(5000, 5400)
    out[f"{tag}_resample_theta"] = np.array([s.theta for s in draws])
    sigma = np.linspace(0.1, 0.5, d)
    s = stats.predictive_summary(ev, root_seed=77, observation_sigma=sigma,
                                 surrogate_variance=np.full(d, 0.01),
                                 discrepancy_variance=None)
    out[f"{tag}_sigma"] = sigma
    out[f"{tag}_samples"] = np.array(s.samples)
    out[f"{tag}_latent_mean"] = np.array(s.latent_mean)
    out[f"{tag}_latent_variance"] = np.array(s.latent_variance)
    out[f"{tag}_total_variance"] = np.array(s.total_variance)
    print(tag, n, d, len(draws), flush=True)

rng = np.random.default_rng(42)
for n in (1, 19, 1000, 20000):
    scores = np.abs(rng.standard_t(3, size=n))
    out[f"scores_{n}"] = scores
    out[f"quantile_{n}"] = np.array([stats.conformal_quantile(scores, a)
                                     for a in (0.05, 0.1, 0.5, 0.9)])
cal_y, cal_p = rng.normal(size=500), rng.normal(size=500)
test_p = rng.normal(size=300)
lo, hi = stats.split_conformal_intervals(cal_y, cal_p, test_p, alpha=0.1)
out.update(cal_y=cal_y, cal_p=cal_p, test_p=test_p, split_lo=lo, split_hi=hi)
np.savez_compressed(HERE / "statistics_ref.npz", **out)
print("written", len(out))
