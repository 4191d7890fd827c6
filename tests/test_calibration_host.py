"""The calibration stages (rans_uq_b200.calibration) against the reference's own
stage functions run on the same analytic log-likelihood (golden vectors of
tests/golden/make_calibration_golden.py): the same stage-1 winner, pattern-search
path, Laplace fit, Student-t draws, importance weights and resampled draws. The
importance weights here use a host restatement of the reference's rule
(exp(l - max) / fsum); tests/test_gpu_calibration.py repeats this with the GPU
weights."""
import json
import math
from pathlib import Path

import numpy as np

import rans_uq_b200.calibration as cal

GOLD = json.loads((Path(__file__).parent / "golden" / "calibration_stages.json").read_text())


def analytic_loglik(theta):
    """The function of make_calibration_golden.py."""
    d = (np.asarray(theta) - np.array([0.3137, 0.0912])) / np.array([0.002, 0.0007])
    rho = 0.4
    q = (d[0] ** 2 - 2 * rho * d[0] * d[1] + d[1] ** 2) / (1 - rho ** 2)
    return float(-0.5 * q - 0.02 * q * q)


def evaluator(ids, theta):
    return ["Converged"] * len(theta), np.array([analytic_loglik(t) for t in theta])


def host_weights(v):
    m = max(v)
    w = [math.exp(x - m) for x in v]
    return np.asarray(w) / math.fsum(w)


def check(out, weight_rtol):
    np.testing.assert_array_equal(out.stage1_best, GOLD["stage1_best"])
    np.testing.assert_array_equal(np.asarray(out.path), np.asarray(GOLD["path"]))
    np.testing.assert_array_equal(out.optimum, GOLD["optimum"])
    np.testing.assert_array_equal(out.step, GOLD["step"])
    np.testing.assert_allclose(out.laplace["peak"], GOLD["laplace"]["peak"], rtol=1e-12)
    np.testing.assert_allclose(out.laplace["covariance"], GOLD["laplace"]["covariance"],
                               rtol=1e-12)
    np.testing.assert_allclose(out.center, GOLD["center"], rtol=1e-14)
    np.testing.assert_allclose(out.scale, GOLD["scale"], rtol=1e-12)
    for got, want in zip(out.importance, (GOLD["main"], GOLD["replicate"])):
        np.testing.assert_allclose(got["theta"], want["theta"], rtol=1e-14)
        np.testing.assert_allclose(got["log_q"], want["log_q"], rtol=1e-13)
        np.testing.assert_allclose(got["weights"], want["weights"], rtol=weight_rtol)
        assert abs(got["effective_sample_size"] - want["effective_sample_size"]) < \
            1e-10 * want["effective_sample_size"]
        assert got["distinct_draws"] == want["distinct_draws"]
        np.testing.assert_allclose(got["theta_mean"], want["theta_mean"], rtol=1e-13)
        np.testing.assert_allclose(got["theta_sd"], want["theta_sd"], rtol=1e-9)


def test_stages_match_reference_functions():
    out = cal.calibrate(evaluator, weights=host_weights)
    check(out, 1e-15)
    # 24 + 8 per pattern-search step + 25 + 2 x 64 solves
    assert out.solves == 24 + 8 * (len(out.path) - 1 + 3) + 25 + 128
    assert [s.name for s in out.stages] == ["uniform design", "pattern search", "Laplace grid",
                                            "importance", "replicate"]


def test_resample_order_invariance():
    rng = np.random.default_rng(1)
    theta = rng.normal(size=(10, 2))
    w = rng.random(10)
    w /= w.sum()
    ids = list(range(50, 60))
    perm = rng.permutation(10)
    a = cal.resample(ids, theta, w, range(5), 7)
    b = cal.resample([ids[k] for k in perm], theta[perm], w[perm], range(5), 7)
    np.testing.assert_array_equal(a, b)


# ---- the whole study: predictive ranges, split-conformal recalibration, coverage.
# The golden is the reference's calibrate() itself (make_calibration_golden.py) on the
# analytic log-likelihood with 30 analytic station predictions and a synthetic profile.
STUDY = GOLD["study"]


def station_speed(y):
    """The stand-in profile of make_calibration_golden.py."""
    yp = np.asarray(y) * 182.088
    return 2.5 * np.log1p(yp) + 5.0 * (1.0 - np.exp(-yp / 11.0))


def study_evaluator(ids, theta):
    y = np.asarray(STUDY["y_plus"]) / 182.088
    pred = np.array([station_speed(y) * (1 + 4 * (t[0] - 0.3137) - 9 * (t[1] - 0.0912))
                     for t in theta])
    return ["Converged"] * len(theta), np.array([analytic_loglik(t) for t in theta]), pred


class HostStats:
    """cfdr.statistics.predictive_summary (:277-339) and split_conformal_intervals
    (:358-378) restated with numpy, for the CPU run of the study."""

    @staticmethod
    def predictive_summary(sample_ids, predictions, *, root_seed, observation_sigma):
        from types import SimpleNamespace

        from rans_uq_b200.workloads import sample_rng

        ids = list(sample_ids)
        latent = np.asarray(predictions, dtype=float)
        obs = np.asarray(observation_sigma, dtype=float) ** 2
        samples = latent.copy()
        for i, sid in enumerate(ids):
            samples[i] += sample_rng(root_seed, sid, "observation-noise").normal(
                0, np.sqrt(obs), latent.shape[1])
        canonical = latent[np.argsort(ids)]
        return SimpleNamespace(samples=samples, latent_mean=canonical.mean(axis=0),
                               latent_variance=canonical.var(axis=0, ddof=0),
                               observation_variance=obs)

    @staticmethod
    def split_conformal_intervals(y, p, t, *, alpha):
        scores = np.abs(np.asarray(y) - np.asarray(p))
        k = math.ceil((scores.size + 1) * (1 - alpha))
        r = math.inf if k > scores.size else float(np.partition(scores, k - 1)[k - 1])
        return np.asarray(t) - r, np.asarray(t) + r


def check_study(study):
    for key in ("prediction", "standard_low", "standard_high", "recalibrated_low",
                "recalibrated_high", "latent_variance", "observation_variance"):
        np.testing.assert_array_equal(study[key], STUDY[key], err_msg=key)
    for key in ("standard_covered", "recalibrated_covered", "held_out", "group"):
        assert study[key] == STUDY[key], key
    for key in ("prediction", "standard_low", "standard_high", "standard_covered"):
        np.testing.assert_array_equal(study["replicate"][key], STUDY["replicate"][key],
                                      err_msg=key)


def test_study_ranges_and_recalibration_match_reference():
    out = cal.calibrate(study_evaluator, weights=host_weights, truth=STUDY["truth"],
                        sigma=STUDY["sigma"], stats=HostStats)
    check(out, 1e-15)
    check_study(out.study)
    samples = np.asarray(out.importance[0]["predictive"].samples)
    np.testing.assert_array_equal(samples[:3], STUDY["predictive_samples_head"])
