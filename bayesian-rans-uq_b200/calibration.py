"""The calibration stages of the reference's channel study, with every stage's
solves run as one batch on the GPU (docs/figures/calibration_coverage.py:116-262):

1. a seeded uniform design of 24 draws over the stage-1 box; its best draw
2. a 3 x 3 pattern search from there, halving the step three times when the
   centre wins (:125-142)
3. a 5 x 5 grid of +/- 2 final steps and a least-squares quadratic of the
   log-likelihood on it: the Laplace centre and covariance (:145-167, :244-256)
4. two independent Student-t importance samples of 64 draws (nu = 4) from that
   centre and scale (:170-184), each weighted by likelihood over proposal
   density on the GPU in FP64 (statistics.posterior_weights) and resampled
   (cfdr.statistics.resample_posterior, rans-uq/python/cfdr/statistics.py:235-259);
   with the stations' noise sigma, the 400 resampled draws' predictions give the
   posterior predictive summary and its 90 % ranges (importance_posterior, :183-222)
5. with the observed profile, the split-conformal recalibration of those ranges on
   the log scale and their coverage of the held-out third of the stations
   (calibrate, :257-288).

The stage logic follows the reference step for step (same seeds, sample ids,
identity strings and tie rules) so the same log-likelihoods give the same path,
fit and draws; only the forward model changed.

`evaluator(ids, theta) -> (status names, log-likelihoods[, predictions])` is the
forward model of a stage: `batch_evaluator(ForwardBatch)` runs one GPU batch per
stage and returns the station predictions too.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import statistics as gpu_stats
from .workloads import sample_rng

SEED = 20261010
STAGE1_BOX = ((0.28, 0.084), (0.34, 0.096))
SEARCH_STEP = (0.004, 0.001)
PROPOSAL_DRAWS = 64
PROPOSAL_DOF = 4
ALPHA = 0.1


def batch_evaluator(batch):
    """A stage evaluator over a ForwardBatch: one GPU batch for all of a stage's draws."""
    def evaluate(ids, theta):
        res = batch.evaluate(np.asarray(theta, dtype=np.float64))
        return ([r.result.status.name for r in res.rows],
                np.array([r.result.log_lik for r in res.rows], dtype=np.float64),
                np.array([r.result.predictions for r in res.rows], dtype=np.float64))
    return evaluate


def _evaluate(evaluator, ids, theta, with_predictions=False):
    out = evaluator(list(ids), np.asarray(theta, dtype=np.float64))
    status, ll = out[0], out[1]
    failed = sum(1 for s, v in zip(status, ll) if s != "Converged" or not math.isfinite(v))
    if failed:
        raise RuntimeError(f"{failed} solves failed; the posterior is undefined")
    ll = np.asarray(ll, dtype=np.float64)
    if with_predictions:
        return ll, (np.asarray(out[2], dtype=np.float64) if len(out) > 2 else None)
    return ll


def uniform_design(ids, lower, upper, root_seed):
    lo, hi = np.asarray(lower, dtype=float), np.asarray(upper, dtype=float)
    return np.array([sample_rng(root_seed, i, "prior-design").uniform(lo, hi) for i in ids])


def pattern_search(evaluator, start, start_ll, step=SEARCH_STEP):
    """Compass search on the 3 x 3 grid of points one step apart around the centre:
    the centre moves to the grid's highest log-likelihood; when the centre itself is
    highest the step shrinks by half, up to three times. Returns (centre, final step,
    path of [a1, beta*, loglik])."""
    center, best, step = np.asarray(start, dtype=float), float(start_ll), np.asarray(step)
    path, halvings, solves = [[*center, best]], 0, 0
    offsets = [(i, j) for i in (-1, 0, 1) for j in (-1, 0, 1) if (i, j) != (0, 0)]
    while halvings < 3:
        theta = np.array([center + step * np.asarray(o) for o in offsets])
        ll = _evaluate(evaluator, range(len(offsets)), theta)
        solves += len(offsets)
        k = int(np.argmax(ll))  # the first of equal maxima, as max() over records
        if ll[k] > best:
            center, best = theta[k], float(ll[k])
            path.append([*center, best])
        else:
            step, halvings = step / 2, halvings + 1
    return center, step, path, solves


def laplace_fit(log_likelihood, x):
    """Least-squares quadratic c + g.x - x.C.x / 2 in scaled coordinates x: its peak
    C^-1 g, covariance C^-1, residual rms and range. C must be positive definite."""
    design = np.column_stack([np.ones(len(x)), x[:, 0], x[:, 1], x[:, 0] ** 2,
                              x[:, 0] * x[:, 1], x[:, 1] ** 2])
    coef, *_ = np.linalg.lstsq(design, log_likelihood, rcond=None)
    curvature = -np.array([[2 * coef[3], coef[4]], [coef[4], 2 * coef[5]]])
    if np.any(np.linalg.eigvalsh(curvature) <= 0):
        raise RuntimeError("the log-likelihood is not concave on the fitting grid")
    residual = log_likelihood - design @ coef
    return {"peak": np.linalg.solve(curvature, coef[1:3]),
            "covariance": np.linalg.inv(curvature),
            "residual_rms": float(np.sqrt(np.mean(residual ** 2))),
            "range": float(np.ptp(log_likelihood))}


def student_t_draws(center, scale, ids, seed, nu=PROPOSAL_DOF):
    """Seeded multivariate Student-t draws and the log proposal density of each."""
    center = np.asarray(center, dtype=float)
    dim = len(center)
    chol, precision = np.linalg.cholesky(scale), np.linalg.inv(scale)
    constant = (math.lgamma((nu + dim) / 2) - math.lgamma(nu / 2)
                - dim / 2 * math.log(nu * math.pi) - 0.5 * math.log(np.linalg.det(scale)))
    theta, log_q = [], []
    for i in ids:
        rng = sample_rng(seed, i, "student-t-proposal")
        z, chi2 = rng.standard_normal(dim), rng.chisquare(nu)
        offset = chol @ z * math.sqrt(nu / chi2)
        theta.append(center + offset)
        log_q.append(constant - (nu + dim) / 2 * math.log1p(offset @ precision @ offset / nu))
    return np.array(theta), np.array(log_q)


def resample_picks(ids_in, weights, out_ids, root_seed):
    """Indices (into ids_in) of IID multinomial draws from the weighted sample: inputs
    in sample-id order, one stream per output id."""
    order = np.argsort(np.asarray(ids_in), kind="stable")
    w = np.asarray(weights)[order]
    picks = [int(sample_rng(root_seed, i, "posterior-resample").choice(len(w), p=w))
             for i in out_ids]
    return order[picks]


def resample(ids_in, theta, weights, out_ids, root_seed):
    """The drawn theta rows (resample_posterior's draws, in output-id order)."""
    return np.asarray(theta)[resample_picks(ids_in, weights, out_ids, root_seed)]


@dataclass
class Stage:
    name: str
    solves: int
    seconds: float = 0.0


@dataclass
class Calibration:
    stage1_best: np.ndarray
    optimum: np.ndarray
    step: np.ndarray
    path: list
    laplace: dict
    center: np.ndarray
    scale: np.ndarray
    importance: list = field(default_factory=list)   # main, replicate
    stages: list = field(default_factory=list)
    study: dict = field(default_factory=dict)        # ranges, recalibration, coverage

    @property
    def solves(self) -> int:
        return sum(s.solves for s in self.stages)


def importance_stage(evaluator, center, scale, ids, seed, weights=None, sigma=None,
                     stats=None):
    """One Student-t importance sample (importance_posterior, :183-222): weights,
    400 resampled draws and, given the stations' sigma and predictions from the
    evaluator, the posterior predictive summary of the draws and its 90 % ranges."""
    theta, log_q = student_t_draws(center, scale, ids, seed)
    ll, pred = _evaluate(evaluator, ids, theta, with_predictions=True)
    # flat prior: a draw from q weighs L / q
    w = (weights or gpu_stats.posterior_weights)(ll - log_q)
    mean = w @ theta
    picks = resample_picks(list(ids), w, range(1000, 1400), seed + 1)
    draws = theta[picks]
    out = {"solves": len(ids), "effective_sample_size": float(1 / np.sum(w ** 2)),
           "max_weight": float(w.max()),
           "distinct_draws": len({tuple(t) for t in draws}),
           "theta_mean": mean.tolist(),
           "theta_sd": np.sqrt(w @ (theta - mean) ** 2).tolist(),
           "weights": w, "theta": theta, "log_q": log_q, "log_lik": ll}
    if sigma is not None and pred is not None:
        # each draw repeats an evaluated theta: its predictions are reused, not re-solved
        predictive = (stats or gpu_stats).predictive_summary(
            range(1000, 1400), pred[picks], root_seed=seed + 2, observation_sigma=sigma)
        samples = np.asarray(predictive.samples)
        low, high = np.quantile(samples, [ALPHA / 2, 1 - ALPHA / 2], axis=0)
        out.update(predictive=predictive, low=low, high=high, posterior_latent=pred[picks])
    return out


def calibrate(evaluator, clock=None, weights=None, trace=None, truth=None, sigma=None,
              stats=None) -> Calibration:
    """All stages, each one batch of solves (pattern-search steps one batch each).
    weights: the importance-weight function (default: FP64 on the GPU); trace (a
    dict, optional) receives each stage's intermediate results as they appear, so
    a stage that raises leaves the earlier ones behind. With the stations' observed
    profile `truth` and noise `sigma` (and an evaluator that returns predictions),
    the study's predictive ranges, split-conformal recalibration and coverage follow
    (out.study); `stats` supplies predictive_summary and split_conformal_intervals
    (default: the GPU ones)."""
    import time

    clock = clock or time.perf_counter
    trace = {} if trace is None else trace
    stages = []
    t = clock()
    lower, upper = STAGE1_BOX
    th1 = uniform_design(range(24), lower, upper, SEED)
    ll1 = _evaluate(evaluator, range(24), th1)
    k = int(np.argmax(ll1))
    stages.append(Stage("uniform design", 24, clock() - t))
    trace["stage1"] = {"best": th1[k].tolist(), "best_loglik": float(ll1[k])}
    t = clock()
    optimum, step, path, n_search = pattern_search(evaluator, th1[k], ll1[k])
    stages.append(Stage("pattern search", n_search, clock() - t))
    trace["pattern_search"] = {"path": path, "step": step.tolist()}
    t = clock()
    offsets = np.array([(i, j) for i in range(-2, 3) for j in range(-2, 3)], dtype=float)
    grid = np.array([optimum + step * o for o in offsets])
    llg = _evaluate(evaluator, range(200, 225), grid)
    trace["laplace_grid"] = {"theta": grid.tolist(), "loglik": llg.tolist()}
    fit = laplace_fit(llg, (grid - optimum) / step)
    center = optimum + step * fit["peak"]
    scale = np.diag(step) @ fit["covariance"] @ np.diag(step)
    if np.any(np.abs(fit["peak"]) > 2):
        raise RuntimeError("the fitted peak lies outside the fitting grid")
    stages.append(Stage("Laplace grid", 25, clock() - t))
    out = Calibration(th1[k], optimum, step, path, fit, center, scale, stages=stages)
    for name, ids, seed in (("importance", range(300, 300 + PROPOSAL_DRAWS), SEED + 1),
                            ("replicate", range(400, 400 + PROPOSAL_DRAWS), SEED + 11)):
        t = clock()
        out.importance.append(importance_stage(evaluator, center, scale, ids, seed, weights,
                                               sigma, stats))
        stages.append(Stage(name, len(ids), clock() - t))
    if truth is not None and "predictive" in out.importance[0]:
        out.study = coverage_study(out.importance[0], out.importance[1],
                                   np.asarray(truth, dtype=float), stats or gpu_stats)
    return out


def coverage_study(main, replicate, truth, stats):
    """The study's ranges and their honesty (calibrate, :257-288): stations split
    into thirds by index (likelihood, conformal calibration, held out); the
    split-conformal correction of the main sample's latent mean on the log scale;
    how many held-out stations each range covers."""
    group = np.arange(len(truth)) % 3
    cal, test = group == 1, group == 2
    prediction = np.asarray(main["predictive"].latent_mean)
    log_lo, log_hi = stats.split_conformal_intervals(np.log(truth[cal]), np.log(prediction[cal]),
                                                     np.log(prediction), alpha=ALPHA)
    low, high = main["low"], main["high"]
    rec_low, rec_high = np.exp(log_lo), np.exp(log_hi)
    r_low, r_high = replicate["low"], replicate["high"]
    return {"group": group.tolist(), "prediction": prediction.tolist(),
            "standard_low": low.tolist(), "standard_high": high.tolist(),
            "recalibrated_low": rec_low.tolist(), "recalibrated_high": rec_high.tolist(),
            "latent_variance": list(main["predictive"].latent_variance),
            "observation_variance": list(main["predictive"].observation_variance),
            "standard_covered": int(np.sum((truth >= low) & (truth <= high) & test)),
            "recalibrated_covered": int(np.sum((truth >= rec_low) & (truth <= rec_high) & test)),
            "held_out": int(test.sum()),
            "replicate": {"prediction": list(replicate["predictive"].latent_mean),
                          "standard_low": r_low.tolist(), "standard_high": r_high.tolist(),
                          "standard_covered": int(np.sum((truth >= r_low) & (truth <= r_high)
                                                         & test))}}
