"""Statistics of an ensemble on the GPU, in FP64: the importance weights of
cfdr.statistics.posterior_weights (rans-uq/python/cfdr/statistics.py:208-232) with
the optional proposal density of the Student-t importance stage
(docs/figures/calibration_coverage.py:165-180), and resampling, the predictive
mixture moments and split-conformal quantiles (statistics.py:235-378) with numpy's
rounding.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .core import EvaluationStatus, ForwardBatchResult


def _logliks(evaluations) -> np.ndarray:
    if isinstance(evaluations, ForwardBatchResult):
        rows = evaluations.rows
        if not rows:
            raise ValueError("at least one evaluation is required")
        failed = sum(1 for r in rows if r.result.status != EvaluationStatus.Converged or r.error)
        if failed:
            raise ValueError(f"{failed} unresolved evaluations; posterior is undefined")
        return np.array([r.result.log_lik for r in rows], dtype=np.float64)
    ll = np.ascontiguousarray(np.asarray(evaluations, dtype=np.float64).ravel())
    if ll.size == 0:
        raise ValueError("at least one evaluation is required")
    return ll


def posterior_weights(evaluations, log_q=None, return_log_evidence: bool = False):
    """Normalised weights w_i proportional to exp(l_i - log q_i). `evaluations` is a
    ForwardBatchResult (every row must be Converged, as the reference requires) or
    an array of log-likelihoods; log_q (optional) the proposal log densities."""
    ll = _logliks(evaluations)
    lq = None
    if log_q is not None:
        lq = np.ascontiguousarray(np.asarray(log_q, dtype=np.float64).ravel())
        if lq.shape != ll.shape:
            raise ValueError("log_q must have one value per evaluation")
    w = np.empty_like(ll)
    ev = C.c_double()
    N.call("rq_posterior_weights", N.dptr(ll), N.dptr(lq) if lq is not None else None,
           C.c_int64(ll.size), N.dptr(w), C.byref(ev))
    return (w, float(ev.value)) if return_log_evidence else w


def posterior_weight_parts(loglik, log_q=None):
    """(weights, m, s): the normalised weights of these draws with the two parts of
    their log-sum-exp, m = max(l - log q) and s = sum exp(l - log q - m)
    (rq_posterior_weights_parts), for combining shards of one ensemble."""
    ll = _logliks(loglik)
    lq = None
    if log_q is not None:
        lq = np.ascontiguousarray(np.asarray(log_q, dtype=np.float64).ravel())
        if lq.shape != ll.shape:
            raise ValueError("log_q must have one value per evaluation")
    w = np.empty_like(ll)
    m, s = C.c_double(), C.c_double()
    N.call("rq_posterior_weights_parts", N.dptr(ll), N.dptr(lq) if lq is not None else None,
           C.c_int64(ll.size), N.dptr(w), C.byref(m), C.byref(s))
    return w, float(m.value), float(s.value)


# ---- the rest of the statistics of a finished ensemble (cfdr.statistics,
# rans-uq/python/cfdr/statistics.py:235-378), computed on the GPU with numpy's rounding.
# Random draws come from the reference's per-sample streams (workloads.sample_rng) on
# the host; everything that scales with the ensemble runs on the device.

def resample_indices(weights, uniforms) -> np.ndarray:
    """Indices numpy's Generator.choice(len(weights), p=weights) returns for each of
    the given first uniforms (rq_resample_indices)."""
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).ravel())
    u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64).ravel())
    idx = np.empty(u.size, dtype=np.int64)
    N.call("rq_resample_indices", N.dptr(w), C.c_int64(w.size), N.dptr(u), C.c_int64(u.size),
           idx.ctypes.data_as(C.POINTER(C.c_int64)))
    return idx


@dataclass(frozen=True)
class Sample:
    """A drawn design point (cfdr.statistics.Sample, statistics.py:60-66)."""
    sample_id: int
    theta: tuple


def _records(evaluations):
    """(ids, theta rows, log-likelihoods, predictions) of an evaluation set with the
    reference's record fields (EvaluationSet.records: sample_id, theta, status, error,
    log_likelihood, predictions), every record required to be a success (_resolved,
    statistics.py:208-214)."""
    recs = tuple(evaluations.records)
    if not recs:
        raise ValueError("at least one evaluation is required")
    failed = sum(1 for r in recs if r.status != "Converged" or r.error)
    if failed:
        raise ValueError(f"{failed} unresolved evaluations; posterior is undefined")
    return ([int(r.sample_id) for r in recs], np.array([r.theta for r in recs], dtype=float),
            np.array([r.log_likelihood for r in recs], dtype=float),
            np.array([r.predictions for r in recs], dtype=float))


def resample_posterior(design_ids, theta=None, evaluations=None, sample_ids=None, *,
                       root_seed: int):
    """resample_posterior (statistics.py:235-259): IID multinomial draws from the
    importance posterior of a design. Called as the reference is,
    resample_posterior(evaluation_set, sample_ids, root_seed=...), with records carrying
    sample_id / theta / log_likelihood; or with arrays: design ids, theta rows, and a
    ForwardBatchResult or log-likelihoods in design order. Inputs are put in sample-id
    order, output id i draws from its own "posterior-resample" stream. Returns Samples."""
    from .workloads import sample_rng

    if hasattr(design_ids, "records"):  # the reference's call form
        sample_ids = theta
        design_ids, theta, evaluations, _ = _records(design_ids)
    ids = [int(i) for i in design_ids]
    out_ids = [int(i) for i in sample_ids]
    if len(set(ids)) != len(ids) or len(set(out_ids)) != len(out_ids):
        raise ValueError("sample IDs must be unique")
    if any(i < 0 for i in ids + out_ids) or isinstance(root_seed, bool) or root_seed < 0:
        raise ValueError("sample IDs and the root seed must be nonnegative integers")
    order = np.argsort(np.asarray(ids), kind="stable")
    ll = _logliks(evaluations)
    if ll.size != len(ids):
        raise ValueError("one evaluation per design sample is required")
    th = np.asarray(theta, dtype=np.float64)[order]
    w = posterior_weights(ll[order])
    u = [sample_rng(root_seed, i, "posterior-resample").random() for i in out_ids]
    picks = resample_indices(w, u)
    return tuple(Sample(i, tuple(float(x) for x in th[k])) for i, k in zip(out_ids, picks))


@dataclass(frozen=True)
class PredictiveSummary:
    """PredictiveSummary (statistics.py:262-274)."""
    sample_ids: tuple
    samples: tuple
    latent_mean: tuple
    latent_variance: tuple
    surrogate_variance: tuple
    discrepancy_variance: tuple
    observation_variance: tuple
    total_variance: tuple
    includes_surrogate_noise: bool
    includes_discrepancy: bool
    includes_observation_noise: bool


def predictive_moments(latent) -> tuple[np.ndarray, np.ndarray]:
    """Column mean and population variance of an n x d matrix, summed in numpy's order
    (rq_predictive_moments)."""
    x = np.ascontiguousarray(np.asarray(latent, dtype=np.float64))
    if x.ndim != 2 or x.shape[0] == 0 or x.shape[1] == 0:
        raise ValueError("successful predictions must be finite equal-length nonempty vectors")
    mean, var = np.empty(x.shape[1]), np.empty(x.shape[1])
    N.call("rq_predictive_moments", N.dptr(x), C.c_int64(x.shape[0]), C.c_int32(x.shape[1]),
           N.dptr(mean), N.dptr(var))
    return mean, var


def predictive_summary(sample_ids, predictions=None, *, root_seed: int, observation_sigma=None,
                       surrogate_variance=None, discrepancy_variance=None) -> PredictiveSummary:
    """predictive_summary (statistics.py:277-339) for converged evaluations, given as the
    reference takes them (an evaluation set whose records carry sample_id and
    predictions) or as sample ids and prediction rows: the equal-weight latent mixture's
    mean and variance (on the GPU, canonical sample-id order) plus the specified
    Gaussian components, and one noisy sample per evaluation from the reference's
    per-sample streams."""
    from .workloads import sample_rng

    if hasattr(sample_ids, "records"):  # the reference's call form
        sample_ids, _, _, predictions = _records(sample_ids)
    ids = [int(i) for i in sample_ids]
    if not ids:
        raise ValueError("at least one evaluation is required")
    if isinstance(root_seed, bool) or root_seed < 0:
        raise ValueError("root seed must be a nonnegative integer")
    latent = np.asarray(predictions, dtype=float)
    if latent.ndim != 2 or latent.shape[0] != len(ids) or latent.shape[1] == 0 \
            or not np.isfinite(latent).all():
        raise ValueError("successful predictions must be finite equal-length nonempty vectors")
    dimension = latent.shape[1]

    def component(value):
        result = np.zeros(dimension) if value is None else np.asarray(value, dtype=float)
        if result.shape != (dimension,) or not np.isfinite(result).all() or np.any(result < 0):
            raise ValueError("noise components must be finite nonnegative output-length vectors")
        return result

    observation = component(observation_sigma) ** 2
    surrogate, discrepancy = component(surrogate_variance), component(discrepancy_variance)
    samples = latent.copy()
    for i, sid in enumerate(ids):
        for purpose, variance in (("surrogate-noise", surrogate), ("discrepancy", discrepancy),
                                  ("observation-noise", observation)):
            if np.any(variance):
                samples[i] += sample_rng(root_seed, sid, purpose).normal(
                    0, np.sqrt(variance), dimension)
    canonical = latent[np.argsort(ids)]
    mean, variance = predictive_moments(canonical)
    total = variance + surrogate + discrepancy + observation
    if not np.isfinite(samples).all() or not np.isfinite(total).all():
        raise ValueError("predictive samples and total variance must be finite")
    return PredictiveSummary(tuple(ids), tuple(tuple(float(x) for x in row) for row in samples),
                             tuple(mean), tuple(variance), tuple(surrogate), tuple(discrepancy),
                             tuple(observation), tuple(total), bool(np.any(surrogate)),
                             bool(np.any(discrepancy)), bool(np.any(observation)))


def conformal_quantile(scores, alpha: float) -> float:
    """conformal_quantile (statistics.py:349-355): the ceil((n+1)(1-alpha))-th smallest
    score, or +inf when that rank exceeds n (rq_conformal_quantile)."""
    v = np.ascontiguousarray(np.asarray(scores, dtype=np.float64))
    if v.ndim != 1 or v.size == 0 or not np.isfinite(v).all():
        raise ValueError("conformal scores must be a finite nonempty vector")
    q = C.c_double()
    N.call("rq_conformal_quantile", N.dptr(v), C.c_int64(v.size), C.c_double(alpha),
           C.byref(q))
    return float(q.value)


def split_conformal_intervals(calibration_y, calibration_prediction, test_prediction, *,
                              alpha: float):
    """split_conformal_intervals (statistics.py:358-378): test predictions -/+ the
    conformal quantile of the calibration set's absolute residuals (rq_split_conformal)."""
    y = np.ascontiguousarray(np.asarray(calibration_y, dtype=np.float64))
    p = np.ascontiguousarray(np.asarray(calibration_prediction, dtype=np.float64))
    t = np.ascontiguousarray(np.asarray(test_prediction, dtype=np.float64))
    for a, name in ((y, "calibration targets"), (p, "calibration predictions"),
                    (t, "test predictions")):
        if a.ndim != 1 or a.size == 0 or not np.isfinite(a).all():
            raise ValueError(f"{name} must be a finite nonempty vector")
    if y.shape != p.shape:
        raise ValueError("calibration target and prediction shapes must match")
    lo, hi = np.empty_like(t), np.empty_like(t)
    N.call("rq_split_conformal", N.dptr(y), N.dptr(p), C.c_int64(y.size), N.dptr(t),
           C.c_int64(t.size), C.c_double(alpha), N.dptr(lo), N.dptr(hi))
    return lo, hi
