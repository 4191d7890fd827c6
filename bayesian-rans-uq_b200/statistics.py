"""Posterior weights of a calibration stage on the GPU, in FP64: the
importance-weight step of cfdr.statistics.posterior_weights
(rans-uq/python/cfdr/statistics.py:208-232) with the optional proposal density
of the Student-t importance stage (docs/figures/calibration_coverage.py:165-180).
"""
from __future__ import annotations

import ctypes as C

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
