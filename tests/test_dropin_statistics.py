"""Drop-in check of the Python boundary: the reference's own statistics layer
(rans-uq/python/cfdr/statistics.py, loaded from the reference sources where they
are present) runs unchanged with this package standing in for the compiled
cfdr._core. evaluate_batch type-checks the batch against _core.ForwardBatch and
reads every row's status name, predictions, log_lik, simple_iters and error, which
must all be this package's result types. No GPU is used: the batch's rows are built
by the same decoding the GPU path uses (_rows_from_native over rq_row_out records),
and posterior_weights / resample_posterior / predictive_summary then run on them."""
import os
import importlib.util
import sys
import types
from pathlib import Path

import numpy as np
import pytest

import rans_uq_b200 as rq
import rans_uq_b200._native as N
from rans_uq_b200 import core

REF = Path(os.environ.get("RQ_REFERENCE_DIR", "/root/reference"))
pytestmark = pytest.mark.skipif(not (REF / "rans-uq/python/cfdr/statistics.py").exists(),
                                reason="reference sources not present")


def reference_statistics():
    pkg = types.ModuleType("cfdr")
    pkg.__path__ = [str(REF / "rans-uq" / "python" / "cfdr")]
    saved = {k: sys.modules.get(k) for k in ("cfdr", "cfdr._core", "cfdr.statistics")}
    sys.modules["cfdr"], sys.modules["cfdr._core"] = pkg, rq
    pkg._core = rq
    try:
        spec = importlib.util.spec_from_file_location(
            "cfdr.statistics", REF / "rans-uq/python/cfdr/statistics.py")
        stats = importlib.util.module_from_spec(spec)
        sys.modules["cfdr.statistics"] = stats
        spec.loader.exec_module(stats)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return stats


def fake_batch(statuses, logliks, n_obs=3):
    """A ForwardBatch whose evaluate decodes native rq_row_out records, as the GPU path
    does after its launch."""
    batch = object.__new__(core.ForwardBatch)

    def evaluate(theta, workers=1):
        theta = np.asarray(theta)
        out = []
        pred = np.zeros((len(theta), n_obs))
        for i, (st, ll) in enumerate(zip(statuses, logliks)):
            r = N.RowOut()
            r.status, r.iterations, r.loglik = int(st), 100 + i, ll
            out.append(r)
            pred[i] = theta[i, 0] * np.arange(1, n_obs + 1)
        return core.ForwardBatchResult(core._rows_from_native(out, pred, n_obs, 2), n_obs)

    batch.evaluate = evaluate
    return batch


def test_reference_statistics_run_on_this_packages_batch():
    stats = reference_statistics()
    samples = stats.independent_uniform_design(range(6), (0.28, 0.084), (0.34, 0.096),
                                               root_seed=7)
    lls = [-3.0, -1.5, -2.0, -7.0, -1.0, -4.0]
    ev = stats.evaluate_batch(samples, fake_batch([0] * 6, lls), workers=1)
    assert [r.status for r in ev.records] == ["Converged"] * 6
    assert [r.log_likelihood for r in ev.records] == lls
    assert [r.iterations for r in ev.records] == list(range(100, 106))
    np.testing.assert_allclose(ev.records[2].predictions,
                               samples[2].theta[0] * np.arange(1, 4))
    w = stats.posterior_weights(ev)
    assert abs(w.sum() - 1.0) < 1e-15 and int(np.argmax(w)) == 4
    draws = stats.resample_posterior(ev, range(100, 110), root_seed=3)
    assert len(draws) == 10 and all(d.theta in {s.theta for s in samples} for d in draws)
    summary = stats.predictive_summary(ev, root_seed=5, observation_sigma=[0.1, 0.2, 0.3])
    assert len(summary.samples) == 6 and summary.includes_observation_noise


def test_reference_statistics_see_failed_rows_as_failures():
    stats = reference_statistics()
    samples = stats.independent_uniform_design(range(4), (0.28, 0.084), (0.34, 0.096),
                                               root_seed=7)
    st = [core.EvaluationStatus.Converged, core.EvaluationStatus.DivergenceDetected,
          core.EvaluationStatus.InvalidParameters, core.EvaluationStatus.Unconverged]
    ev = stats.evaluate_batch(samples, fake_batch(st, [-1.0, -1e6, -1e30, -2.0]))
    assert [r.status for r in ev.records] == ["Converged", "DivergenceDetected",
                                              "InvalidParameters", "Unconverged"]
    assert ev.failure_count == 3
    assert ev.records[1].predictions == () and ev.records[2].predictions == ()
    with pytest.raises(ValueError, match="unresolved"):
        stats.posterior_weights(ev)
