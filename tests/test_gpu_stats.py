"""Posterior weights on the GPU (rq_posterior_weights) against the reference's
rule restated on the host (cfdr.statistics.posterior_weights,
rans-uq/python/cfdr/statistics.py:217-232: exp(l - max) / math.fsum). The device
sums with compensated FP64 arithmetic: weights agree to 4 ulp-level relative
error (1e-15) and sum to one."""
import math

import numpy as np
import pytest

import rans_uq_b200.statistics as st

pytestmark = pytest.mark.gpu


def reference_weights(ll, lq=None):
    v = [a - (b if lq is not None else 0.0) for a, b in zip(ll, lq if lq is not None else ll)]
    m = max(v)
    w = [math.exp(x - m) for x in v]
    s = math.fsum(w)
    return np.asarray(w) / s, m + math.log(s)


@pytest.mark.parametrize("n", [1, 7, 256, 100003])
def test_weights_match_reference_rule(n):
    rng = np.random.default_rng(n)
    ll = -0.5 * rng.chisquare(30, n) * rng.uniform(0.5, 40.0)
    lq = rng.normal(0.0, 3.0, n)
    for q in (None, lq):
        w, ev = st.posterior_weights(ll, q, return_log_evidence=True)
        want, ev_ref = reference_weights(ll, q)
        np.testing.assert_allclose(w, want, rtol=1e-15, atol=0)
        assert abs(ev - ev_ref) <= 1e-14 * max(1.0, abs(ev_ref))
        assert abs(math.fsum(w) - 1.0) < 1e-14


def test_nonfinite_loglik_rejected():
    with pytest.raises(ValueError, match="finite"):
        st.posterior_weights(np.array([-1.0, np.nan, -3.0]))
    with pytest.raises(ValueError, match="finite"):
        st.posterior_weights(np.array([-1.0, -np.inf]))


# ---- resampling, predictive moments and split conformal (rq_resample_indices,
# rq_predictive_moments, rq_conformal_quantile, rq_split_conformal) against the
# reference's own cfdr.statistics functions (fixture tests/golden/statistics_ref.npz,
# written by tests/golden/make_statistics_golden.py) and numpy: exact equality, since
# the device reproduces numpy's summation order and rounding.
from pathlib import Path  # noqa: E402

from rans_uq_b200.workloads import sample_rng  # noqa: E402

REF = np.load(Path(__file__).parent / "golden" / "statistics_ref.npz")


def test_resample_indices_equal_numpy_choice():
    rng = np.random.default_rng(3)
    for n in (1, 2, 9, 300, 20000):
        w = rng.exponential(size=n) ** 3
        w /= w.sum()
        ids = range(100, 400)
        u = [sample_rng(11, i, "posterior-resample").random() for i in ids]
        want = [int(sample_rng(11, i, "posterior-resample").choice(n, p=w)) for i in ids]
        np.testing.assert_array_equal(st.resample_indices(w, u), want)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_resample_posterior_matches_reference(tag):
    draws = st.resample_posterior(REF[f"{tag}_ids"], REF[f"{tag}_theta"], REF[f"{tag}_ll"],
                                  REF[f"{tag}_resample_ids"], root_seed=20261010)
    assert [d.sample_id for d in draws] == REF[f"{tag}_resample_ids"].tolist()
    np.testing.assert_array_equal(np.array([d.theta for d in draws]),
                                  REF[f"{tag}_resample_theta"])


def _evaluation_set(tag):
    """An object shaped as cfdr.statistics.EvaluationSet (records with sample_id, theta,
    status, error, log_likelihood, predictions), from the fixture's ensemble."""
    from types import SimpleNamespace

    recs = [SimpleNamespace(sample_id=int(i), theta=tuple(t), status="Converged", error="",
                            log_likelihood=float(ll), predictions=tuple(p))
            for i, t, ll, p in zip(REF[f"{tag}_ids"], REF[f"{tag}_theta"], REF[f"{tag}_ll"],
                                   REF[f"{tag}_pred"])]
    return SimpleNamespace(records=tuple(recs))


@pytest.mark.parametrize("tag", ["a", "c"])
def test_reference_call_forms(tag):
    """resample_posterior(evaluation_set, ids, root_seed=) and
    predictive_summary(evaluation_set, ...) as the reference is called."""
    ev = _evaluation_set(tag)
    draws = st.resample_posterior(ev, REF[f"{tag}_resample_ids"], root_seed=20261010)
    np.testing.assert_array_equal(np.array([d.theta for d in draws]),
                                  REF[f"{tag}_resample_theta"])
    d = REF[f"{tag}_pred"].shape[1]
    s = st.predictive_summary(ev, root_seed=77, observation_sigma=REF[f"{tag}_sigma"],
                              surrogate_variance=np.full(d, 0.01))
    np.testing.assert_array_equal(np.array(s.samples), REF[f"{tag}_samples"])
    np.testing.assert_array_equal(np.array(s.latent_variance), REF[f"{tag}_latent_variance"])
    bad = _evaluation_set(tag)
    bad.records[0].status = "DivergenceDetected"
    with pytest.raises(ValueError, match="unresolved"):
        st.resample_posterior(bad, [1], root_seed=1)


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_predictive_summary_matches_reference(tag):
    d = REF[f"{tag}_pred"].shape[1]
    s = st.predictive_summary(REF[f"{tag}_ids"], REF[f"{tag}_pred"], root_seed=77,
                              observation_sigma=REF[f"{tag}_sigma"],
                              surrogate_variance=np.full(d, 0.01))
    np.testing.assert_array_equal(np.array(s.latent_mean), REF[f"{tag}_latent_mean"])
    np.testing.assert_array_equal(np.array(s.latent_variance), REF[f"{tag}_latent_variance"])
    np.testing.assert_array_equal(np.array(s.total_variance), REF[f"{tag}_total_variance"])
    np.testing.assert_array_equal(np.array(s.samples), REF[f"{tag}_samples"])
    assert s.includes_surrogate_noise and s.includes_observation_noise
    assert not s.includes_discrepancy


@pytest.mark.parametrize("n", [1, 19, 1000, 20000])
def test_conformal_quantile_matches_reference(n):
    got = [st.conformal_quantile(REF[f"scores_{n}"], a) for a in (0.05, 0.1, 0.5, 0.9)]
    np.testing.assert_array_equal(got, REF[f"quantile_{n}"])


def test_split_conformal_matches_reference():
    lo, hi = st.split_conformal_intervals(REF["cal_y"], REF["cal_p"], REF["test_p"], alpha=0.1)
    np.testing.assert_array_equal(lo, REF["split_lo"])
    np.testing.assert_array_equal(hi, REF["split_hi"])


def test_statistics_reject_what_the_reference_rejects():
    with pytest.raises(ValueError, match="sum to 1"):
        st.resample_indices([0.5, 0.6], [0.1])
    with pytest.raises(ValueError, match="non-negative"):
        st.resample_indices([1.5, -0.5], [0.1])
    with pytest.raises(ValueError, match="nonnegative"):
        st.conformal_quantile([1.0, -2.0], 0.1)
    with pytest.raises(ValueError, match="alpha"):
        st.conformal_quantile([1.0, 2.0], 1.0)
    assert st.conformal_quantile([3.0, 1.0, 2.0], 0.05) == np.inf  # rank 4 > n


def test_weight_parts_match_weights():
    """rq_posterior_weights_parts: the same weights as rq_posterior_weights, with the
    log-sum-exp split into its maximum and its scaled sum (the inputs of the sharded
    combination in rans_uq_b200.replicas, whose two-rank collectives are tested on CPU)."""
    rng = np.random.default_rng(8)
    ll = -0.5 * rng.chisquare(30, 5000) * 9.0
    lq = rng.normal(0.0, 2.0, 5000)
    w, ev = st.posterior_weights(ll, lq, return_log_evidence=True)
    w2, m, s = st.posterior_weight_parts(ll, lq)
    np.testing.assert_array_equal(w2, w)
    assert m == np.max(ll - lq)
    assert abs(m + math.log(s) - ev) <= 1e-15 * abs(ev)
