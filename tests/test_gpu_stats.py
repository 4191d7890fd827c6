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
