"""The launch-shape autotuner (rq_problem_tune): it times capped solves of the mesh
class for every candidate CTA size and shared-memory arena, applies the fastest, and
the tuned class gives the default class's results -- verdict and iteration count
identical, predictions and log-likelihood within 1e-10 relative. A different CTA size
changes only the order of the block sums, so the outer iteration at which the
convergence test first passes may move by a few iterations (allowed: 1 %)."""
import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def test_tuner_measures_candidates_and_applies_the_fastest(rq):
    batch = cases.product_batch(rq, cases.small_channel(max_iter=20000))
    chosen, measured = batch.tune(theta=[0.31, 0.09], iters=50,
                                  candidates=[(256, 0), (512, -1), (768, 0), (1024, -1)])
    assert len(measured) == 4
    times = [m[2] for m in measured]
    assert all(t > 0 for t in times), measured
    best = min(range(4), key=lambda k: times[k])
    assert chosen == measured[best][:2]
    assert batch.launch() == chosen


def test_tuned_class_matches_default(rq):
    thetas = np.array([[0.31, 0.09], [0.30, 0.088]])
    default = cases.product_batch(rq, cases.small_channel())
    tuned = cases.product_batch(rq, cases.small_channel())
    chosen, _ = tuned.tune(theta=thetas[0], iters=50)   # the library's own candidate set
    want = default.evaluate(thetas).rows
    got = tuned.evaluate(thetas).rows
    for w, g in zip(want, got):
        assert g.result.status == w.result.status == rq.EvaluationStatus.Converged
        assert abs(g.result.simple_iters - w.result.simple_iters) <= 0.01 * w.result.simple_iters
        np.testing.assert_allclose(g.result.predictions, w.result.predictions, rtol=RTOL, atol=0)
        assert abs(g.result.log_lik - w.result.log_lik) <= RTOL * abs(w.result.log_lik)
    # every shape of the built-in set gives the same verdicts
    for block, arena in ((256, 0), (768, 0)):
        tuned.set_launch(block, arena)
        for w, g in zip(want, tuned.evaluate(thetas).rows):
            assert g.result.status == w.result.status
            np.testing.assert_allclose(g.result.predictions, w.result.predictions, rtol=RTOL,
                                       atol=0)


def test_set_launch_rejects_unknown_block(rq):
    batch = cases.product_batch(rq, cases.small_channel(max_iter=5))
    with pytest.raises(ValueError):
        batch.set_launch(300, 0)
