"""Calibration stages with the importance weights on the GPU: the same results as
the reference's stage functions on the analytic log-likelihood of the golden
vectors (weights to 1e-14 relative: the device's compensated FP64 sum against
math.fsum)."""
import pytest

import rans_uq_b200.calibration as cal
import test_calibration_host as host

pytestmark = pytest.mark.gpu


def test_stages_with_gpu_weights_match_reference_functions():
    out = cal.calibrate(host.evaluator)
    host.check(out, 1e-14)


def test_study_with_gpu_statistics_matches_reference():
    """The whole study with the GPU weights, predictive moments and split-conformal
    quantile: the same ranges, recalibration and coverage as the reference's calibrate()."""
    from test_calibration_host import STUDY, check_study, study_evaluator

    out = cal.calibrate(study_evaluator, truth=STUDY["truth"], sigma=STUDY["sigma"])
    check_study(out.study)
