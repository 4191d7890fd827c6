"""Host-side admission of the posterior weights (no GPU): a stage with any row
that is not Converged has no posterior, as in cfdr.statistics._resolved
(rans-uq/python/cfdr/statistics.py:208-214), and empty input is rejected."""
import numpy as np
import pytest

import rans_uq_b200 as rq
import rans_uq_b200.statistics as st


def result(statuses):
    rows = [rq.ForwardBatchRow(rq.EvaluationResult(rq.EvaluationStatus[s], -1.0 * k, np.ones(2), 10),
                               0.0, 0.9, False, "") for k, s in enumerate(statuses)]
    return rq.ForwardBatchResult(rows, 2)


def test_unresolved_rows_have_no_posterior():
    with pytest.raises(ValueError, match="1 unresolved"):
        st.posterior_weights(result(["Converged", "Unconverged", "Converged"]))
    with pytest.raises(ValueError, match="required"):
        st.posterior_weights(np.zeros(0))
    with pytest.raises(ValueError, match="one value per evaluation"):
        st.posterior_weights(np.zeros(3), log_q=np.zeros(2))
