"""Handles belong to the device that was current when they were created: a call made
with another device current is rejected (RQ_E_INVALID) before anything is launched,
and destroy works from any device. Needs two GPUs; on one GPU only the same-device
path is exercised."""
import ctypes as C

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def test_same_device_calls_run(rq):
    batch = cases.product_batch(rq, cases.small_channel(max_iter=5))
    res = batch.evaluate(np.array([[0.31, 0.09]]))
    assert res.rows[0].result.simple_iters == 5


def test_other_device_is_rejected(rq):
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    torch.cuda.set_device(0)
    batch = cases.product_batch(rq, cases.small_channel(max_iter=5))
    L = rq.lib()
    theta = np.array([0.31, 0.09])
    rows = (rq._native.RowOut * 1)()
    pred = np.zeros(max(batch.n_observations(), 1))
    try:
        torch.cuda.set_device(1)
        rc = L.rq_evaluate_batch(batch._problem.handle, rq._native.dptr(theta), C.c_int64(1),
                                 rows, rq._native.dptr(pred), None, None, C.c_int32(0))
        assert rc == -1 and b"current device" in L.rq_last_error()
    finally:
        torch.cuda.set_device(0)
