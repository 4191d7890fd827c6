"""The device-buffer entry points against their host-buffer twins, on the GPU:
rq_evaluate_multi_device (θ, rows and predictions in device memory, queued on a
stream; the benchmark's call) equals rq_evaluate_multi bitwise, with a sane clock
record per row; rq_posterior_weights_device equals rq_posterior_weights; and
rq_problem_info describes the class."""
import ctypes as C

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def test_multi_device_equals_multi(rq):
    import torch

    a = cases.product_batch(rq, cases.small_channel())
    b = cases.product_batch(rq, cases.small_channel(ny=32, re_tau=250.0, nu=1 / 250.0))
    cls = np.array([0, 1, 1, 0], dtype=np.int32)
    theta = np.array([[0.31, 0.09], [0.30, 0.088], [0.95, 0.09], [0.29, 0.085]])
    host = rq.evaluate_multi([a, b], cls, theta)
    dev = torch.device("cuda", 0)
    th = torch.tensor(theta, dtype=torch.float64, device=dev)
    rows = torch.zeros(len(theta) * 40, dtype=torch.uint8, device=dev)
    pred = torch.zeros((len(theta), 8), dtype=torch.float64, device=dev)
    clock = torch.zeros((len(theta), 12), dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rq.evaluate_multi_device([a, b], cls, th.data_ptr(), rows.data_ptr(), pred.data_ptr(),
                             stream.cuda_stream, clock.data_ptr())
    torch.cuda.synchronize()
    recs = rq.rows_from_device_bytes(rows.cpu().numpy())
    p = pred.cpu().numpy()
    ck = clock.cpu().numpy()
    for i, r in enumerate(host.rows):
        assert int(recs["status"][i]) == int(r.result.status)
        assert int(recs["iterations"][i]) == r.result.simple_iters
        if r.result.status.name == "Converged":
            np.testing.assert_array_equal(p[i], r.result.predictions)
            assert float(recs["loglik"][i]) == r.result.log_lik
            assert ck[i, 1] > ck[i, 0] > 0 and ck[i, 2] > 0 and ck[i, 3] > 0
    assert recs["status"][2] == 3  # out of bounds: InvalidParameters


def test_posterior_weights_device_equals_host(rq):
    import torch

    import rans_uq_b200.statistics as st

    rng = np.random.default_rng(4)
    ll = -0.5 * rng.chisquare(10, 3000) * 7.0
    lq = rng.normal(0.0, 1.0, 3000)
    want, ev = st.posterior_weights(ll, lq, return_log_evidence=True)
    dev = torch.device("cuda", 0)
    dl, dq = torch.tensor(ll, device=dev), torch.tensor(lq, device=dev)
    w = torch.empty(3000, dtype=torch.float64, device=dev)
    out = torch.empty(3, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = rq.lib().rq_posterior_weights_device(C.c_void_p(dl.data_ptr()),
                                              C.c_void_p(dq.data_ptr()), 3000,
                                              C.c_void_p(w.data_ptr()),
                                              C.c_void_p(out.data_ptr()),
                                              C.c_void_p(stream.cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(w.cpu().numpy(), want)
    m, s, bad = out.cpu().numpy()
    assert bad == 0 and abs(m + np.log(s) - ev) <= 1e-15 * abs(ev)


def test_problem_info(rq):
    batch = cases.product_batch(rq, cases.small_channel())
    n, no, na, lev = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
    assert rq.lib().rq_problem_info(batch._problem.handle, C.byref(n), C.byref(no), C.byref(na),
                                    C.byref(lev)) == 0
    assert (n.value, no.value, na.value) == (72, 8, 2) and lev.value >= 1
