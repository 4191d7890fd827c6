"""rq_evaluate_noalloc: one draw solved in the library's fixed scratch array, for
callers that must not allocate GPU memory while they run (a sampler inside a
host application with a memory budget fixed at start-up, or a latency-bound
loop where cudaMalloc would stall the device). Called through the C ABI with
device buffers the test owns; its rows must equal rq_evaluate_batch's for the
same draws on two calls in a row (tolerance 1e-12 relative; the same per-solve
code runs at the same CTA size, so the results are expected to be bitwise
equal). A mesh class whose scratch exceeds the fixed 8 MiB is rejected.

The file name sorts last so that a run stopping at its first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _noalloc_two_calls(rq, case, thetas):
    import torch

    batch = cases.product_batch(rq, case)
    want = batch.evaluate(thetas).rows
    L = rq.lib()
    handle = batch._problem.handle
    n_obs = batch.n_observations()
    dev = torch.device("cuda", 0)
    theta_dev = torch.zeros(2, dtype=torch.float64, device=dev)
    row_dev = torch.zeros(40, dtype=torch.uint8, device=dev)
    pred_dev = torch.zeros(n_obs, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    for k in range(2):  # two calls in a row share the scratch array
        theta_dev.copy_(torch.from_numpy(thetas[k]))
        torch.cuda.synchronize()
        rc = L.rq_evaluate_noalloc(handle, C.c_void_p(theta_dev.data_ptr()),
                                   C.c_void_p(row_dev.data_ptr()), C.c_void_p(pred_dev.data_ptr()),
                                   C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.rq_last_error()
        torch.cuda.synchronize()
        row = rq.rows_from_device_bytes(row_dev.cpu().numpy())[0]
        ref = want[k].result
        assert int(row["status"]) == int(ref.status)
        assert int(row["iterations"]) == ref.simple_iters
        assert abs(float(row["loglik"]) - ref.log_lik) <= RTOL * abs(ref.log_lik)
        np.testing.assert_allclose(pred_dev.cpu().numpy(), ref.predictions, rtol=RTOL, atol=0)
    return want


def test_noalloc_matches_batch_on_two_calls(rq):
    """The 72-cell class: 512-thread CTA, whole working set in the shared-memory arena;
    both draws converge."""
    thetas = np.array([[0.31, 0.09], [0.30, 0.088]])
    want = _noalloc_two_calls(rq, cases.small_channel(), thetas)
    assert all(int(w.result.status) == 0 for w in want)


def test_noalloc_matches_batch_above_768_cells(rq):
    """The 1536-cell class (3 x 512, Re_tau 1000): 768-thread CTA, no arena, the
    scratch array holding every array of the solve; capped at 40 outer iterations
    (Unconverged rows carry their predictions too)."""
    case = cases.small_channel(ny=512, re_tau=1000.0, nu=1e-3, yplus=0.5, max_iter=40)
    thetas = np.array([[0.31, 0.09], [0.33, 0.092]])
    want = _noalloc_two_calls(rq, case, thetas)
    assert all(w.result.simple_iters == 40 for w in want)


def test_noalloc_rejects_mesh_above_scratch(rq):
    import torch

    big = cases.product_batch(rq, cases.small_channel(ny=8000, max_iter=1))
    dev = torch.device("cuda", 0)
    buf = torch.zeros(64, dtype=torch.float64, device=dev)
    L = rq.lib()
    rc = L.rq_evaluate_noalloc(big._problem.handle, C.c_void_p(buf.data_ptr()),
                               C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), None)
    assert rc == -1  # RQ_E_INVALID
    assert b"at most" in L.rq_last_error()
