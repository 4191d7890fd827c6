"""Warm starts of the sequential ForwardModel on the GPU (WarmStartCache,
rans-uq/include/ForwardModel.hpp:21-157; lookup and store in
ForwardModel::evaluateWithDiagnostics, rans-uq/src/ForwardModel.cpp:79-82, 114-117).

One model evaluates the same theta sequence as the compiled reference did for the
golden fixtures (tests/golden/make_golden.py): which calls start warm, the verdicts
and iteration counts (including the reference's Diverged-after-5-iterations verdict
of a warm start next to a converged state) and the cache's retained bytes must be
identical; predictions and log-likelihoods of converged calls agree to 1e-10
relative, as cold converged solves do. The cached states never leave the device.
"""
import numpy as np
import pytest

import cases
from oracle import checker as ck

pytestmark = pytest.mark.gpu
GOLDEN = cases.__file__.replace("cases.py", "golden/")
RTOL = 1e-10


def run_sequence(rq, thetas, budget=None, case=None):
    model = cases.product_batch(rq, case or cases.small_channel(), model_class=rq.ForwardModel)
    if budget is not None:
        model.cache().set_byte_budget(budget)
    out = []
    for th in thetas:
        ev = model.evaluate_with_diagnostics(th)
        out.append((ck.STATUS[int(ev.result.status)], ev.result.simple_iters, ev.used_warm_start,
                    model.cache().retained_bytes(), ev.result.log_lik,
                    np.asarray(ev.result.predictions, float), ev.fields))
    return model, out


def check_against(golden, out):
    g = np.load(GOLDEN + golden + ".npz")
    for i, (status, iters, warm, kept, ll, pred, _) in enumerate(out):
        assert status == str(g["status"][i]), (i, status, g["status"][i])
        assert iters == int(g["iterations"][i]), (i, iters, g["iterations"][i])
        assert warm == bool(g["used_warm"][i]), i
        assert kept == int(g["retained"][i]), i
        if status == "Converged":
            assert abs(ll - g["loglik"][i]) <= RTOL * abs(g["loglik"][i]), i
            np.testing.assert_allclose(pred, g["predictions"][i], rtol=RTOL, atol=0)
        else:
            assert ll == g["loglik"][i]


def test_warm_sequence_matches_reference(rq):
    model, out = run_sequence(rq, cases.WARM_SEQUENCE)
    check_against("warm_sequence_ref", out)
    assert model.cache().size() == 2


def test_byte_budget_evicts_oldest(rq):
    model, out = run_sequence(rq, cases.WARM_BUDGET_SEQUENCE, budget=cases.WARM_BUDGET_BYTES)
    check_against("warm_budget_ref", out)
    assert model.cache().size() == 1 and model.cache().byte_budget() == cases.WARM_BUDGET_BYTES


def test_warm_start_from_own_state_matches_oracle(rq):
    """The same theta twice: the second solve starts from the first one's device state and
    stops at the turbulence start; its fields equal the oracle's second call."""
    case = cases.small_channel()
    th = [(0.31, 0.09), (0.31, 0.09)]
    want = ck.solve_sequence(case, th, "oracle")
    _, out = run_sequence(rq, th)
    assert [o[0] for o in out] == want.status and [o[1] for o in out] == list(want.iterations)
    assert [o[2] for o in out] == [False, True]
    np.testing.assert_allclose(out[1][5], want.predictions[1], rtol=RTOL, atol=0)


def test_cache_api_and_unconverged_not_stored(rq):
    model, out = run_sequence(rq, [(0.31, 0.09), (0.31, 0.09)],
                              case=cases.small_channel(max_iter=200))
    assert [o[0] for o in out] == ["Unconverged", "Unconverged"]
    assert [o[2] for o in out] == [False, False] and model.cache().size() == 0
    model2, _ = run_sequence(rq, [(0.2, 0.05)])
    c = model2.cache()
    assert c.size() == 1 and c.retained_bytes() == 6880
    assert c.byte_budget() == 64 * 1024 * 1024
    c.set_byte_budget(100)  # below one entry: evicted
    assert c.size() == 0 and c.retained_bytes() == 0
    c.set_byte_budget(1 << 20)
    ev = model2.evaluate_with_diagnostics((0.2, 0.05))
    assert not ev.used_warm_start and c.size() == 1
    c.clear()
    assert c.size() == 0 and c.retained_bytes() == 0
    with pytest.raises(ValueError):
        rq.WarmStartCache(model2._batch._problem, -1, 0.5)


@pytest.mark.parametrize("fixture,max_iter,rtol", [("snapshot_small_channel_ref", 60000, 1e-10),
                                                   ("snapshot_small_channel_capped_ref", 300, 1e-9)])
def test_snapshot_matches_reference(rq, fixture, max_iter, rtol):
    """evaluate_with_diagnostics(theta, snapshot=True) against the reference's
    OwnedFlowSnapshot (ForwardModel.hpp:162-186) of the same cold solve: cell fields,
    boundary-face values, face fluxes in the mesh's face order, and the turbulence marker
    (False for a solve capped before the end of the start-up floor window)."""
    g = np.load(GOLDEN + fixture + ".npz")
    case = cases.small_channel(max_iter=max_iter)
    model = cases.product_batch(rq, case, model_class=rq.ForwardModel)
    ev = model.evaluate_with_diagnostics((case.coeffs[9], case.coeffs[8]), snapshot=True)
    assert ck.STATUS[int(ev.result.status)] == str(g["status"])
    assert ev.result.simple_iters == int(g["iterations"])
    s = ev.snapshot
    assert s["turb_established"] == bool(g["turb_established"])
    cells, bnd = g["cells"], g["boundary"]
    np.testing.assert_array_equal(s["U"][:, 2], 0.0)
    uscale = np.max(np.abs(cells[0]))
    assert np.max(np.abs(s["U"][:, 0] - cells[0])) <= rtol * uscale
    assert np.max(np.abs(s["U"][:, 1] - cells[1])) <= rtol * uscale
    assert np.max(np.abs(s["p"] - cells[3])) < 1e-9  # round-off noise in a periodic channel
    for i, name in ((4, "k"), (5, "omega"), (6, "nuT"), (7, "F1"), (8, "F2"), (9, "Pk"),
                    (10, "CDkw")):
        scale = max(np.max(np.abs(cells[i])), 1e-300)
        assert np.max(np.abs(s[name] - cells[i])) <= rtol * scale, name
    b = s["boundary"]
    np.testing.assert_array_equal(b["U"], bnd[0:3].T)
    for i, name in ((4, "k"), (6, "nuT"), (7, "F1"), (8, "F2"), (9, "Pk"), (10, "CDkw")):
        np.testing.assert_array_equal(b[name], bnd[i], err_msg=name)
    np.testing.assert_allclose(b["omega"], bnd[5], rtol=1e-14, atol=0)
    assert np.max(np.abs(b["p"] - bnd[3])) < 1e-9
    flux = g["face_fluxes"]
    assert s["face_fluxes"].shape == flux.shape
    assert np.max(np.abs(s["face_fluxes"] - flux)) <= rtol * np.max(np.abs(flux))


def test_no_snapshot_for_invalid_parameters(rq):
    model = cases.product_batch(rq, cases.small_channel(), model_class=rq.ForwardModel)
    ev = model.evaluate_with_diagnostics((0.95, 0.09), snapshot=True)
    assert ev.result.status.name == "InvalidParameters" and ev.snapshot is None


def test_last_fields_as_the_reference_binding_returns_them(rq):
    """last_fields() is the binding's dict (extractFields, bindings.cpp:272-287);
    set_retain_last_fields(False) drops and stops keeping them (ForwardModel.hpp:221-227)."""
    case = cases.small_channel(max_iter=50)
    model = cases.product_batch(rq, case, model_class=rq.ForwardModel)
    ev = model.evaluate_with_diagnostics((0.31, 0.09))
    assert ev.result.status.name == "Unconverged" and model.has_last_fields()
    lf = model.last_fields()
    assert set(lf) == {"U", "p", "k", "omega", "nuT", "F1", "F2", "Pk", "CDkw"}
    assert lf["U"].shape == (case.n_cells, 3)
    np.testing.assert_array_equal(lf["U"][:, 0], ev.fields[0])
    np.testing.assert_array_equal(lf["omega"], ev.fields[5])
    model.set_retain_last_fields(False)
    assert not model.has_last_fields()
    model.evaluate((0.31, 0.09))
    assert not model.has_last_fields()
    with pytest.raises(RuntimeError, match="No fields available"):
        model.last_fields()
    assert model.param_set() is not None and not model.has_target_anisotropy()


def test_diverged_call_reports_no_state(rq):
    """A warm start that the reference classifies Diverged leaves no valid state: the C
    ABI's fields buffer comes back NaN (not the previous solve's state), and no snapshot
    or last fields are kept."""
    import ctypes as C

    import rans_uq_b200._native as N

    model = cases.product_batch(rq, cases.small_channel(), model_class=rq.ForwardModel)
    assert model.evaluate((0.2, 0.05)).status.name == "Converged"
    nc = model._batch._problem.n_cells
    fields = np.zeros((11, nc))
    pred = np.zeros(8)
    row = N.RowOut()
    used = C.c_int32()
    theta = np.array([0.21, 0.052])
    N.call("rq_evaluate_cached", model.cache().handle, N.dptr(theta), C.byref(row),
           N.dptr(pred), N.dptr(fields), None, None, None, C.byref(used))
    assert row.status == 2 and used.value == 1
    assert np.isnan(fields).all()
    ev = model.evaluate_with_diagnostics((0.21, 0.052), snapshot=True)
    assert ev.result.status.name == "DivergenceDetected" and ev.snapshot is None
    assert not model.has_last_fields()
