"""GPU parity of the B200 forward model against the CPU checkers.

* Trajectory parity: the fields after N outer iterations equal the C++
  restatement (oracle/rq_oracle.cpp) run with the same linear solvers, to
  round-off (rtol 1e-9 on the max-norm; the differences are reduction order).
* Converged parity: converged profiles equal the compiled reference's own
  ForwardModel (golden fixtures made by tests/golden/make_golden.py) to 1e-10
  relative, with identical convergence verdicts.
"""
import numpy as np
import pytest

import cases
from oracle import checker as ck

pytestmark = pytest.mark.gpu

GOLDEN = cases.__file__.replace("cases.py", "golden/")
RTOL_TRAJ = 1e-9
RTOL_CONV = 1e-10


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("solver,ps", [("AMG", ck.P_AMG), ("PCG", ck.P_PCG)])
@pytest.mark.parametrize("n_iter", [1, 7, 40])
def test_fields_after_n_iterations(rq, checker, solver, ps, n_iter):
    case = cases.small_channel(max_iter=n_iter, pressure_solver=ps)
    want = checker.solve(case, "oracle", hist_cap=n_iter)
    batch = cases.product_batch(rq, case, pressure_solver=solver)
    res, fields, hist = batch.evaluate_fields([[case.coeffs[9], case.coeffs[8]]], hist_cap=n_iter)
    row = res.rows[0]
    assert row.result.status.name == "Unconverged" and row.result.simple_iters == n_iter
    for name in ("Ux", "k", "omega", "nuT", "F1", "Pk"):
        i = ck.FIELD_NAMES.index(name)
        scale = max(np.max(np.abs(want.fields[i])), 1e-300)
        err = np.max(np.abs(fields[0, i] - want.fields[i])) / scale
        assert err < RTOL_TRAJ, (name, err)
    # Uy and p are round-off noise (~1e-13, ~1e-12) in a fully developed channel:
    # compare them on the velocity scale and on an absolute pressure scale
    uscale = np.max(np.abs(want.field("Ux")))
    assert np.max(np.abs(fields[0, 1] - want.field("Uy"))) / uscale < RTOL_TRAJ
    assert np.max(np.abs(fields[0, 3] - want.field("p"))) < 1e-9
    # residual history: initial residual of the x-momentum solve, the scaled momentum
    # residual and the relative change of U judged by the convergence test; the
    # continuity residuals are round-off in an x-invariant channel (compared absolutely)
    h, g = hist[0], want.history
    for col in (1, 7, 9):
        assert rel(h[:, col], g[:, col]) < 1e-8, col
    assert np.max(np.abs(h[:, 4] - g[:, 4])) < 1e-10


@pytest.mark.parametrize("fixture,solver", [("small_channel_ref", "AMG"),
                                            ("small_channel_pcg_ref", "PCG")])
def test_converged_small_channel_matches_reference(rq, fixture, solver):
    g = np.load(GOLDEN + fixture + ".npz")
    case = cases.small_channel()
    batch = cases.product_batch(rq, case, pressure_solver=solver)
    res, fields, _ = batch.evaluate_fields([[case.coeffs[9], case.coeffs[8]]])
    row = res.rows[0]
    assert row.result.status.name == str(g["status"])
    assert rel(row.result.predictions, g["predictions"]) < RTOL_CONV
    assert rel(fields[0, 0], g["Ux"]) < RTOL_CONV
    assert rel(fields[0, 4], g["k"]) < 1e-8
    assert abs(row.result.simple_iters - int(g["iterations"])) <= 0.02 * int(g["iterations"])


def test_config1_matches_reference(rq):
    """Plain small case: 3x128 channel, tol 1e-10 -- profiles within 1e-10 of the reference."""
    g = np.load(GOLDEN + "config1_ref.npz")
    case = ck.config1_case()
    batch = cases.product_batch(rq, case)
    res, fields, _ = batch.evaluate_fields([[0.31, 0.09]])
    row = res.rows[0]
    assert row.result.status.name == "Converged" == str(g["status"])
    assert rel(row.result.predictions, g["predictions"]) < RTOL_CONV
    assert rel(fields[0, 0], g["Ux"]) < RTOL_CONV


def test_batch_rows_independent_of_composition(rq):
    case = cases.small_channel()
    batch = cases.product_batch(rq, case)
    thetas = np.array([[0.31, 0.09], [0.29, 0.085], [0.33, 0.095], [0.9, 0.09], [0.31, 0.09]])
    full = batch.evaluate(thetas)
    alone = batch.evaluate(thetas[1:2])
    rev = batch.evaluate(thetas[::-1])
    assert full.rows[3].result.status.name == "InvalidParameters"
    assert np.all(np.isnan(full.rows[3].result.predictions))
    assert full.rows[3].result.log_lik == -1e30
    np.testing.assert_array_equal(full.rows[1].result.predictions, alone.rows[0].result.predictions)
    np.testing.assert_array_equal(full.rows[0].result.predictions, full.rows[4].result.predictions)
    np.testing.assert_array_equal(full.rows[2].result.predictions, rev.rows[2].result.predictions)
    assert full.rows[1].result.simple_iters == alone.rows[0].result.simple_iters


def test_multi_class_launch_equals_separate(rq):
    a = cases.product_batch(rq, cases.small_channel())
    b = cases.product_batch(rq, cases.small_channel(ny=32, re_tau=250.0, nu=1 / 250.0))
    theta = np.array([[0.31, 0.09], [0.30, 0.088], [0.31, 0.09]])
    multi = rq.evaluate_multi([a, b], [0, 1, 1], theta)
    sa = a.evaluate(theta[:1])
    sb = b.evaluate(theta[1:])
    np.testing.assert_array_equal(multi.rows[0].result.predictions, sa.rows[0].result.predictions)
    np.testing.assert_array_equal(multi.rows[1].result.predictions, sb.rows[0].result.predictions)
    np.testing.assert_array_equal(multi.rows[2].result.predictions, sb.rows[1].result.predictions)


@pytest.mark.parametrize("solver", ["AMG", "PCG"])
def test_mixed_precision_small_channel_within_1e6(rq, solver):
    """Mixed form (FP32 inner Krylov/AMG, FP64 refinement): converged profiles within
    1e-6 relative of the reference's FP64 solve, same verdict."""
    g = np.load(GOLDEN + "small_channel_ref.npz")
    case = cases.small_channel()
    batch = cases.product_batch(rq, case, pressure_solver=solver, precision="mixed")
    res, fields, _ = batch.evaluate_fields([[case.coeffs[9], case.coeffs[8]]])
    row = res.rows[0]
    assert row.result.status.name == str(g["status"])
    assert rel(row.result.predictions, g["predictions"]) < 1e-6
    assert rel(fields[0, 0], g["Ux"]) < 1e-6


def test_config1_mixed_within_1e6(rq):
    g = np.load(GOLDEN + "config1_ref.npz")
    batch = cases.product_batch(rq, ck.config1_case(), precision="mixed")
    res, fields, _ = batch.evaluate_fields([[0.31, 0.09]])
    row = res.rows[0]
    assert row.result.status.name == "Converged"
    assert rel(row.result.predictions, g["predictions"]) < 1e-6
    assert rel(fields[0, 0], g["Ux"]) < 1e-6


def test_768_thread_cta_matches_reference(rq):
    """768-thread CTAs (the default above 1024 cells) on the small channel: the same
    converged profile as the reference to 1e-10 (the CTA size changes only the order
    of the block reductions)."""
    g = np.load(GOLDEN + "small_channel_ref.npz")
    case = cases.small_channel()
    batch = cases.product_batch(rq, case, block_threads=768)
    res, fields, _ = batch.evaluate_fields([[case.coeffs[9], case.coeffs[8]]])
    row = res.rows[0]
    assert row.result.status.name == str(g["status"])
    assert rel(row.result.predictions, g["predictions"]) < RTOL_CONV
    assert rel(fields[0, 0], g["Ux"]) < RTOL_CONV


def ensemble_case(re_tau, ny, max_iter):
    """The benchmark's class (workloads.channel_batch) as a checker case."""
    import rans_uq_b200.workloads as wl

    x, y = wl.channel_probes(re_tau)
    return ck.Case(ny=ny, re_tau=re_tau, nu=1 / re_tau, yplus=0.5, alpha_u=wl.ALPHA_U,
                   tol=wl.TOL, max_iter=max_iter, obs_x=x, obs_y=y, obs_value=np.zeros(30),
                   obs_sigma=np.ones(30)).with_theta(0.31, 0.09)


@pytest.mark.parametrize("n_iter", [40, 600])
def test_1536_cell_class_fields_after_n_iterations(rq, checker, n_iter):
    """The benchmark's largest class (Re_tau 1000, 3 x 512 cells, 768-thread CTAs) against
    the restatement after 40 and 600 outer iterations (past the turbulence start at 500)."""
    import rans_uq_b200.workloads as wl

    want = checker.solve(ensemble_case(1000.0, 512, n_iter), "oracle")
    batch = wl.channel_batch(1000.0, 512, max_iter=n_iter)
    assert batch._problem.n_cells == 1536
    res, fields, _ = batch.evaluate_fields([[0.31, 0.09]])
    assert res.rows[0].result.simple_iters == n_iter
    for name in ("Ux", "k", "omega", "nuT"):
        i = ck.FIELD_NAMES.index(name)
        assert rel(fields[0, i], want.fields[i]) < RTOL_TRAJ, name


def test_1536_cell_class_repeats_bit_for_bit(rq):
    """Every sweep of the 768-thread CTA reads only what a barrier has published: two
    launches of the same draws (past the turbulence start) give the same bits, fields
    and predictions, whichever CTA took which draw."""
    import rans_uq_b200.workloads as wl

    batch = wl.channel_batch(1000.0, 512, max_iter=700)
    theta = [[0.31, 0.09], [0.30, 0.088]]
    r1, f1, _ = batch.evaluate_fields(theta)
    r2, f2, _ = batch.evaluate_fields(theta[::-1])
    np.testing.assert_array_equal(f1[0], f2[1])
    np.testing.assert_array_equal(f1[1], f2[0])
    for a, b in ((0, 1), (1, 0)):
        np.testing.assert_array_equal(r1.rows[a].result.predictions, r2.rows[b].result.predictions)
        assert r1.rows[a].result.simple_iters == r2.rows[b].result.simple_iters == 700


def test_ensemble_classes_match_reference(rq):
    """The benchmark's three classes at (0.31, 0.09), one multi-class launch: each
    converges to the reference's own converged profile (the ensemble's synthetic
    truth, written by tests/golden/make_channel_truth.py from oracle/_ref) to 1e-10, in an
    iteration count within 2 % of the reference's (12460, 58690, 258900)."""
    import json

    import rans_uq_b200.workloads as wl

    from pathlib import Path

    truth = json.loads((Path(wl.__file__).parent / "data" / "channel_truth.json").read_text())
    batches = [wl.channel_batch(re, ny) for re, ny in wl.CLASSES]
    res = rq.evaluate_multi(batches, [0, 1, 2], np.array([[0.31, 0.09]] * 3))
    for c, row in enumerate(res.rows):
        want = truth[str(c)]
        assert row.result.status.name == want["status"] == "Converged"
        assert rel(row.result.predictions, want["profile"]) < RTOL_CONV, c
        assert abs(row.result.simple_iters - want["iterations"]) <= 0.02 * want["iterations"], c


def test_rq_solve_equals_batch_row(rq):
    """rq_solve (all eleven coefficients, SIMPLESolver::initUniform + solve) gives the
    same row, predictions, fields and residual history as the batch row of the same
    coefficients: the same per-solve code on a class view whose every coefficient is
    active."""
    import ctypes as C

    import rans_uq_b200._native as N

    case = cases.small_channel(max_iter=300)
    batch = cases.product_batch(rq, case)
    res, fields, hist = batch.evaluate_fields([[case.coeffs[9], case.coeffs[8]]], hist_cap=300)
    coeffs = np.array(case.coeffs, dtype=float)
    n = batch._problem.n_cells
    row = N.RowOut()
    pred = np.zeros(len(case.obs_x))
    f = np.zeros((11, n))
    h = np.zeros((300, 11))
    N.call("rq_solve", batch._problem.handle, N.dptr(coeffs), C.byref(row), N.dptr(pred),
           N.dptr(f), N.dptr(h), C.c_int32(300))
    want = res.rows[0].result
    assert row.status == int(want.status) and row.iterations == want.simple_iters == 300
    np.testing.assert_array_equal(pred, want.predictions)
    np.testing.assert_array_equal(f, fields[0])
    np.testing.assert_array_equal(h, hist[0])


def test_batch_edge_cases(rq):
    """ForwardBatch::evaluate's edge cases (ForwardBatch.hpp:52-124, bindings.cpp:893-905):
    an empty batch returns no rows; a theta of the wrong shape or a worker count below
    one is rejected; non-finite parameters are InvalidParameters rows with the -1e30
    sentinel and NaN predictions, as out-of-bound ones are."""
    batch = cases.product_batch(rq, cases.small_channel(max_iter=5))
    empty = batch.evaluate(np.zeros((0, 2)))
    assert empty.rows == [] and empty.predictions.shape == (0, 8)
    with pytest.raises(ValueError, match="shape"):
        batch.evaluate(np.zeros((2, 3)))
    with pytest.raises(ValueError, match="workers"):
        batch.evaluate(np.array([[0.31, 0.09]]), workers=0)
    res = batch.evaluate(np.array([[np.nan, 0.09], [0.31, np.inf], [0.31, 0.09]]))
    for r in res.rows[:2]:
        assert r.result.status.name == "InvalidParameters" and r.result.log_lik == -1e30
        assert np.all(np.isnan(r.result.predictions))
    assert res.rows[2].result.status.name == "Unconverged"
