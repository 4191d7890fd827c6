"""The oracle (oracle/rq_oracle.cpp) pinned against the reference itself: the
compiled reference sources (oracle/_ref) where present, and the reference's own
golden case and known-answer values (tests/golden/reference_goldens.json)."""
import json
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import checker as ck

GOLDEN = Path(__file__).parent / "golden"
GOLD = json.loads((GOLDEN / "reference_goldens.json").read_text())
need_ref = pytest.mark.skipif(not ck.have("ref"), reason="oracle/_ref not built here")


def test_oracle_built(checker):
    assert checker.have("oracle")


@need_ref
@pytest.mark.parametrize("mk", [ck.config1_case, lambda: cases.bump_case(40, 20)])
def test_mesh_bitwise_equal_to_reference(checker, mk):
    case = mk()
    c1, f1, n1 = checker.mesh(case, "ref")
    c2, f2, n2 = checker.mesh(case, "oracle")
    assert n1 == n2
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(f1, f2)


@need_ref
@pytest.mark.parametrize("ps", [ck.P_PCG, ck.P_BICGSTAB])
def test_trajectory_bitwise_equal_to_reference(checker, ps):
    """With the reference's own linear solvers the restatement reproduces the compiled
    reference exactly: every field after 300 outer iterations, and the history."""
    case = cases.small_channel(max_iter=300, pressure_solver=ps)
    a = checker.solve(case, "ref", hist_cap=300)
    b = checker.solve(case, "oracle", hist_cap=300)
    np.testing.assert_array_equal(a.fields, b.fields)
    np.testing.assert_array_equal(a.predictions, b.predictions)
    fin = np.isfinite(a.history)
    np.testing.assert_array_equal(a.history[fin], b.history[fin])


@need_ref
@pytest.mark.parametrize("ps", [ck.P_PCG, ck.P_BICGSTAB])
def test_bump_trajectory_bitwise_equal_to_reference(checker, ps):
    case = cases.bump_case(24, 16, max_iter=40, pressure_solver=ps)
    a = checker.solve(case, "ref")
    b = checker.solve(case, "oracle")
    np.testing.assert_array_equal(a.fields, b.fields)


def test_oracle_reproduces_reference_golden_case(checker):
    """periodic_channel_re180 golden (tests/golden/constrained_omega/periodic_channel_re180.json,
    recorded by the reference with Apple clang): the restatement with the device-style AMG
    reaches the same verdict, iteration count and U+ probes (the golden reproduces on Linux
    only to ~6e-11 with the reference's own AMG)."""
    m, s = GOLD["mesh"], GOLD["settings"]
    x = np.full(20, 0.5)
    y = np.array(GOLD["probe_y_over_delta"])
    case = ck.Case(nx=m["nx"], ny=m["ny"], re_tau=m["Re_tau"], yplus=m["yplus_target"],
                   nu=GOLD["nu"], max_iter=s["max_iterations"], tol=s["convergence_tol"],
                   alpha_u=s["alpha_u"], alpha_p=s["alpha_p"], obs_x=np.r_[x],
                   obs_y=y, obs_value=np.zeros(20), obs_sigma=np.full(20, 0.1))
    o = checker.solve(case, "oracle")
    assert o.status == "Converged"
    assert abs(o.iterations - GOLD["result"]["final_iter"]) <= 20
    np.testing.assert_allclose(o.predictions, GOLD["u_plus_probes"], rtol=1e-6)
    ns = GOLD["field_norms"]
    np.testing.assert_allclose(np.sum(o.field("Ux") ** 2), ns["sumsq_ux"], rtol=1e-6)
    np.testing.assert_allclose(np.sum(o.field("k") ** 2), ns["sumsq_k"], rtol=1e-6)


def test_oracle_known_answer_grid_convergence_coarse(checker):
    """test_sst_channel_grid_convergence.cpp (level 0, 2x16 cells): the solve converges,
    the wall force balances the body force and the RMS error against the reference's
    independent half-channel U+ values is the one the reference measures (~0.150)."""
    st = GOLD["grid_convergence_stations"]
    ref = np.array(GOLD["grid_convergence_uplus"])
    half = 16
    first = 1 + np.tanh(2 * (1.0 / half - 1)) / np.tanh(2.0)
    case = ck.Case(ny=2 * half, yplus=first * 182.088, tol=1e-8, max_iter=150000, alpha_u=0.5,
                   obs_x=np.full(7, 0.5), obs_y=np.array(st), obs_value=np.zeros(7),
                   obs_sigma=np.ones(7))
    o = checker.solve(case, "oracle")
    assert o.status == "Converged"
    rms = float(np.sqrt(np.mean((o.predictions - ref) ** 2)))
    assert 0.10 < rms < 0.20


def test_device_amg_matches_reference_amg_solution(checker):
    """A pressure-correction system (from 50 iterations of the small channel): the
    device-style AMG-PCG of the GPU path and the reference's Gauss-Seidel AMG-PCG
    reach the same solution at tight tolerance."""
    if not ck.have("ref"):
        pytest.skip("oracle/_ref not built here")
    rng = np.random.default_rng(3)
    nx, ny = 3, 40
    n = nx * ny
    own, nbr, up = [], [], []
    for j in range(ny):
        for i in range(nx):
            c = j * nx + i
            own.append(c); nbr.append(j * nx + (i + 1) % nx); up.append(-0.05 * rng.uniform(0.5, 2))
    for j in range(ny - 1):
        for i in range(nx):
            own.append(j * nx + i); nbr.append((j + 1) * nx + i); up.append(-3.0 * rng.uniform(0.5, 2))
    up = np.array(up)
    d = np.zeros(n)
    for o_, b_, u_ in zip(own, nbr, up):
        d[o_] -= u_; d[b_] -= u_
    d[0] *= 2
    b = rng.standard_normal(n)
    xa, ra = checker.linear_solve(0, d, up, up, b, own, nbr, np.zeros(n), 500, 1e-12, "ref")
    xo, ro = checker.linear_solve(10, d, up, up, b, own, nbr, np.zeros(n), 500, 1e-12, "oracle")
    assert ra["converged"] and ro["converged"]
    assert np.max(np.abs(xa - xo)) / np.max(np.abs(xa)) < 1e-9
    xp, rp = checker.linear_solve(1, d, up, up, b, own, nbr, np.zeros(n), 2000, 1e-12, "ref")
    xq, rq_ = checker.linear_solve(1, d, up, up, b, own, nbr, np.zeros(n), 2000, 1e-12, "oracle")
    np.testing.assert_array_equal(xp, xq)


def _same_sequence(a, b, rtol=1e-12):
    """Verdicts, iteration counts, warm/cold and retained bytes exactly; predictions and
    log-likelihoods to 1e-12 (the fields are bitwise equal; the probe interpolation of the
    restatement rounds differently, ~1e-14)."""
    assert a.status == b.status
    assert np.array_equal(a.iterations, b.iterations)
    assert np.array_equal(a.used_warm, b.used_warm)
    assert np.array_equal(a.retained, b.retained)
    ok = np.array([s in ("Converged", "Unconverged") for s in a.status])
    np.testing.assert_allclose(a.loglik, b.loglik, rtol=rtol, atol=0)
    np.testing.assert_allclose(a.predictions[ok], b.predictions[ok], rtol=rtol, atol=0)


def test_warm_sequence_oracle_matches_reference_fixture(checker):
    """The warm-start cache of the sequential model: which calls start warm, the
    verdicts (a warm start next to a converged state is Diverged after 5 iterations
    in the reference too), eviction by the byte budget, and bitwise results."""
    for name, seq, budget in (("warm_sequence_ref", cases.WARM_SEQUENCE, 64 << 20),
                              ("warm_budget_ref", cases.WARM_BUDGET_SEQUENCE,
                               cases.WARM_BUDGET_BYTES)):
        g = np.load(GOLDEN / f"{name}.npz")
        assert np.array_equal(g["thetas"], np.asarray(seq, float))
        want = ck.SequenceOut(list(g["status"]), g["iterations"], g["loglik"], g["predictions"],
                              g["used_warm"], g["retained"])
        got = ck.solve_sequence(cases.small_channel(), seq, "oracle", byte_budget=budget)
        _same_sequence(got, want)


@need_ref
def test_warm_sequence_unconverged_not_stored():
    case = cases.small_channel(max_iter=200)
    th = [(0.31, 0.09), (0.31, 0.09)]
    a = ck.solve_sequence(case, th, "oracle")
    b = ck.solve_sequence(case, th, "ref")
    _same_sequence(a, b)
    assert not a.used_warm.any() and a.retained.tolist() == [0, 0]


@need_ref
def test_full_size_bump_trajectory_bitwise_equal_to_reference(checker):
    """The benchmark's bump-wall mesh (200 x 100 cells): the restatement's fields after 3
    outer iterations with the PCG pressure solver equal the reference's bit for bit."""
    case = cases.bump_case(200, 100, max_iter=3, pressure_solver=ck.P_PCG)
    a = checker.solve(case, "ref")
    b = checker.solve(case, "oracle")
    np.testing.assert_array_equal(a.fields, b.fields)
