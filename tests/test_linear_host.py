"""Standalone linear solves, host side (no GPU): the C ABI's admission of LDU
systems follows the reference's LinearSystem::validate / validateSolve rules and
factory names (core/include/LinearSolver.hpp:63-92, 988-998), and the oracle's
restatement of the device AMG variant converges to the reference AMG's solution
on the Poisson systems of the linear-solve workload."""
import numpy as np
import pytest

import rans_uq_b200.linear as lin
import rans_uq_b200.workloads as wl
from oracle import checker as ck


def small():
    return wl.poisson_system(8, 3)


def test_invalid_connectivity_rejected():
    s = small()
    s.nbr = s.nbr.copy()
    s.nbr[4] = s.n_cells  # out of range
    with pytest.raises(ValueError, match="connectivity"):
        lin.make_solver("PCG").solve(s, np.zeros(s.n_cells), 100, 1e-8)


def test_nonfinite_coefficients_rejected():
    s = small()
    s.upper = s.upper.copy()
    s.upper[0] = np.nan
    with pytest.raises(ValueError, match="finite"):
        lin.solve_batch([s], kind="AMG")


def test_unknown_and_gauss_seidel_kinds():
    with pytest.raises(ValueError):
        lin.make_solver("Jacobi")
    s = small()
    with pytest.raises(NotImplementedError):
        lin.make_solver("GaussSeidel").solve(s, np.zeros(s.n_cells), 10, 1e-8)


def test_poisson_system_is_symmetric_and_dominant():
    s = wl.poisson_system(16, 9)
    np.testing.assert_array_equal(s.upper, s.lower)
    off = np.zeros(s.n_cells)
    np.add.at(off, s.own, np.abs(s.upper))
    np.add.at(off, s.nbr, np.abs(s.lower))
    assert np.all(s.diag >= off - 1e-12)
    assert np.sum(s.diag > off + 1e-12) == 16  # the Dirichlet column only
    assert s.n_if == 2 * 16 * 15


@pytest.mark.skipif(not ck.have("ref"), reason="oracle/_ref not built")
@pytest.mark.parametrize("n", [32, 64])
def test_oracle_device_amg_matches_reference_amg(n):
    s = wl.poisson_system(n, 5)
    args = (s.diag, s.upper, s.lower, s.source, s.own, s.nbr, np.zeros(n * n), 500, 1e-10)
    xr, ir = ck.linear_solve(0, *args, lib_kind="ref")
    xo, io = ck.linear_solve(10, *args, lib_kind="oracle")
    assert ir["converged"] and io["converged"]
    assert ck.rel_err(xo, xr) < 1e-9
