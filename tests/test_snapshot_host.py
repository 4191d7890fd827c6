"""The boundary-value rules the snapshot export relies on, checked on the reference's
own snapshots (fixtures written by tests/golden/make_golden.py from
evaluateWithDiagnostics(theta, snapshot=True)): on the all-wall periodic channel, U, k,
nuT, Pk and CDkw are 0 at the walls, F1 and F2 are 1, p takes the owner cell's value and
omega_b = 60 nu / (beta1 y1^2) (BoundaryCondition.hpp:279-384). The device returns cell
values and face fluxes; the host fills the boundary values by exactly these rules."""
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import checker as ck

GOLDEN = Path(__file__).parent / "golden"


@pytest.mark.parametrize("fixture,max_iter", [("snapshot_small_channel_ref", 60000),
                                              ("snapshot_small_channel_capped_ref", 300)])
def test_reference_snapshot_boundary_rules(checker, fixture, max_iter):
    g = np.load(GOLDEN / f"{fixture}.npz")
    case = cases.small_channel(max_iter=max_iter)
    _, faces, ni = ck.mesh(case, "oracle")
    nx = case.nx
    own = faces[ni:, 0].astype(int)
    # wall faces in face order: the bottom row's, then the top row's
    assert own.tolist() == list(range(nx)) + [(case.ny - 1) * nx + i for i in range(nx)]
    bnd, cells = g["boundary"], g["cells"]
    assert bnd.shape == (11, 2 * nx) and g["face_fluxes"].shape == (len(faces),)
    for i in (0, 1, 2, 4, 6, 9, 10):
        np.testing.assert_array_equal(bnd[i], 0.0)
    np.testing.assert_array_equal(bnd[7], 1.0)
    np.testing.assert_array_equal(bnd[8], 1.0)
    np.testing.assert_array_equal(bnd[3], cells[3][own])
    y1 = np.maximum(faces[ni:, 7], 1e-20)
    np.testing.assert_array_equal(bnd[5], 60.0 * case.nu / (case.coeffs[2] * y1 * y1))
    # no mass crosses a wall
    np.testing.assert_array_equal(np.abs(g["face_fluxes"][ni:]), 0.0)
