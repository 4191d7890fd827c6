"""The C ABI library loads on a CPU-only machine, exports every symbol of
include/rq_b200.h, and its host-side set-up (mesh, AMG hierarchy, admission)
agrees with the reference and the oracle. No kernel is launched here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle import checker as ck

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "rq_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s+(rq_\w+)\(", text, re.M)))


def test_library_exports_every_header_symbol(rq):
    lib = rq.lib()
    syms = header_symbols()
    assert "rq_evaluate_batch" in syms and "rq_linear_solve" in syms
    for s in syms:
        assert hasattr(lib, s), s


def test_python_binding_covers_header():
    import rans_uq_b200._native as N
    assert set(header_symbols()) <= set(N.SIGNATURES)


@pytest.mark.parametrize("mk", [lambda: ck.config1_case(), lambda: cases.bump_case(40, 20),
                                lambda: ck.Case(ny=512, re_tau=1000.0, yplus=0.5)])
def test_product_mesh_bitwise_equal_to_oracle(rq, checker, mk):
    case = mk()
    if case.curved:
        m = rq.Mesh.make_curved_channel_periodic_2d(case.x_nodes, case.y_bottom, case.y_top,
                                                   case.ny, case.re_mesh, case.yplus)
    else:
        m = rq.Mesh.make_periodic_channel_2d(case.nx, case.ny, case.lx, case.h, case.re_tau,
                                             case.yplus)
    cells, faces, ni = checker.mesh(case, "oracle")
    np.testing.assert_array_equal(m.cell_geometry(), cells)


def test_default_settings_match_reference(rq):
    import rans_uq_b200._native as N
    s = N.Settings()
    N.call("rq_default_settings", C.byref(s))
    d = rq.SolverSettings()
    assert s.max_iterations == d.max_iterations == 500
    assert s.alpha_u == d.alpha_u == 0.7 and s.alpha_p == 0.3
    assert s.inner_iterations == 200 and s.inner_tolerance == 1e-3
    assert s.convergence_window == 25 and s.monitor_interval == 10
    assert s.k_min == 1e-10 and s.omega_min == 1e-6


def test_parameter_set_mirrors_reference(rq):
    p = rq.InferenceParameterSet.a1_betaStar()
    assert p.active_names() == ["a1", "betaStar"]
    assert p.in_bounds([0.31, 0.09]) and not p.in_bounds([0.9, 0.09])
    assert not p.in_bounds([float("nan"), 0.09]) and not p.in_bounds([0.31])
    assert p.unpack([0.3, 0.08])[9] == 0.3 and p.unpack([0.3, 0.08])[8] == 0.08
    with pytest.raises(ValueError):
        rq.InferenceParameterSet.from_indices("bad", [1, 1])


def test_unsupported_settings_fail_loudly(rq):
    with pytest.raises(NotImplementedError):
        rq.SolverSettings(use_wall_functions=True).native()
    with pytest.raises(NotImplementedError):
        rq.SolverSettings(legacy_convergence=True).native()
    with pytest.raises(ValueError):
        rq.SolverSettings(pressure_solver="GMRES").native()


def test_observation_validation(rq):
    obs = rq.ObservationOperator()
    with pytest.raises(ValueError):
        obs.add_velocity_profile(rq.Vec3(0.5, float("nan"), 0), 0, 1.0, 0.1)
    with pytest.raises(ValueError):
        obs.add_velocity_profile(rq.Vec3(0.5, 0.1, 0), 0, 1.0, 0.0)
    obs.add_velocity_profile(rq.Vec3(0.5, 0.1, 0), 0, 1.0, 0.5)
    assert obs.log_likelihood_from_predictions([2.0]) == pytest.approx(-0.5 * 1.0 / 0.25)
