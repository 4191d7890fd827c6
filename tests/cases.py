"""Shared case construction for the parity tests: one description drives the
B200 product (through its reference-style API) and the CPU checkers."""
from __future__ import annotations

import dataclasses

import numpy as np

from oracle import checker as ck


def product_mesh(rq, case: ck.Case):
    """The product's Mesh for the checker case's generator call."""
    if case.curved:
        return rq.Mesh.make_curved_channel_periodic_2d(case.x_nodes, case.y_bottom, case.y_top,
                                                      case.ny, case.re_mesh, case.yplus)
    return rq.Mesh.make_periodic_channel_2d(case.nx, case.ny, case.lx, case.h, case.re_tau,
                                            case.yplus)


def product_batch(rq, case: ck.Case, pressure_solver: str = "AMG", precision: str = "fp64",
                  block_threads: int = 0, model_class=None):
    """A ForwardBatch (or model_class, e.g. rq.ForwardModel) on the GPU path with the same
    inputs as the checker case."""
    mesh = product_mesh(rq, case)
    mesh.compute_wall_distance()
    obs = rq.ObservationOperator()
    for x, y, v, s in zip(case.obs_x, case.obs_y, case.obs_value, case.obs_sigma):
        obs.add_velocity_profile(rq.Vec3(float(x), float(y), 0.0), case.obs_component, float(v),
                                 float(s))
    st = rq.SolverSettings(
        max_iterations=case.max_iter, convergence_tol=case.tol, alpha_u=case.alpha_u,
        alpha_p=case.alpha_p, alpha_k=case.alpha_k, alpha_omega=case.alpha_w,
        inner_iterations=case.inner_iter, inner_tolerance=case.inner_tol,
        turb_start_iter=case.turb_start, nut_floor_iters=case.nut_floor_iters,
        convergence_window=case.conv_window, monitor_interval=case.monitor_interval,
        body_force=rq.Vec3(*case.body_force), divergence_limit=case.div_limit,
        k_min=case.k_min, k_max=case.k_max, omega_min=case.omega_min, verbose=False,
        pressure_solver=pressure_solver, precision=precision, block_threads=block_threads)
    params = rq.InferenceParameterSet("a1_betaStar", (9, 8), base=tuple(case.coeffs))
    bcs = rq.FlowBoundaryConditions.channel_defaults(mesh, *case.bc)
    return (model_class or rq.ForwardBatch)(mesh, params, obs, bcs, case.nu, st,
                                            rq.Vec3(*case.init_u), case.init_p, case.init_k,
                                            case.init_w)


def small_channel(**kw) -> ck.Case:
    """Re_tau 182.088 channel on 3x24 cells with 8 probes: converges in seconds."""
    x, y = ck.channel_probes(182.088, n=8, lo=2.0, hi=150.0)
    base = ck.Case(ny=24, yplus=1.0, tol=1e-8, max_iter=60000, obs_x=x, obs_y=y,
                   obs_value=np.zeros(8), obs_sigma=np.full(8, 1e-3))
    return dataclasses.replace(base, **kw)


# Warm-start sequences on small_channel() (one ForwardModel, calls in order), with what
# the reference does on each call:
#   (0.2, 0.05)    cold, Converged, stored
#   (0.72, 0.12)   0.525 from the entry (>= 0.5): cold, Converged, stored
#   (0.2, 0.05)    warm from its own state: Converged at the turbulence start, replaces it
#   (0.21, 0.052)  warm from (0.2, 0.05): the iteration-0 residual norms are round-off
#                  of a converged state, so the normalised residual blows past the
#                  divergence limit: Diverged, not stored
#   (0.95, 0.09)   a1 above its bound: InvalidParameters, no lookup
#   (0.72, 0.12)   warm from itself again
WARM_SEQUENCE = [(0.2, 0.05), (0.72, 0.12), (0.2, 0.05), (0.21, 0.052), (0.95, 0.09),
                 (0.72, 0.12)]
# A budget of one entry (6880 payload bytes on the 3 x 24 mesh): the second store evicts
# the first, so the third call starts cold.
WARM_BUDGET_SEQUENCE = [(0.2, 0.05), (0.72, 0.12), (0.2, 0.05)]
WARM_BUDGET_BYTES = 6900


def bump_case(nx=24, ny=16, **kw) -> ck.Case:
    """Config-3 geometry (bump of height h=1, L=9h, W=4h, top 3.04h) on a coarse mesh."""
    xn = np.linspace(0.0, 9.0, nx + 1)
    yb = np.where(np.abs(xn - 4.5) < 2.0, 0.5 * (1 + np.cos(2 * np.pi * (xn - 4.5) / 4.0)), 0.0)
    yb[0] = yb[-1] = 0.0
    x = np.full(6, 2.0)
    y = np.linspace(0.2, 2.8, 6)
    base = ck.Case(nx=nx, ny=ny, curved=True, x_nodes=xn, y_bottom=yb, y_top=3.04,
                   re_mesh=5600.0, yplus=1.0, nu=1.0 / 5600.0, bc=(1.0, 1e-4, 10.0),
                   init_u=(0.3, 0.0, 0.0), init_k=1e-4, init_w=10.0, alpha_u=0.4,
                   alpha_p=0.25, body_force=(4e-3, 0.0, 0.0), tol=1e-6, max_iter=200,
                   obs_x=x, obs_y=y, obs_value=np.zeros(6), obs_sigma=np.full(6, 1e-2))
    return dataclasses.replace(base, **kw)


# Generator calls whose binary mesh files (Mesh::saveBinary) are pinned by digest.
MESH_BINARY_CASES = {
    "channel_3x24": ck.Case(ny=24, yplus=1.0),
    "channel_3x128_config1": ck.config1_case(),
    "channel_3x512_re1000": ck.Case(ny=512, re_tau=1000.0, yplus=0.5),
    "bump_24x16": bump_case(24, 16),
    "bump_200x100": bump_case(200, 100),
}
