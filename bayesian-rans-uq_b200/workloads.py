"""Synthetic stand-ins for the reference's calibration workloads (its Lee-Moser
DNS data are not shipped): the seeded channel ensemble of the calibration's
prior design, with a synthetic observed profile per Reynolds-number class.

Draws restate cfdr.statistics.sample_rng / independent_uniform_design
(rans-uq/python/cfdr/statistics.py:42-57, 69-91): SHA-256 of the identity
string "cfdr-statistics-v1:{seed}:{id}:{purpose}" seeds a PCG64 stream, and
each draw is rng.uniform(lower, upper), so the GPU and the reference see
bit-identical coefficients.
"""
from __future__ import annotations

import hashlib
import json
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import core

SEED = 20261010
BOX_LO = (0.28, 0.084)  # (a1, beta*) -- calibration_coverage.py STAGE1_BOX
BOX_HI = (0.34, 0.096)
CLASSES = ((182.088, 128), (550.0, 256), (1000.0, 512))
ALPHA_U = 0.8           # fixed once by the CPU pilot; the converged state does not depend on it
MAX_ITER = 300000
TOL = 1e-8
NOISE = 0.0014          # relative synthetic observation noise


def sample_rng(root_seed: int, sample_id: int, purpose: str) -> np.random.Generator:
    identity = f"cfdr-statistics-v1:{root_seed}:{sample_id}:{purpose}"
    digest = hashlib.sha256(identity.encode("utf-8")).digest()
    words = [int.from_bytes(digest[i:i + 4], "little") for i in range(0, 32, 4)]
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence(words)))


def uniform_design(ids, lower=BOX_LO, upper=BOX_HI, root_seed=SEED) -> np.ndarray:
    lo, hi = np.asarray(lower, float), np.asarray(upper, float)
    return np.array([sample_rng(root_seed, i, "prior-design").uniform(lo, hi) for i in ids])


def channel_probes(re_tau: float, n: int = 30):
    """30 stations log-spaced in y+ over [1, 175] at x = 0.5 (u_tau = 1, h = 1)."""
    yp = np.geomspace(1.0, 175.0, n)
    return np.full(n, 0.5), yp / re_tau


def channel_batch(re_tau: float, ny: int, observed=None, sigma=None, precision="fp64",
                  alpha_u=ALPHA_U, max_iter=MAX_ITER, tol=TOL, pressure_solver="AMG",
                  block_threads=0) -> core.ForwardBatch:
    """One Re_tau class of the channel ensemble as a ForwardBatch (the calibration's
    forward_batch, docs/figures/calibration_coverage.py:81-113, on 3 x ny cells, y+ 0.5)."""
    mesh = core.Mesh.make_periodic_channel_2d(3, ny, 1.0, 1.0, re_tau, 0.5)
    mesh.compute_wall_distance()
    x, y = channel_probes(re_tau)
    obs = core.ObservationOperator()
    observed = np.zeros(len(x)) if observed is None else observed
    sigma = np.ones(len(x)) if sigma is None else sigma
    for xi, yi, ui, si in zip(x, y, observed, sigma):
        obs.add_velocity_profile(core.Vec3(float(xi), float(yi), 0.0), 0, float(ui), float(si))
    st = core.SolverSettings(max_iterations=max_iter, convergence_tol=tol, alpha_u=alpha_u,
                             body_force=core.Vec3(1.0, 0.0, 0.0), verbose=False,
                             precision=precision, pressure_solver=pressure_solver,
                             block_threads=block_threads)
    bcs = core.FlowBoundaryConditions.channel_defaults(mesh, 1.0, 1.0, 10.0)
    return core.ForwardBatch(mesh, core.InferenceParameterSet.a1_betaStar(), obs, bcs,
                             1.0 / re_tau, st, core.Vec3(15.0, 0.0, 0.0), 0.0, 1.0, 10.0)


@dataclass
class Ensemble:
    batches: list            # one ForwardBatch per Re_tau class
    theta: np.ndarray        # (n, 2) draws
    cls: np.ndarray          # (n,) class of each draw
    truth: list              # per class: noise-free synthetic profile


def stored_truth(c: int):
    """Noise-free probe profile of class c from data/channel_truth.json (the
    reference solver's own converged solve at (0.31, 0.09)), or None."""
    path = Path(__file__).parent / "data" / "channel_truth.json"
    if not path.exists():
        return None
    rec = json.loads(path.read_text()).get(str(c))
    if rec is None or rec["ny"] != CLASSES[c][1] or rec["status"] != "Converged":
        return None
    return np.asarray(rec["profile"], dtype=np.float64)


def class_observation(c: int, truth=None):
    """(observed, sigma) of class c: truth x (1 + 0.0014 eps), eps seeded per class,
    sigma = 0.0014 |truth|. Host arithmetic only (no solve)."""
    u = stored_truth(c) if truth is None else np.asarray(truth, dtype=np.float64)
    if u is None:
        raise FileNotFoundError("data/channel_truth.json holds no converged profile for "
                                f"class {c}")
    eps = sample_rng(SEED, c, "synthetic-observation-noise").standard_normal(len(u))
    return u * (1 + NOISE * eps), NOISE * np.abs(u)


def channel_ensemble(n: int = 256, precision: str = "fp64", first_id: int = 0,
                     alpha_u=ALPHA_U, max_iter=MAX_ITER) -> Ensemble:
    """The 256-draw channel ensemble: draw i -> class i mod 3. The synthetic observed
    profile of each class is that class's FP64 solve at (a1, beta*) = (0.31, 0.09)
    times (1 + 0.0014 eps), eps ~ N(0,1) seeded; sigma_i = 0.0014 |u_i|. The
    noise-free profiles come from data/channel_truth.json (the reference solver's
    own converged solve, written by data/make_channel_truth.py) when present, else
    from a GPU solve here."""
    batches, truth = [], []
    for c, (re_tau, ny) in enumerate(CLASSES):
        u = stored_truth(c)
        if u is None:
            probe = channel_batch(re_tau, ny, alpha_u=alpha_u, max_iter=MAX_ITER)
            res = probe.evaluate(np.array([[0.31, 0.09]]))
            u = np.asarray(res.rows[0].result.predictions)
        observed, sigma = class_observation(c, u)
        batches.append(channel_batch(re_tau, ny, observed, sigma, precision=precision,
                                     alpha_u=alpha_u, max_iter=max_iter))
        truth.append(u)
    ids = np.arange(first_id, first_id + n)
    return Ensemble(batches, uniform_design(ids), ids % 3, truth)


# ---------------------------------------------------------------- linear systems
LINEAR_SIZES = (64, 128, 256, 512)
LINEAR_SEED = 20261011


def poisson_system(n: int, seed: int):
    """Variable-coefficient 5-point Poisson system on an n x n grid of unit cells:
    face coefficients log-normal (sigma 1), a Dirichlet right edge by diagonal
    augmentation (twice a log-normal coefficient: the half-cell distance, as the
    reference adds area/delta for outlet faces, core/tests/test_amg_reuse.cpp:55-63),
    Neumann elsewhere, right-hand side N(0, 1). Faces: x-faces row by row, then
    y-faces row by row; cell c = j*n + i."""
    from .linear import LinearSystem

    rng = np.random.default_rng(seed)
    idx = np.arange(n * n).reshape(n, n)           # [j, i]
    own_x, nbr_x = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    own_y, nbr_y = idx[:-1, :].ravel(), idx[1:, :].ravel()
    own = np.concatenate([own_x, own_y]).astype(np.int32)
    nbr = np.concatenate([nbr_x, nbr_y]).astype(np.int32)
    c = np.exp(rng.standard_normal(len(own)))
    diag = np.zeros(n * n)
    np.add.at(diag, own, c)
    np.add.at(diag, nbr, c)
    diag[idx[:, -1]] += 2.0 * np.exp(rng.standard_normal(n))
    source = rng.standard_normal(n * n)
    return LinearSystem.from_arrays(diag, -c, -c, source, own, nbr)


def linear_batch_sizes(count: int = 512, seed: int = LINEAR_SEED) -> np.ndarray:
    """n of each system, uniform over {64, 128, 256, 512}."""
    return np.random.default_rng(seed).choice(LINEAR_SIZES, size=count)


def linear_workload(count: int = 512, seed: int = LINEAR_SEED, sizes=None):
    """The batch of `count` systems; system k uses seed + 1 + k."""
    sizes = linear_batch_sizes(count, seed) if sizes is None else sizes
    return [poisson_system(int(n), seed + 1 + k) for k, n in enumerate(sizes)]


# ---------------------------------------------------------------- bump-wall channel
def bump_geometry(nx: int = 200, h: float = 1.0, length: float = 9.0, width: float = 4.0):
    """Streamwise nodes and lower-wall heights of the periodic bump channel:
    y_w(x) = 0.5 h (1 + cos(2 pi (x - L/2) / W)) for |x - L/2| < W/2, else 0."""
    xn = np.linspace(0.0, length, nx + 1)
    yb = np.where(np.abs(xn - length / 2) < width / 2,
                  0.5 * h * (1 + np.cos(2 * np.pi * (xn - length / 2) / width)), 0.0)
    yb[0] = yb[-1] = 0.0
    return xn, yb


def bump_batch(nx: int = 200, ny: int = 100, max_iter: int = 200, tol: float = 1e-8,
               body_force: float = 4e-3, re: float = 5600.0,
               block_threads: int = 0) -> core.ForwardBatch:
    """The bump-wall channel (top 3.04 h, Re 5600 on h, y+ 1) as a ForwardBatch with
    6 velocity probes at x = 2; the body force drives a bulk velocity of order one."""
    xn, yb = bump_geometry(nx)
    mesh = core.Mesh.make_curved_channel_periodic_2d(xn, yb, 3.04, ny, re, 1.0)
    mesh.compute_wall_distance()
    obs = core.ObservationOperator()
    for yi in np.linspace(0.2, 2.8, 6):
        obs.add_velocity_profile(core.Vec3(2.0, float(yi), 0.0), 0, 0.0, 1e-2)
    st = core.SolverSettings(max_iterations=max_iter, convergence_tol=tol, alpha_u=0.4,
                             alpha_p=0.25, body_force=core.Vec3(body_force, 0.0, 0.0),
                             verbose=False, block_threads=block_threads)
    bcs = core.FlowBoundaryConditions.channel_defaults(mesh, 1.0, 1e-4, 10.0)
    return core.ForwardBatch(mesh, core.InferenceParameterSet.a1_betaStar(), obs, bcs,
                             1.0 / re, st, core.Vec3(0.3, 0.0, 0.0), 0.0, 1e-4, 10.0)


# ---------------------------------------------------------------- calibration study
CAL_HALF_CELLS = 64
CAL_TRUE_THETA = (0.3137, 0.0912)


def calibration_batch(observed=None, sigma=None) -> core.ForwardBatch:
    """The calibration study's channel (docs/figures/calibration_coverage.py:81-113):
    Re_tau 182.088 on 3 x 128 cells whose first cell matches a uniform 64-cell
    half-height tanh stretching, alpha_U 0.5, tol 1e-8, cap 150000, 30 stations;
    sigma[i] = inf drops station i from the likelihood (sigma 1e6)."""
    first_height = 1 + math.tanh(2 * (1 / CAL_HALF_CELLS - 1)) / math.tanh(2)
    mesh = core.Mesh.make_periodic_channel_2d(3, 2 * CAL_HALF_CELLS, 1.0, 1.0, 182.088,
                                              first_height * 182.088)
    mesh.compute_wall_distance()
    x, y = channel_probes(182.088)
    observed = np.zeros(len(x)) if observed is None else observed
    sigma = np.ones(len(x)) if sigma is None else sigma
    obs = core.ObservationOperator()
    for xi, yi, ui, si in zip(x, y, observed, sigma):
        obs.add_velocity_profile(core.Vec3(float(xi), float(yi), 0.0), 0, float(ui),
                                 float(si) if np.isfinite(si) else 1e6)
    st = core.SolverSettings(max_iterations=150000, convergence_tol=1e-8, alpha_u=0.5,
                             body_force=core.Vec3(1.0, 0.0, 0.0), verbose=False)
    bcs = core.FlowBoundaryConditions.channel_defaults(mesh, 1.0, 1.0, 10.0)
    return core.ForwardBatch(mesh, core.InferenceParameterSet.a1_betaStar(), obs, bcs,
                             1.0 / 182.088, st, core.Vec3(15.0, 0.0, 0.0), 0.0, 1.0, 10.0)


def calibration_study_batch():
    """The study's batch with a synthetic observed profile (the DNS profile is not
    shipped): this solver's own profile at CAL_TRUE_THETA times (1 + 0.0014 eps), and
    sigma_i = 0.0014 |u_i| on every third station (the likelihood third), the rest
    dropped."""
    probe = calibration_batch()
    res = probe.evaluate(np.array([CAL_TRUE_THETA]))
    if res.rows[0].result.status != core.EvaluationStatus.Converged:
        raise RuntimeError("the synthetic truth solve did not converge")
    u = np.asarray(res.rows[0].result.predictions)
    eps = sample_rng(SEED, 99, "synthetic-observation-noise").standard_normal(len(u))
    group = np.arange(len(u)) % 3
    sigma = np.where(group == 0, NOISE * np.abs(u), np.inf)
    return calibration_batch(u * (1 + NOISE * eps), sigma), u
