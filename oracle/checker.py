"""Test infrastructure only: ctypes access to the two CPU checkers under oracle/.

* ``oracle/_ref/libcfdr_ref.so`` -- the reference's own C++ sources compiled with
  g++ (oracle/Makefile) behind a thin C-ABI harness (oracle/ref_harness.cpp).
* ``oracle/librq_oracle.so`` -- the C++ restatement of the reference algorithm
  (oracle/rq_oracle.cpp), which also exposes the device-style linear solvers so
  the GPU path can be checked iteration by iteration.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py use
this module. The product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libcfdr_ref.so"
ORACLE_LIB = HERE / "librq_oracle.so"

# SSTCoefficients defaults (core/include/SSTModel.hpp:12-27), InferenceParameterSet order
# (core/include/InferenceParameters.hpp:11-14).
DEFAULT_COEFFS = (0.85, 0.5, 0.075, 5.0 / 9.0, 1.0, 0.856, 0.0828, 0.44, 0.09, 0.31, 0.41)
P_AMG, P_PCG, P_BICGSTAB = 0, 1, 2
STATUS = ("Converged", "Unconverged", "Diverged", "InvalidParameters", "Unknown")
NFIELD, NHIST = 11, 11
FIELD_NAMES = ("Ux", "Uy", "Uz", "p", "k", "omega", "nuT", "F1", "F2", "Pk", "CDkw")


class OrcCase(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("curved", C.c_int32), ("pad0", C.c_int32),
        ("lx", C.c_double), ("h", C.c_double), ("re_tau", C.c_double), ("yplus", C.c_double),
        ("x_nodes", C.POINTER(C.c_double)), ("y_bottom", C.POINTER(C.c_double)),
        ("y_top", C.c_double), ("re_mesh", C.c_double),
        ("nu", C.c_double), ("bc_u", C.c_double), ("bc_k", C.c_double), ("bc_w", C.c_double),
        ("init_u", C.c_double * 3), ("init_p", C.c_double), ("init_k", C.c_double),
        ("init_w", C.c_double),
        ("max_iter", C.c_int32), ("inner_iter", C.c_int32), ("conv_window", C.c_int32),
        ("monitor_interval", C.c_int32), ("turb_start", C.c_int32),
        ("nut_floor_iters", C.c_int32), ("pressure_solver", C.c_int32), ("pad1", C.c_int32),
        ("tol", C.c_double), ("inner_tol", C.c_double), ("alpha_u", C.c_double),
        ("alpha_p", C.c_double), ("alpha_k", C.c_double), ("alpha_w", C.c_double),
        ("body_force", C.c_double * 3), ("div_limit", C.c_double), ("k_min", C.c_double),
        ("k_max", C.c_double), ("omega_min", C.c_double),
        ("coeffs", C.c_double * 11),
        ("n_obs", C.c_int32), ("obs_component", C.c_int32),
        ("obs_x", C.POINTER(C.c_double)), ("obs_y", C.POINTER(C.c_double)),
        ("obs_value", C.POINTER(C.c_double)), ("obs_sigma", C.POINTER(C.c_double)),
    ]


class OrcResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int32), ("converged", C.c_int32),
        ("diverged", C.c_int32), ("stalled", C.c_int32), ("n_hist", C.c_int32),
        ("loglik", C.c_double), ("final_worst", C.c_double), ("contraction_rate", C.c_double),
    ]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Case:
    """One periodic-channel (or curved periodic) SIMPLE + SST solve description."""

    nx: int = 3
    ny: int = 128
    curved: bool = False
    lx: float = 1.0
    h: float = 1.0
    re_tau: float = 182.088
    yplus: float = 0.5
    x_nodes: np.ndarray | None = None
    y_bottom: np.ndarray | None = None
    y_top: float = 0.0
    re_mesh: float = 0.0
    nu: float = 1.0 / 182.088
    bc: tuple = (1.0, 1.0, 10.0)
    init_u: tuple = (15.0, 0.0, 0.0)
    init_p: float = 0.0
    init_k: float = 1.0
    init_w: float = 10.0
    max_iter: int = 150000
    inner_iter: int = 200
    conv_window: int = 25
    monitor_interval: int = 10
    turb_start: int = 5
    nut_floor_iters: int = 500
    pressure_solver: int = P_AMG
    tol: float = 1e-10
    inner_tol: float = 1e-3
    alpha_u: float = 0.5
    alpha_p: float = 0.3
    alpha_k: float = 0.5
    alpha_w: float = 0.5
    body_force: tuple = (1.0, 0.0, 0.0)
    div_limit: float = 1e6
    k_min: float = 1e-10
    k_max: float = 1e10
    omega_min: float = 1e-6
    coeffs: tuple = DEFAULT_COEFFS
    obs_x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    obs_y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    obs_value: np.ndarray = field(default_factory=lambda: np.zeros(0))
    obs_sigma: np.ndarray = field(default_factory=lambda: np.zeros(0))
    obs_component: int = 0

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny

    def with_theta(self, a1: float, beta_star: float) -> "Case":
        c = list(self.coeffs)
        c[9], c[8] = a1, beta_star
        import dataclasses

        return dataclasses.replace(self, coeffs=tuple(c))

    def struct(self):
        """ctypes struct plus the arrays it points into (kept alive by the caller)."""
        keep = []

        def arr(a):
            a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
            keep.append(a)
            return _dptr(a)

        s = OrcCase()
        s.nx, s.ny, s.curved = self.nx, self.ny, int(self.curved)
        s.lx, s.h, s.re_tau, s.yplus = self.lx, self.h, self.re_tau, self.yplus
        if self.curved:
            s.x_nodes, s.y_bottom = arr(self.x_nodes), arr(self.y_bottom)
        s.y_top, s.re_mesh, s.nu = self.y_top, self.re_mesh, self.nu
        s.bc_u, s.bc_k, s.bc_w = self.bc
        s.init_u[:] = self.init_u
        s.init_p, s.init_k, s.init_w = self.init_p, self.init_k, self.init_w
        s.max_iter, s.inner_iter = self.max_iter, self.inner_iter
        s.conv_window, s.monitor_interval = self.conv_window, self.monitor_interval
        s.turb_start, s.nut_floor_iters = self.turb_start, self.nut_floor_iters
        s.pressure_solver = self.pressure_solver
        s.tol, s.inner_tol = self.tol, self.inner_tol
        s.alpha_u, s.alpha_p, s.alpha_k, s.alpha_w = (
            self.alpha_u, self.alpha_p, self.alpha_k, self.alpha_w)
        s.body_force[:] = self.body_force
        s.div_limit, s.k_min, s.k_max, s.omega_min = (
            self.div_limit, self.k_min, self.k_max, self.omega_min)
        s.coeffs[:] = self.coeffs
        s.n_obs, s.obs_component = len(self.obs_x), self.obs_component
        if len(self.obs_x):
            s.obs_x, s.obs_y = arr(self.obs_x), arr(self.obs_y)
            s.obs_value, s.obs_sigma = arr(self.obs_value), arr(self.obs_sigma)
        return s, keep


@dataclass
class SolveOut:
    status: str
    iterations: int
    converged: bool
    diverged: bool
    stalled: bool
    loglik: float
    final_worst: float
    contraction_rate: float
    fields: np.ndarray  # (11, nCells)
    predictions: np.ndarray
    history: np.ndarray  # (n, 11)

    def field(self, name: str) -> np.ndarray:
        return self.fields[FIELD_NAMES.index(name)]


def channel_probes(re_tau: float, n: int = 30, lo: float = 1.0, hi: float = 175.0):
    """Probe locations at n log-spaced y+ in [lo, hi] (u_tau = 1, h = 1), x = 0.5,
    as the calibration stations (docs/figures/calibration_coverage.py:71-78)."""
    yp = np.geomspace(lo, hi, n)
    return np.full(n, 0.5), yp / re_tau


def config1_case(**kw) -> Case:
    """Plain small case: Re_tau 182.088 channel on 3x128 cells, y+ 0.5, tol 1e-10."""
    x, y = channel_probes(182.088)
    base = Case(obs_x=x, obs_y=y, obs_value=np.zeros(30), obs_sigma=np.full(30, 1e-3))
    import dataclasses

    return dataclasses.replace(base, **kw)


def _lib(path: Path):
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
    return C.CDLL(str(path), mode=os.RTLD_NOW)


_LIBS: dict[str, C.CDLL] = {}


def lib(kind: str) -> C.CDLL:
    if kind not in _LIBS:
        _LIBS[kind] = _lib(REF_LIB if kind == "ref" else ORACLE_LIB)
    return _LIBS[kind]


def have(kind: str) -> bool:
    return (REF_LIB if kind == "ref" else ORACLE_LIB).exists()


def solve(case: Case, kind: str = "ref", hist_cap: int = 0) -> SolveOut:
    """Run one ForwardModel evaluation through the reference ('ref') or the
    restatement ('oracle')."""
    L = lib(kind)
    fn = L.ref_solve if kind == "ref" else L.orc_solve
    s, keep = case.struct()
    res = OrcResult()
    n = case.n_cells
    fields = np.zeros((NFIELD, n))
    pred = np.zeros(max(len(case.obs_x), 1))
    hist = np.zeros((max(hist_cap, 1), NHIST))
    rc = fn(C.byref(s), C.byref(res), _dptr(fields), _dptr(pred), _dptr(hist),
            C.c_int32(hist_cap))
    if rc != 0:
        err = (L.ref_last_error if kind == "ref" else L.orc_last_error)
        err.restype = C.c_char_p
        raise RuntimeError(err().decode())
    nh = min(res.n_hist, hist_cap)
    return SolveOut(STATUS[res.status], res.iterations, bool(res.converged), bool(res.diverged),
                    bool(res.stalled), res.loglik, res.final_worst, res.contraction_rate, fields,
                    pred[: len(case.obs_x)], hist[:nh])


@dataclass
class SequenceOut:
    """One ForwardModel's calls in order: verdicts, iterations, log-likelihoods,
    predictions (calls x probes), whether each call started warm, and the warm-start
    cache's retained bytes after each call."""
    status: list
    iterations: np.ndarray
    loglik: np.ndarray
    predictions: np.ndarray
    used_warm: np.ndarray
    retained: np.ndarray


def solve_sequence(case: Case, thetas, kind: str = "ref", max_size: int = 50,
                   threshold: float = 0.5, byte_budget: int = 64 * 1024 * 1024) -> SequenceOut:
    """Evaluate theta rows (a1, betaStar) one after another on ONE ForwardModel with its
    warm-start cache, through the reference ('ref') or the restatement ('oracle')."""
    L = lib(kind)
    fn = L.ref_solve_sequence if kind == "ref" else L.orc_solve_sequence
    th = np.ascontiguousarray(np.asarray(thetas, dtype=np.float64).reshape(-1, 2))
    m = len(th)
    s, keep = case.struct()
    res = (OrcResult * m)()
    nobs = len(case.obs_x)
    pred = np.zeros((m, max(nobs, 1)))
    used = np.zeros(m, dtype=np.int32)
    kept = np.zeros(m, dtype=np.int64)
    rc = fn(C.byref(s), _dptr(th), C.c_int32(m), C.c_int32(max_size), C.c_double(threshold),
            C.c_int64(byte_budget), res, _dptr(pred), used.ctypes.data_as(C.POINTER(C.c_int32)),
            kept.ctypes.data_as(C.POINTER(C.c_int64)))
    if rc != 0:
        err = (L.ref_last_error if kind == "ref" else L.orc_last_error)
        err.restype = C.c_char_p
        raise RuntimeError(err().decode())
    return SequenceOut([STATUS[r.status] for r in res], np.array([r.iterations for r in res]),
                       np.array([r.loglik for r in res]), pred[:, :nobs], used.astype(bool), kept)


def solve_snapshot(case: Case) -> dict | None:
    """The reference's evaluateWithDiagnostics(theta, snapshot=True) on a cold model:
    {'status', 'iterations', 'cells' (11, nC), 'boundary' (11, nB), 'face_fluxes' (nF),
    'turb_established'}, blocks Ux Uy Uz p k omega nuT F1 F2 Pk CDkw; None without a
    snapshot. Reference only (the restatement keeps no snapshot)."""
    L = lib("ref")
    s, keep = case.struct()
    cells_, faces_, ni = mesh(case, "ref")
    nc, nf = len(cells_), len(faces_)
    nb = nf - ni
    res = OrcResult()
    cells = np.zeros((NFIELD, nc))
    bnd = np.zeros((NFIELD, max(nb, 1)))
    flux = np.zeros(nf)
    est, has = C.c_int32(), C.c_int32()
    rc = L.ref_solve_snapshot(C.byref(s), C.byref(res), _dptr(cells), _dptr(bnd), _dptr(flux),
                              C.byref(est), C.byref(has))
    if rc != 0:
        L.ref_last_error.restype = C.c_char_p
        raise RuntimeError(L.ref_last_error().decode())
    if not has.value:
        return None
    return dict(status=STATUS[res.status], iterations=res.iterations, loglik=res.loglik,
                cells=cells, boundary=bnd[:, :nb], face_fluxes=flux,
                turb_established=bool(est.value))


def mesh_save_binary(case: Case, path) -> None:
    """The reference's Mesh::saveBinary of the case's generated mesh (reference only)."""
    L = lib("ref")
    s, keep = case.struct()
    if L.ref_mesh_save_binary(C.byref(s), os.fsencode(path)) != 0:
        L.ref_last_error.restype = C.c_char_p
        raise RuntimeError(L.ref_last_error().decode())


def mesh(case: Case, kind: str = "ref"):
    """Cell (cx, cy, vol, wd) and face (owner, nbr, cx, cy, nx, ny, area, delta, dx, dy,
    weight, shift_x, patch) arrays of the mesh as the checker builds it."""
    L = lib(kind)
    fn = L.ref_mesh if kind == "ref" else L.orc_mesh
    s, keep = case.struct()
    nc, nf, ni = C.c_int32(), C.c_int32(), C.c_int32()
    rc = fn(C.byref(s), C.byref(nc), C.byref(nf), C.byref(ni), None, None)
    assert rc == 0
    cells = np.zeros((nc.value, 4))
    faces = np.zeros((nf.value, 13))
    rc = fn(C.byref(s), C.byref(nc), C.byref(nf), C.byref(ni), _dptr(cells), _dptr(faces))
    assert rc == 0
    return cells, faces, ni.value


def linear_solve(kind_solver: int, diag, upper, lower, source, own, nbr, x0, max_iter, tol,
                 lib_kind: str = "ref"):
    """kind_solver: 0 AMG 1 PCG 2 BiCGSTAB 3 GaussSeidel (reference factory names)."""
    L = lib(lib_kind)
    fn = L.ref_linear_solve if lib_kind == "ref" else L.orc_linear_solve
    n, nif = len(diag), len(upper)
    x = np.array(x0, dtype=np.float64).copy()
    d = [np.ascontiguousarray(np.asarray(a, np.float64)) for a in (diag, upper, lower, source)]
    o = np.ascontiguousarray(np.asarray(own, np.int32))
    b = np.ascontiguousarray(np.asarray(nbr, np.int32))
    it, fr, ir, cv = C.c_int32(), C.c_double(), C.c_double(), C.c_int32()
    rc = fn(C.c_int32(kind_solver), C.c_int32(n), C.c_int32(nif), _dptr(d[0]), _dptr(d[1]),
            _dptr(d[2]), _dptr(d[3]), o.ctypes.data_as(C.POINTER(C.c_int32)),
            b.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(x), C.c_int32(max_iter),
            C.c_double(tol), C.byref(it), C.byref(fr), C.byref(ir), C.byref(cv))
    assert rc == 0
    return x, dict(iterations=it.value, final_res=fr.value, initial_res=ir.value,
                   converged=bool(cv.value))


def rel_err(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


__all__ = ["Case", "config1_case", "channel_probes", "solve", "solve_sequence", "solve_snapshot", "mesh_save_binary", "mesh", "linear_solve", "have",
           "rel_err", "DEFAULT_COEFFS", "P_AMG", "P_PCG", "P_BICGSTAB", "FIELD_NAMES", "math"]
