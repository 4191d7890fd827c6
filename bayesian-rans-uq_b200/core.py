"""Host-side mirror of the reference forward-model API (the ``cfdr._core``
pybind11 module, rans-uq/python/bindings.cpp:452-975) on the B200 path.

Same names, argument meaning and error behaviour as the reference for the calls
a calibration makes: ``Mesh.make_periodic_channel_2d`` /
``make_curved_channel_periodic_2d``, ``SolverSettings``,
``FlowBoundaryConditions.channel_defaults``, ``InferenceParameterSet``,
``ObservationOperator.add_velocity_profile``, ``ForwardBatch(...).evaluate``
and ``ForwardModel.evaluate[_with_diagnostics]``. Every solve runs on the GPU
through the C ABI (include/rq_b200.h); nothing here computes a flow field.
"""
from __future__ import annotations

import ctypes as C
import os
import enum
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


class EvaluationStatus(enum.IntEnum):
    """EvaluationStatus (core/include/EvaluationTypes.hpp:6); Python names as bindings.cpp:464-469."""

    Converged = 0
    Unconverged = 1
    DivergenceDetected = 2
    InvalidParameters = 3
    Unknown = 4


@dataclass
class Vec3:
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0


@dataclass
class Mesh:
    """A streamwise-periodic mesh description (the GPU path's mesh family)."""

    kind: int
    nx: int
    ny: int
    lx: float = 1.0
    h: float = 1.0
    re_tau: float = 0.0
    yplus: float = 1.0
    x_nodes: np.ndarray | None = None
    y_bottom: np.ndarray | None = None
    y_top: float = 0.0
    re: float = 0.0
    _wall_distance: bool = False
    _stored: dict | None = None

    @staticmethod
    def make_periodic_channel_2d(nx, ny, Lx, h, re_tau, yplus_target=1.0) -> "Mesh":
        """Mesh::makePeriodicChannel2D (core/src/Mesh.cpp:511-521)."""
        if nx < 3 or ny < 1 or not (Lx > 0 and h > 0 and re_tau > 0 and yplus_target > 0):
            raise ValueError("periodic channel needs nx >= 3, ny >= 1 and positive sizes")
        return Mesh(N.MESH_CHANNEL, int(nx), int(ny), float(Lx), float(h), float(re_tau),
                    float(yplus_target))

    @staticmethod
    def make_curved_channel_periodic_2d(x_nodes, y_bottom, y_top, ny, re=0.0,
                                        yplus_target=1.0) -> "Mesh":
        """Mesh::makeCurvedChannelPeriodic2D (core/src/Mesh.cpp:490-509)."""
        x = np.ascontiguousarray(np.asarray(x_nodes, dtype=np.float64))
        y = np.ascontiguousarray(np.asarray(y_bottom, dtype=np.float64))
        if x.ndim != 1 or x.shape != y.shape or len(x) < 4:
            raise ValueError("makeCurvedChannelPeriodic2D: need nx+1 x nodes and matching "
                             "yBottom samples")
        return Mesh(N.MESH_CURVED, len(x) - 1, int(ny), x_nodes=x, y_bottom=y,
                    y_top=float(y_top), re=float(re), yplus=float(yplus_target))

    def compute_wall_distance(self) -> None:
        self._wall_distance = True

    def wall_distance_valid(self) -> bool:
        return self._wall_distance

    def n_cells(self) -> int:
        return self.nx * self.ny

    def desc(self) -> N.MeshDesc:
        d = N.MeshDesc()
        d.kind, d.nx, d.ny = self.kind, self.nx, self.ny
        d.lx, d.h, d.re_tau, d.yplus = self.lx, self.h, self.re_tau, self.yplus
        if self.kind == N.MESH_CURVED:
            d.x_nodes, d.y_bottom = N.dptr(self.x_nodes), N.dptr(self.y_bottom)
            d.y_top, d.re = self.y_top, self.re
        return d

    def cell_geometry(self) -> np.ndarray:
        """(n_cells, 4): centre x, centre y, volume, wall distance."""
        d = self.desc()
        nc = C.c_int32()
        N.call("rq_mesh_geometry", C.byref(d), C.byref(nc), None)
        out = np.zeros((nc.value, 4))
        N.call("rq_mesh_geometry", C.byref(d), C.byref(nc), N.dptr(out))
        return out

    def save_binary(self, path) -> None:
        """Mesh::saveBinary (core/src/Mesh.cpp:751-811): the reference's MSH2 binary mesh
        file, byte-identical to the reference's for the same generator call."""
        d = self.desc()
        N.call("rq_mesh_save_binary", C.byref(d), os.fsencode(path))

    # ---- introspection as the reference binding exposes it (rans-uq/python/bindings.cpp:
    # 128-246, 556-571), read back from the mesh's own binary file so that every array is
    # the reference's, in its face, node and patch order
    def _mesh_record(self) -> dict:
        if self._stored is None:
            import tempfile

            with tempfile.TemporaryDirectory() as d:
                path = os.path.join(d, "mesh.bin")
                self.save_binary(path)
                with open(path, "rb") as f:
                    self._stored = _read_mesh_binary(f.read())
        return self._stored

    def n_faces(self) -> int:
        return len(self._mesh_record()["faces"])

    def n_internal_faces(self) -> int:
        return self._mesh_record()["n_internal"]

    def n_nodes(self) -> int:
        return len(self._mesh_record()["nodes"])

    def n_patches(self) -> int:
        return len(self._mesh_record()["patches"])

    def patch_names(self) -> list:
        return [p["name"] for p in self._mesh_record()["patches"]]

    def patch_types(self) -> list:
        return [p["type"] for p in self._mesh_record()["patches"]]

    def cell_centers(self) -> np.ndarray:
        """(n_cells, 3) cell centres (z = half the unit depth)."""
        return self._mesh_record()["cell_centers"].copy()

    def cell_volumes(self) -> np.ndarray:
        return self._mesh_record()["cell_volumes"].copy()

    def node_coords(self) -> np.ndarray:
        return self._mesh_record()["nodes"].copy()

    def face_centers(self) -> np.ndarray:
        return np.ascontiguousarray(self._mesh_record()["faces"]["center"])

    def wall_patch_data(self, name: str) -> dict:
        """meshWallPatchData (bindings.cpp:186-233): owner, delta, centre, normal and area
        of the named patch's faces, in patch order."""
        rec = self._mesh_record()
        for p in rec["patches"]:
            if p["name"] == name:
                f = rec["faces"][p["faces"]]
                return {"name": p["name"], "type": p["type"], "n_faces": len(f),
                        "owner": f["owner"].astype(np.int32), "delta": f["delta"].copy(),
                        "center": np.ascontiguousarray(f["center"]),
                        "normal": np.ascontiguousarray(f["normal"]),
                        "area": f["area"].copy()}
        raise RuntimeError(f"Mesh::wall_patch_data: unknown patch '{name}'")


_FACE_RECORD = np.dtype([("owner", "<i4"), ("neighbor", "<i4"), ("patch", "<i4"),
                         ("center", "<f8", 3), ("normal", "<f8", 3), ("area", "<f8"),
                         ("delta", "<f8"), ("d", "<f8", 3), ("weight", "<f8"),
                         ("shift", "<f8", 3)])


def _read_mesh_binary(data: bytes) -> dict:
    """The arrays of an MSH2 binary mesh file (Mesh::loadBinary's layout,
    core/src/Mesh.cpp:813-905): nodes, face records, cell centres / volumes / face
    lists, and named patches with their face indices."""
    if np.frombuffer(data, "<u4", 1)[0] != 0x4D534832:
        raise ValueError("not an MSH2 binary mesh")
    nc, nf, nn, npatch, n_internal = (int(v) for v in np.frombuffer(data, "<i4", 5, 4))
    off = 24
    nodes = np.frombuffer(data, "<f8", 3 * nn, off).reshape(nn, 3).copy()
    off += 24 * nn
    faces = np.frombuffer(data, _FACE_RECORD, nf, off).copy()
    off += _FACE_RECORD.itemsize * nf
    centers, volumes, cell_faces = np.empty((nc, 3)), np.empty(nc), []
    for c in range(nc):
        rec = np.frombuffer(data, "<f8", 4, off)
        centers[c], volumes[c] = rec[:3], rec[3]
        k = int(np.frombuffer(data, "<i4", 1, off + 32)[0])
        cell_faces.append(np.frombuffer(data, "<i4", k, off + 36).copy())
        off += 36 + 4 * k
    patches = []
    for _ in range(npatch):
        text = []
        for _field in range(2):
            k = int(np.frombuffer(data, "<i4", 1, off)[0])
            text.append(data[off + 4:off + 4 + k].decode())
            off += 4 + k
        k = int(np.frombuffer(data, "<i4", 1, off)[0])
        patches.append({"name": text[0], "type": text[1],
                        "faces": np.frombuffer(data, "<i4", k, off + 4).copy()})
        off += 4 + 4 * k
    if off != len(data):
        raise ValueError("unexpected trailing bytes in the binary mesh")
    return {"n_internal": n_internal, "nodes": nodes, "faces": faces, "cell_centers": centers,
            "cell_volumes": volumes, "cell_faces": cell_faces, "patches": patches}


@dataclass
class SolverSettings:
    """SolverSettings (core/include/FlowFields.hpp:70-241) with the reference defaults."""

    max_iterations: int = 500
    convergence_tol: float = 1e-5
    divergence_limit: float = 1e6
    legacy_convergence: bool = False
    convergence_window: int = 25
    monitor_interval: int = 10
    alpha_u: float = 0.7
    alpha_p: float = 0.3
    alpha_k: float = 0.5
    alpha_omega: float = 0.5
    inner_iterations: int = 200
    inner_tolerance: float = 1e-3
    turb_start_iter: int = 5
    turb_update_interval: int = 1
    nut_floor_iters: int = 500
    legacy_rhie_chow_gate: bool = False
    legacy_omega_wall_pinning: bool = False
    momentum_convection: str = "limitedLinearUpwind"
    turbulence_convection: str = "limitedLinearUpwind"
    alpha_injection: float = 0.3
    body_force: Vec3 = field(default_factory=Vec3)
    k_min: float = 1e-10
    k_max: float = 1e10
    omega_min: float = 1e-6
    report_interval: int = 10
    verbose: bool = True
    pressure_solver: str = "AMG"
    momentum_solver: str = "BiCGSTAB"
    turbulence_solver: str = "BiCGSTAB"
    use_wall_functions: bool = False
    alpha_t: float = 0.7       # compressible solver only; kept for the settings' shape
    von_karman: float = 0.41   # wall functions only (rejected on this path)
    sst_variant: int = 0
    # B200 path only
    precision: str = "fp64"
    block_threads: int = 0

    def native(self) -> N.Settings:
        unsupported = []
        if self.legacy_convergence:
            unsupported.append("legacy_convergence")
        if self.legacy_rhie_chow_gate:
            unsupported.append("legacy_rhie_chow_gate")
        if self.legacy_omega_wall_pinning:
            unsupported.append("legacy_omega_wall_pinning")
        if self.momentum_convection != "limitedLinearUpwind" or \
                self.turbulence_convection != "limitedLinearUpwind":
            unsupported.append("convection schemes other than limitedLinearUpwind")
        if self.use_wall_functions:
            unsupported.append("wall functions")
        if self.sst_variant != 0:
            unsupported.append("SST variants other than Full")
        if self.momentum_solver != "BiCGSTAB" or self.turbulence_solver != "BiCGSTAB":
            unsupported.append("momentum/turbulence solvers other than BiCGSTAB")
        if unsupported:
            raise NotImplementedError("outside the B200 forward-model path: " + ", ".join(unsupported))
        for name in ("momentum_convection", "turbulence_convection"):
            if getattr(self, name) not in ("upwind", "linearUpwind", "limitedLinearUpwind"):
                raise ValueError(f"unknown SIMPLE convection scheme: {getattr(self, name)}")
        if self.pressure_solver not in N.SOLVERS:
            raise ValueError(f"unknown linear solver: '{self.pressure_solver}'")
        if self.precision not in N.PRECISIONS:
            raise ValueError(f"unknown precision: '{self.precision}'")
        s = N.Settings()
        s.max_iterations, s.inner_iterations = self.max_iterations, self.inner_iterations
        s.convergence_window, s.monitor_interval = self.convergence_window, self.monitor_interval
        s.turb_start_iter, s.turb_update_interval = self.turb_start_iter, self.turb_update_interval
        s.nut_floor_iters = self.nut_floor_iters
        s.pressure_solver = N.SOLVERS[self.pressure_solver]
        s.precision = N.PRECISIONS[self.precision]
        s.block_threads = self.block_threads
        s.convergence_tol, s.inner_tolerance = self.convergence_tol, self.inner_tolerance
        s.divergence_limit = self.divergence_limit
        s.alpha_u, s.alpha_p, s.alpha_k, s.alpha_omega = (
            self.alpha_u, self.alpha_p, self.alpha_k, self.alpha_omega)
        s.body_force[:] = (self.body_force.x, self.body_force.y, self.body_force.z)
        s.k_min, s.k_max, s.omega_min = self.k_min, self.k_max, self.omega_min
        return s


@dataclass
class FlowBoundaryConditions:
    u_in: float
    k_in: float
    omega_in: float

    @staticmethod
    def channel_defaults(mesh: Mesh, u_in: float, k_in: float, omega_in: float):
        """FlowBoundaryConditions::channelDefaults (BoundaryCondition.hpp:113-167): every
        patch of the periodic meshes is a no-slip k-omega wall."""
        return FlowBoundaryConditions(float(u_in), float(k_in), float(omega_in))


# SSTCoefficients defaults (core/include/SSTModel.hpp:12-27), InferenceParameterSet order
SST_DEFAULTS = (0.85, 0.5, 0.075, 5.0 / 9.0, 1.0, 0.856, 0.0828, 0.44, 0.09, 0.31, 0.41)
SST_NAMES = ("sigma_k1", "sigma_w1", "beta1", "alpha1", "sigma_k2", "sigma_w2", "beta2",
             "alpha2", "betaStar", "a1", "kappa")
_LO = (0.1, 0.1, 0.01, 0.1, 0.1, 0.1, 0.01, 0.1, 0.01, 0.1, 0.35)
_HI = (2.0, 2.0, 0.2, 1.5, 2.0, 2.0, 0.2, 1.5, 0.2, 0.8, 0.50)


@dataclass
class InferenceParameterSet:
    """InferenceParameterSet (core/include/InferenceParameters.hpp:18-188)."""

    name: str
    active_indices: tuple
    base: tuple = SST_DEFAULTS

    def validate(self) -> None:
        if not self.active_indices:
            raise ValueError("inference parameters require at least one active index")
        if any(i < 0 or i > 10 for i in self.active_indices):
            raise ValueError("inference parameter index must be in [0,10]")
        if len(set(self.active_indices)) != len(self.active_indices):
            raise ValueError("inference parameter indices must be unique")

    def n_active(self) -> int:
        return len(self.active_indices)

    def active_names(self) -> list:
        return [SST_NAMES[i] for i in self.active_indices]

    def lower_bounds(self) -> list:
        return [_LO[i] for i in self.active_indices]

    def upper_bounds(self) -> list:
        return [_HI[i] for i in self.active_indices]

    def in_bounds(self, theta) -> bool:
        theta = list(theta)
        if len(theta) != self.n_active():
            return False
        for v, lo, hi in zip(theta, self.lower_bounds(), self.upper_bounds()):
            if v < lo or v > hi or math.isnan(v) or math.isinf(v):
                return False
        return True

    def unpack(self, theta) -> list:
        if len(theta) != self.n_active():
            raise RuntimeError(f"theta size mismatch: expected {self.n_active()}, got {len(theta)}")
        full = list(self.base)
        for i, v in zip(self.active_indices, theta):
            full[i] = float(v)
        return full

    def pack(self, coeffs) -> list:
        return [coeffs[i] for i in self.active_indices]

    @staticmethod
    def a1_betaStar():
        return InferenceParameterSet("a1_betaStar", (9, 8))

    @staticmethod
    def inlet_turb():
        return InferenceParameterSet("inletTurb", (2, 1))

    @staticmethod
    def near_wall4():
        return InferenceParameterSet("nearWall4", (9, 8, 2, 0))

    @staticmethod
    def all11():
        return InferenceParameterSet("all11", tuple(range(11)))

    @staticmethod
    def live10():
        return InferenceParameterSet("live10", tuple(range(10)))

    @staticmethod
    def from_indices(name, idx):
        p = InferenceParameterSet(name, tuple(int(i) for i in idx))
        p.validate()
        return p


@dataclass
class _Probe:
    location: Vec3
    component: int
    observed: float
    sigma_obs: float
    sigma_model: float


class ObservationOperator:
    """Velocity-profile observations (ObservationOperator::addVelocityProfile,
    core/include/ObservationOperator.hpp:222-234) and the Gaussian log-likelihood."""

    def __init__(self) -> None:
        self._probes: list[_Probe] = []

    def add_velocity_profile(self, location, comp, u_obs, sigma, sigma_model=0.0) -> None:
        loc = location if isinstance(location, Vec3) else Vec3(*location)
        if not all(math.isfinite(v) for v in (loc.x, loc.y, loc.z)):
            raise ValueError("observation location must be finite")
        if comp < 0 or comp > 2:
            raise ValueError("velocity observation component must be in [0,2]")
        var = sigma * sigma + sigma_model * sigma_model
        if not (math.isfinite(u_obs) and math.isfinite(sigma) and sigma >= 0 and
                math.isfinite(sigma_model) and sigma_model >= 0 and math.isfinite(var) and var > 0):
            raise ValueError("Gaussian measurements require finite values, nonnegative "
                             "uncertainties and finite positive total variance")
        if self._probes and comp != self._probes[0].component:
            raise NotImplementedError("one velocity component per problem on the B200 path")
        self._probes.append(_Probe(loc, int(comp), float(u_obs), float(sigma), float(sigma_model)))

    def n_obs(self) -> int:
        return len(self._probes)

    # The integral and feature observables of other flows (bindings.cpp: add_drag,
    # add_skin_friction, add_reattachment_length) and the host-side evaluate(mesh,
    # fields, nu) are not on this path: the probes are evaluated on the GPU inside
    # each solve. They fail loudly rather than being ignored.
    def add_drag(self, *args, **kwargs):
        raise NotImplementedError("drag observations are outside the B200 forward-model path")

    def add_skin_friction(self, *args, **kwargs):
        raise NotImplementedError("skin-friction observations are outside the B200 "
                                  "forward-model path")

    def add_reattachment_length(self, *args, **kwargs):
        raise NotImplementedError("reattachment-length observations are outside the B200 "
                                  "forward-model path")

    def prepare(self, mesh) -> None:
        """Probe stencils are prepared on the host when a batch is built (nothing to do)."""

    def evaluate(self, mesh, fields, nu):
        raise NotImplementedError("predictions are evaluated on the GPU by every solve; "
                                  "use the rows' predictions")

    def log_likelihood_from_predictions(self, predictions) -> float:
        """ObservationOperator::logLikelihood (ObservationOperator.hpp:592-609)."""
        if len(predictions) != len(self._probes):
            raise ValueError("Likelihood prediction count does not match observations")
        ll = 0.0
        for p, v in zip(self._probes, predictions):
            if not math.isfinite(v):
                raise ValueError("Likelihood predictions must be finite")
            var = p.sigma_obs * p.sigma_obs + p.sigma_model * p.sigma_model
            d = v - p.observed
            ll += -0.5 * d * d / var
        return ll

    def arrays(self):
        n = len(self._probes)
        cols = np.zeros((5, n))
        for i, p in enumerate(self._probes):
            cols[:, i] = (p.location.x, p.location.y, p.observed, p.sigma_obs, p.sigma_model)
        return [np.ascontiguousarray(c) for c in cols]


@dataclass
class EvaluationResult:
    status: EvaluationStatus
    log_lik: float
    predictions: np.ndarray
    simple_iters: int


@dataclass
class ForwardBatchRow:
    result: EvaluationResult
    final_worst_measure: float
    contraction_rate_u: float
    stalled: bool
    error: str


@dataclass
class ForwardBatchResult:
    rows: list
    n_observations: int

    @property
    def predictions(self) -> np.ndarray:
        if not self.rows:
            return np.zeros((0, self.n_observations))
        return np.stack([r.result.predictions for r in self.rows])

    @property
    def log_likelihoods(self) -> np.ndarray:
        return np.array([r.result.log_lik for r in self.rows])

    @property
    def statuses(self) -> list:
        return [r.result.status for r in self.rows]

    @property
    def iteration_counts(self) -> np.ndarray:
        return np.array([r.result.simple_iters for r in self.rows], dtype=np.int32)

    @property
    def errors(self) -> list:
        return [r.error for r in self.rows]

    @property
    def convergence_mask(self) -> np.ndarray:
        return np.array([r.result.status == EvaluationStatus.Converged for r in self.rows])


class _Problem:
    """Owns one device-resident mesh class (rq_problem)."""

    def __init__(self, mesh, params, obs, bcs, nu, settings, u_init, p_init, k_init, omega_init):
        params.validate()
        if not mesh.wall_distance_valid():
            raise ValueError("ForwardBatch needs compute_wall_distance before construction")
        self.params, self.obs = params, obs
        self.mesh = mesh
        self._keep = []
        md = mesh.desc()
        bc = N.BcDesc(bcs.u_in, bcs.k_in, bcs.omega_in)
        st = settings.native()
        od = N.ObsDesc()
        od.n_obs = obs.n_obs()
        if od.n_obs:
            arrs = obs.arrays()
            self._keep += arrs
            od.component = obs._probes[0].component
            od.x, od.y, od.observed, od.sigma_obs, od.sigma_model = (N.dptr(a) for a in arrs)
        u = u_init if isinstance(u_init, Vec3) else Vec3(*u_init)
        init = np.array([u.x, u.y, u.z, p_init, k_init, omega_init], dtype=np.float64)
        active = np.array(params.active_indices, dtype=np.int32)
        base = np.array(params.base, dtype=np.float64)
        h = C.c_void_p()
        N.call("rq_problem_create", C.byref(md), C.byref(bc), C.c_double(nu), C.byref(st),
               C.byref(od), N.dptr(init), N.iptr(active), C.c_int32(len(active)), N.dptr(base),
               C.byref(h))
        self.handle = h
        self.n_cells = mesh.n_cells()
        self.nx = mesh.nx

    def workspace_bytes(self) -> int:
        b = C.c_uint64()
        N.call("rq_problem_workspace_bytes", self.handle, C.byref(b))
        return b.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                N.lib().rq_problem_destroy(h)
            except Exception:
                pass
            self.handle = None


def _rows_from_native(out, pred, n_obs, params_n) -> list:
    rows = []
    for i, o in enumerate(out):
        status = EvaluationStatus(o.status)
        err = ""
        if status == EvaluationStatus.InvalidParameters:
            err = "coefficient row is nonfinite or out of bounds"
        p = np.array(pred[i], dtype=np.float64) if n_obs else np.zeros(0)
        rows.append(ForwardBatchRow(EvaluationResult(status, o.loglik, p, o.iterations),
                                    o.final_worst, o.contraction_rate, bool(o.stalled), err))
    return rows


class ForwardBatch:
    """ForwardBatch (rans-uq/include/ForwardBatch.hpp:23-125) on the GPU: every row is a
    cold solve by one persistent CTA; rows are independent of batch order and size."""

    def __init__(self, mesh, param_set, obs_op, bcs, nu, settings=None, u_init=Vec3(1, 0, 0),
                 p_init=0.0, k_init=1e-4, omega_init=1.0):
        settings = settings or SolverSettings()
        self._problem = _Problem(mesh, param_set, obs_op, bcs, nu, settings, u_init, p_init,
                                 k_init, omega_init)
        self.param_set, self.obs_op = param_set, obs_op

    def n_parameters(self) -> int:
        return self.param_set.n_active()

    def n_observations(self) -> int:
        return self.obs_op.n_obs()

    def tune(self, theta=None, iters: int = 200, candidates=None):
        """Times one solve capped at `iters` outer iterations per candidate launch shape
        ((block_threads, arena_kb) pairs; None = the library's set), applies the fastest
        to this mesh class (rq_problem_tune) and returns (chosen, [(block_threads,
        arena_kb, us_per_iteration), ...]). theta defaults to the centre of the bounds."""
        if theta is None:
            theta = 0.5 * (np.asarray(self.param_set.lower_bounds()) +
                           np.asarray(self.param_set.upper_bounds()))
        theta = np.ascontiguousarray(np.asarray(theta, dtype=np.float64).ravel())
        if theta.size != self.n_parameters():
            raise ValueError("theta must have n_parameters values")
        if candidates is None:
            cand, nc = None, 0
            meas = (N.LaunchShape * 9)()
        else:
            nc = len(candidates)
            cand = (N.LaunchShape * nc)(*[N.LaunchShape(int(b), int(a), 0.0)
                                          for b, a in candidates])
            meas = (N.LaunchShape * nc)()
        chosen = N.LaunchShape()
        N.call("rq_problem_tune", self._problem.handle, N.dptr(theta), C.c_int32(iters), cand,
               C.c_int32(nc), meas, C.byref(chosen))
        return ((chosen.block_threads, chosen.arena_kb),
                [(m.block_threads, m.arena_kb, m.us_per_iteration) for m in meas])

    def set_launch(self, block_threads: int, arena_kb: int = -1) -> None:
        """Applies a launch shape (rq_problem_set_launch): CTA size and shared-memory
        arena in KiB (-1 = the default rule, 0 = none)."""
        shape = N.LaunchShape(int(block_threads), int(arena_kb), 0.0)
        N.call("rq_problem_set_launch", self._problem.handle, C.byref(shape))

    def launch(self):
        """The mesh class's current launch shape: (block_threads, arena_kb)."""
        shape = N.LaunchShape()
        N.call("rq_problem_get_launch", self._problem.handle, C.byref(shape))
        return shape.block_threads, shape.arena_kb

    def evaluate(self, theta, workers: int = 1) -> ForwardBatchResult:
        if int(workers) < 1:
            raise ValueError("workers must be positive")
        theta = np.ascontiguousarray(np.asarray(theta, dtype=np.float64))
        if theta.ndim != 2 or theta.shape[1] != self.n_parameters():
            raise ValueError("theta must have shape (n_rows, n_parameters)")
        n, no = theta.shape[0], self.n_observations()
        out = (N.RowOut * max(n, 1))()
        pred = np.full((max(n, 1), max(no, 1)), np.nan)
        if n:
            N.call("rq_evaluate_batch", self._problem.handle, N.dptr(theta), C.c_int64(n), out,
                   N.dptr(pred), None, None, C.c_int32(0))
        return ForwardBatchResult(_rows_from_native(list(out)[:n], pred[:, :no], no,
                                                    self.n_parameters()), no)

    def evaluate_fields(self, theta, hist_cap: int = 0):
        """Rows plus the final fields (n, 11, n_cells) and residual histories."""
        theta = np.ascontiguousarray(np.asarray(theta, dtype=np.float64))
        n, no, nc = theta.shape[0], self.n_observations(), self._problem.n_cells
        out = (N.RowOut * max(n, 1))()
        pred = np.full((max(n, 1), max(no, 1)), np.nan)
        fields = np.zeros((max(n, 1), 11, nc))
        hist = np.zeros((max(n, 1), max(hist_cap, 1), 11))
        N.call("rq_evaluate_batch", self._problem.handle, N.dptr(theta), C.c_int64(n), out,
               N.dptr(pred), N.dptr(fields), N.dptr(hist) if hist_cap else None,
               C.c_int32(hist_cap))
        res = ForwardBatchResult(_rows_from_native(list(out)[:n], pred[:, :no], no,
                                                   self.n_parameters()), no)
        return res, fields[:n], hist[:n, :hist_cap]


def evaluate_multi(batches, problem_of_row, theta) -> ForwardBatchResult:
    """Rows of several ForwardBatch mesh classes in ONE persistent launch
    (rq_evaluate_multi): row i is evaluated by batches[problem_of_row[i]]."""
    nb = len(batches)
    handles = (C.c_void_p * nb)(*[b._problem.handle.value for b in batches])
    pr = np.ascontiguousarray(np.asarray(problem_of_row, dtype=np.int32))
    theta = np.ascontiguousarray(np.asarray(theta, dtype=np.float64))
    n = theta.shape[0]
    stride_t = theta.shape[1]
    no = max(b.n_observations() for b in batches)
    out = (N.RowOut * max(n, 1))()
    pred = np.full((max(n, 1), max(no, 1)), np.nan)
    N.call("rq_evaluate_multi", handles, C.c_int32(nb), N.iptr(pr), N.dptr(theta),
           C.c_int32(stride_t), C.c_int64(n), out, N.dptr(pred), C.c_int32(max(no, 1)))
    rows = []
    for i, o in enumerate(list(out)[:n]):
        b = batches[pr[i]]
        k = b.n_observations()
        rows.extend(_rows_from_native([o], pred[i:i + 1, :k], k, b.n_parameters()))
    return ForwardBatchResult(rows, no)


def evaluate_multi_device(batches, problem_of_row, theta_dev, rows_dev, pred_dev, stream=0,
                          clock_dev=None) -> None:
    """Device-resident form of evaluate_multi (rq_evaluate_multi_device): theta_dev
    (n x max n_active doubles), rows_dev (n x 40-byte rq_row_out), pred_dev
    (n x max n_obs doubles) and clock_dev (n x 12 int64, optional) are device
    pointers (ints); the launch is queued on `stream` and not waited for."""
    nb = len(batches)
    handles = (C.c_void_p * nb)(*[b._problem.handle.value for b in batches])
    pr = np.ascontiguousarray(np.asarray(problem_of_row, dtype=np.int32))
    n = len(pr)
    stride_t = max(b.n_parameters() for b in batches)
    no = max(max(b.n_observations() for b in batches), 1)
    N.call("rq_evaluate_multi_device", handles, C.c_int32(nb), N.iptr(pr), C.c_void_p(theta_dev),
           C.c_int32(stride_t), C.c_int64(n), C.c_void_p(rows_dev), C.c_void_p(pred_dev),
           C.c_int32(no), C.c_void_p(stream), C.c_void_p(clock_dev or 0))


def rows_from_device_bytes(raw: np.ndarray) -> list:
    """Decode n x rq_row_out records copied back from the device."""
    rec = np.frombuffer(raw.tobytes(), dtype=np.dtype([("status", "<i4"), ("iterations", "<i4"),
                                                       ("stalled", "<i4"), ("converged", "<i4"),
                                                       ("loglik", "<f8"), ("final_worst", "<f8"),
                                                       ("contraction_rate", "<f8")]))
    return rec


@dataclass
class ServedResult:
    """Outcome of one served request. `predictions` is None unless the solve
    converged: failed requests are flagged (status, loglik sentinel), not returned."""
    ticket: int
    status: EvaluationStatus
    log_lik: float
    iterations: int
    predictions: np.ndarray | None
    start_ns: int       # GPU global timer at the start / end of the solve
    end_ns: int

    @property
    def flagged(self) -> bool:
        return self.status != EvaluationStatus.Converged


class ForwardServer:
    """Continuous-batching serving loop over several ForwardBatch mesh classes
    (rq_server_*; no counterpart in the reference, which evaluates fixed batches).
    A persistent kernel claims requests in submission order as they arrive; each
    solve runs on its own slot and a slot is reused as soon as its solve retires,
    so requests submitted while others run overlap with them on the device. The
    result of a request does not depend on what else is in flight."""

    def __init__(self, batches, capacity: int = 4096, idle_timeout: float = 2.0,
                 max_slots: int = 0, pool_bytes: int = 0):
        self._batches = list(batches)  # the mesh classes must outlive the server
        nb = len(self._batches)
        handles = (C.c_void_p * nb)(*[b._problem.handle.value for b in self._batches])
        h = C.c_void_p()
        N.call("rq_server_create_pooled", handles, C.c_int32(nb), C.c_int32(capacity),
               C.c_double(idle_timeout), C.c_int32(max_slots), C.c_uint64(pool_bytes),
               C.byref(h))
        self.handle = h
        self._no = max(max(b.n_observations() for b in self._batches), 1)
        self._cls: list[int] = []

    def submit(self, cls: int, theta) -> int:
        th = np.ascontiguousarray(np.asarray(theta, dtype=np.float64).ravel())
        if th.size != self._batches[cls].n_parameters():
            raise ValueError("theta must have the class's n_parameters values")
        t = C.c_int64()
        N.call("rq_server_submit", self.handle, C.c_int32(cls), N.dptr(th), C.byref(t))
        self._cls.append(cls)
        return int(t.value)

    def poll(self, ticket: int) -> ServedResult | None:
        done = C.c_int32()
        row = N.RowOut()
        pred = np.full(self._no, np.nan)
        clk = (C.c_int64 * 12)()
        N.call("rq_server_poll", self.handle, C.c_int64(ticket), C.byref(done), C.byref(row),
               N.dptr(pred), clk)
        if not done.value:
            return None
        status = EvaluationStatus(row.status)
        k = self._batches[self._cls[ticket]].n_observations()
        p = pred[:k].copy() if status == EvaluationStatus.Converged else None
        return ServedResult(ticket, status, row.loglik, row.iterations, p, clk[0], clk[1])

    def wait(self, timeout: float = 3600.0) -> int:
        n = C.c_int64()
        N.call("rq_server_wait", self.handle, C.c_double(timeout), C.byref(n))
        return int(n.value)

    def close(self) -> None:
        N.call("rq_server_close", self.handle)

    def info(self) -> dict:
        slots, lau = C.c_int32(), C.c_int32()
        sub, comp = C.c_int64(), C.c_int64()
        N.call("rq_server_info", self.handle, C.byref(slots), C.byref(sub), C.byref(comp),
               C.byref(lau))
        return {"slots": slots.value, "submitted": sub.value, "completed": comp.value,
                "launches": lau.value}

    def memory(self) -> dict:
        """The workspace pool (rq_server_memory): bytes, bytes held by admitted requests,
        requests waiting for admission, CTAs running now."""
        pool, used, waiting, running = C.c_uint64(), C.c_uint64(), C.c_int64(), C.c_int32()
        N.call("rq_server_memory", self.handle, C.byref(pool), C.byref(used),
               C.byref(waiting), C.byref(running))
        return {"pool_bytes": pool.value, "in_use_bytes": used.value, "waiting": waiting.value,
                "running_ctas": running.value}

    def workspace_bytes(self, cls: int) -> int:
        """Device workspace one solve of mesh class `cls` takes from the pool."""
        return int(self._batches[cls]._problem.workspace_bytes())

    def destroy(self) -> None:
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            N.lib().rq_server_destroy(h)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


@dataclass
class ForwardEvaluationResult:
    result: EvaluationResult
    final_worst_measure: float
    contraction_rate_u: float
    stalled: bool
    error: str
    fields: np.ndarray | None = None
    history: np.ndarray | None = None
    used_warm_start: bool = False
    snapshot: dict | None = None


_SNAPSHOT_SCALARS = ("p", "k", "omega", "nuT", "F1", "F2", "Pk", "CDkw")


def _snapshot(cells, bnd, flux, established) -> dict:
    """The reference binding's snapshot dict (ownedSnapshot, rans-uq/python/bindings.cpp:427-447):
    cell interiors, boundary-face values, face fluxes and the turbulence marker. Blocks of
    cells / bnd are Ux Uy Uz p k omega nuT F1 F2 Pk CDkw."""
    data = {"U": np.ascontiguousarray(cells[0:3].T)}
    boundary = {"U": np.ascontiguousarray(bnd[0:3].T)}
    for i, name in enumerate(_SNAPSHOT_SCALARS):
        data[name] = cells[3 + i].copy()
        boundary[name] = bnd[3 + i].copy()
    data["boundary"] = boundary
    data["face_fluxes"] = flux
    data["turb_established"] = established
    return data


class WarmStartCache:
    """WarmStartCache (rans-uq/include/ForwardModel.hpp:21-157) of one ForwardModel:
    converged states kept in device memory, looked up by Euclidean distance in theta
    (strictly below the threshold) and evicted oldest-first by count and by the
    reference's payload byte count. Same methods as the reference binding
    (rans-uq/python/bindings.cpp:823-828)."""

    def __init__(self, problem, max_size: int = 50, threshold: float = 0.5,
                 byte_budget: int = 64 * 1024 * 1024):
        self._problem = problem  # keeps the mesh class alive while the cache exists
        self.handle = C.c_void_p()
        N.call("rq_warm_cache_create", problem.handle, C.c_int32(max_size),
               C.c_double(threshold), C.c_uint64(byte_budget), C.byref(self.handle))

    def _info(self):
        size, kept, budget = C.c_int32(), C.c_uint64(), C.c_uint64()
        N.call("rq_warm_cache_info", self.handle, C.byref(size), C.byref(kept), C.byref(budget))
        return size.value, kept.value, budget.value

    def size(self) -> int:
        return self._info()[0]

    def clear(self) -> None:
        N.call("rq_warm_cache_clear", self.handle)

    def set_byte_budget(self, byte_budget: int) -> None:
        N.call("rq_warm_cache_set_byte_budget", self.handle, C.c_uint64(byte_budget))

    def byte_budget(self) -> int:
        return self._info()[2]

    def retained_bytes(self) -> int:
        return self._info()[1]

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value:
            try:
                N.lib().rq_warm_cache_destroy(self.handle)
            except Exception:
                pass
            self.handle = C.c_void_p()


class ForwardModel:
    """ForwardModel (rans-uq/include/ForwardModel.hpp:199-281): one GPU solve per call,
    started from the nearest converged state of its warm-start cache (50 entries, distance
    0.5, 64 MiB, as ForwardModel.cpp:14 builds it) or cold when none is near; a Converged
    solve is stored (ForwardModel.cpp:79-82, 114-117). Batches start every row cold."""

    def __init__(self, mesh, param_set, obs_op, bcs, nu, settings=None, u_init=Vec3(1, 0, 0),
                 p_init=0.0, k_init=1e-4, omega_init=1.0):
        self._batch = ForwardBatch(mesh, param_set, obs_op, bcs, nu, settings, u_init, p_init,
                                   k_init, omega_init)
        self._cache = WarmStartCache(self._batch._problem)
        self._last = None
        self._retain = True

    def cache(self) -> WarmStartCache:
        return self._cache

    def evaluate(self, theta) -> EvaluationResult:
        return self.evaluate_with_diagnostics(theta).result

    def evaluate_with_diagnostics(self, theta, snapshot: bool = False,
                                  hist_cap: int = 0) -> ForwardEvaluationResult:
        theta = np.ascontiguousarray(np.asarray(theta, dtype=np.float64).reshape(-1))
        if theta.size != self._batch.n_parameters():
            raise ValueError("theta must have n_parameters values")
        if hist_cap:
            raise NotImplementedError("residual histories come from ForwardBatch.evaluate_fields")
        no, nc = self._batch.n_observations(), self._batch._problem.n_cells
        nx = self._batch._problem.nx
        nb, nf = 2 * nx, 2 * nc + nx
        out = N.RowOut()
        pred = np.full(max(no, 1), np.nan)
        fields = np.zeros((11, nc))
        bnd = np.zeros((11, nb)) if snapshot else None
        flux = np.zeros(nf) if snapshot else None
        est = C.c_int32(0)
        used = C.c_int32(0)
        N.call("rq_evaluate_cached", self._cache.handle, N.dptr(theta), C.byref(out),
               N.dptr(pred), N.dptr(fields), N.dptr(bnd), N.dptr(flux),
               C.byref(est) if snapshot else None, C.byref(used))
        row = _rows_from_native([out], pred[None, :no], no, self._batch.n_parameters())[0]
        keep = row.result.status in (EvaluationStatus.Converged, EvaluationStatus.Unconverged)
        self._last = fields if keep and self._retain else None
        snap = _snapshot(fields, bnd, flux, bool(est.value)) if snapshot and keep else None
        return ForwardEvaluationResult(row.result, row.final_worst_measure, row.contraction_rate_u,
                                       row.stalled, row.error, fields if keep else None, None,
                                       bool(used.value), snap)

    def penalized_log_likelihood(self, theta) -> float:
        r = self.evaluate(theta)
        return r.log_lik if r.status == EvaluationStatus.Converged else -1e30

    def set_retain_last_fields(self, retain: bool) -> None:
        """setRetainLastFields (ForwardModel.hpp:221-227): stop (or resume) keeping the
        last solve's fields; stopping drops the ones kept."""
        self._retain = bool(retain)
        if not self._retain:
            self._last = None

    def param_set(self):
        return self._batch.param_set

    def has_last_fields(self) -> bool:
        return self._last is not None

    def last_fields(self) -> dict:
        """The last solve's cell fields as the reference binding returns them
        (extractFields, rans-uq/python/bindings.cpp:272-287): U as (n_cells, 3) and the
        scalar fields p, k, omega, nuT, F1, F2, Pk, CDkw."""
        if self._last is None:
            raise RuntimeError("No fields available — call evaluate() first")
        f = self._last
        out = {"U": np.ascontiguousarray(f[0:3].T)}
        for i, name in enumerate(_SNAPSHOT_SCALARS):
            out[name] = f[3 + i].copy()
        return out

    def set_target_anisotropy(self, b_target):
        raise NotImplementedError("Reynolds-stress injection is outside the B200 forward-model path")

    def has_target_anisotropy(self) -> bool:
        return False

    def clear_target_anisotropy(self) -> None:
        """Nothing to clear: no target anisotropy is ever set on this path."""
