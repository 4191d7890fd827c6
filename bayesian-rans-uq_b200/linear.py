"""Standalone linear solves on the GPU (rq_linear_solve*, rq_linsys_*): the
reference's LDU LinearSystem (core/include/LinearSolver.hpp:20-116), its solver
factory (makeSolver, :988-998) and SolverResult (:137-143), plus a batch of
systems kept on the device between solves. There is no CPU path: every solve
runs the CUDA library, which raises if it is missing.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

KINDS = {"AMG": 0, "PCG": 1, "BiCGSTAB": 2, "GaussSeidel": 3}


@dataclass
class LinearSystem:
    """LDU system: diag (n), upper/lower per internal face (own -> nbr entry and its
    transpose), source (n), own/nbr (face connectivity)."""
    n_cells: int
    n_if: int
    diag: np.ndarray
    upper: np.ndarray
    lower: np.ndarray
    source: np.ndarray
    own: np.ndarray
    nbr: np.ndarray
    _keep: list = field(default_factory=list, repr=False)

    @staticmethod
    def from_arrays(diag, upper, lower, source, own, nbr) -> "LinearSystem":
        d = np.ascontiguousarray(diag, dtype=np.float64)
        return LinearSystem(len(d), len(own), d, np.ascontiguousarray(upper, dtype=np.float64),
                            np.ascontiguousarray(lower, dtype=np.float64),
                            np.ascontiguousarray(source, dtype=np.float64),
                            np.ascontiguousarray(own, dtype=np.int32),
                            np.ascontiguousarray(nbr, dtype=np.int32))

    def native(self) -> N.Ldu:
        for name in ("diag", "upper", "lower", "source"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.float64))
        self.own = np.ascontiguousarray(self.own, dtype=np.int32)
        self.nbr = np.ascontiguousarray(self.nbr, dtype=np.int32)
        return N.Ldu(int(self.n_cells), int(self.n_if), N.dptr(self.diag), N.dptr(self.upper),
                     N.dptr(self.lower), N.dptr(self.source), N.iptr(self.own), N.iptr(self.nbr))


@dataclass
class SolverResult:
    iterations: int
    final_res: float
    initial_res: float
    converged: bool


def _result(r: N.SolverResult) -> SolverResult:
    return SolverResult(int(r.iterations), float(r.final_res), float(r.initial_res),
                        bool(r.converged))


def _kind(name: str) -> int:
    if name not in KINDS:
        raise ValueError(f"unknown linear solver: '{name}'")
    return KINDS[name]


class LinearSolver:
    """ILinearSolver: solve(A, x, max_iter, tol) updates x in place (FP64, one system)."""

    def __init__(self, name: str):
        self.kind = _kind(name)
        self._name = name

    def name(self) -> str:
        return self._name

    def solve(self, A: LinearSystem, x: np.ndarray, max_iter: int = 500,
              tol: float = 1e-6) -> SolverResult:
        if x.dtype != np.float64 or not x.flags.c_contiguous or x.shape != (A.n_cells,):
            raise ValueError("x must be a contiguous float64 array of n_cells values")
        res = N.SolverResult()
        ldu = A.native()
        N.call("rq_linear_solve", C.byref(ldu), N.dptr(x), C.c_int32(max_iter), C.c_double(tol),
               C.c_int32(self.kind), C.byref(res))
        return _result(res)


def make_solver(name: str) -> LinearSolver:
    return LinearSolver(name)


def _ldu_array(systems):
    arr = (N.Ldu * len(systems))()
    for i, s in enumerate(systems):
        arr[i] = s.native()
    return arr


def _x_pointers(xs):
    ptrs = (N.DP * len(xs))()
    for i, x in enumerate(xs):
        if x.dtype != np.float64 or not x.flags.c_contiguous:
            raise ValueError("every x must be a contiguous float64 array")
        ptrs[i] = N.dptr(x)
    return ptrs


def solve_batch(systems, xs=None, kind: str = "AMG", precision: str = "fp64",
                max_iter: int = 500, tol: float = 1e-6):
    """All systems in one persistent launch; xs (initial guesses, default zero) are
    updated in place and returned with the per-system results."""
    xs = [np.zeros(s.n_cells) for s in systems] if xs is None else xs
    out = (N.SolverResult * len(systems))()
    N.call("rq_linear_solve_batch", _ldu_array(systems), C.c_int32(len(systems)),
           _x_pointers(xs), C.c_int32(max_iter), C.c_double(tol), C.c_int32(_kind(kind)),
           C.c_int32(N.PRECISIONS[precision]), out)
    return [_result(r) for r in out], xs


class LinearBatch:
    """Systems whose operators and AMG hierarchies stay on the device between solves."""

    def __init__(self, systems, kind: str = "AMG", precision: str = "fp64"):
        self.systems = list(systems)
        h = C.c_void_p()
        N.call("rq_linsys_create", _ldu_array(self.systems), C.c_int32(len(self.systems)),
               C.c_int32(_kind(kind)), C.c_int32(N.PRECISIONS[precision]), C.byref(h))
        self.handle = h

    def solve(self, max_iter: int = 500, tol: float = 1e-6, xs=None):
        """From xs (or zero); returns (results, solutions)."""
        out = (N.SolverResult * len(self.systems))()
        sol = [np.zeros(s.n_cells) for s in self.systems] if xs is None else xs
        N.call("rq_linsys_solve", self.handle, C.c_int32(max_iter), C.c_double(tol),
               _x_pointers(sol) if xs is not None else None, out)
        if xs is None:
            N.call("rq_linsys_results", self.handle, None, _x_pointers(sol))
        return [_result(r) for r in out], sol

    def solve_device(self, max_iter: int, tol: float, stream: int = 0) -> None:
        """Queue a zero-start solve of every system on `stream`; does not wait."""
        N.call("rq_linsys_solve_device", self.handle, C.c_int32(max_iter), C.c_double(tol),
               C.c_void_p(stream))

    def results(self, with_x: bool = False):
        out = (N.SolverResult * len(self.systems))()
        sol = [np.zeros(s.n_cells) for s in self.systems] if with_x else None
        N.call("rq_linsys_results", self.handle, out, _x_pointers(sol) if with_x else None)
        return [_result(r) for r in out], sol

    def info(self) -> dict:
        ns, lv = C.c_int32(), C.c_int32()
        rows, nnz = C.c_int64(), C.c_int64()
        N.call("rq_linsys_info", self.handle, C.byref(ns), C.byref(rows), C.byref(nnz),
               C.byref(lv))
        return {"systems": ns.value, "rows": rows.value, "nnz": nnz.value, "max_levels": lv.value}

    def destroy(self) -> None:
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            N.lib().rq_linsys_destroy(h)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
