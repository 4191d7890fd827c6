"""ctypes binding of librq_b200.so (the C ABI declared in include/rq_b200.h).

The library is built in place by ``make -C bayesian-rans-uq_b200``; there is no
CPU fallback: every entry point here raises if the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "librq_b200.so"

RQ_OK, RQ_E_INVALID, RQ_E_CUDA, RQ_E_OOM, RQ_E_UNSUPPORTED = 0, -1, -2, -3, -4
SOLVERS = {"AMG": 0, "PCG": 1, "BiCGSTAB": 2}
PRECISIONS = {"fp64": 0, "mixed": 1}
MESH_CHANNEL, MESH_CURVED = 0, 1
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int32)


class MeshDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("pad", C.c_int32),
                ("lx", C.c_double), ("h", C.c_double), ("re_tau", C.c_double),
                ("yplus", C.c_double), ("x_nodes", DP), ("y_bottom", DP), ("y_top", C.c_double),
                ("re", C.c_double)]


class BcDesc(C.Structure):
    _fields_ = [("u_in", C.c_double), ("k_in", C.c_double), ("omega_in", C.c_double)]


class Settings(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("inner_iterations", C.c_int32),
                ("convergence_window", C.c_int32), ("monitor_interval", C.c_int32),
                ("turb_start_iter", C.c_int32), ("turb_update_interval", C.c_int32),
                ("nut_floor_iters", C.c_int32), ("pressure_solver", C.c_int32),
                ("precision", C.c_int32), ("block_threads", C.c_int32),
                ("convergence_tol", C.c_double), ("inner_tolerance", C.c_double),
                ("divergence_limit", C.c_double), ("alpha_u", C.c_double),
                ("alpha_p", C.c_double), ("alpha_k", C.c_double), ("alpha_omega", C.c_double),
                ("body_force", C.c_double * 3), ("k_min", C.c_double), ("k_max", C.c_double),
                ("omega_min", C.c_double)]


class ObsDesc(C.Structure):
    _fields_ = [("n_obs", C.c_int32), ("component", C.c_int32), ("x", DP), ("y", DP),
                ("observed", DP), ("sigma_obs", DP), ("sigma_model", DP)]


class RowOut(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("stalled", C.c_int32),
                ("converged", C.c_int32), ("loglik", C.c_double), ("final_worst", C.c_double),
                ("contraction_rate", C.c_double)]


class SolverResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("final_res", C.c_double), ("initial_res", C.c_double)]


class LaunchShape(C.Structure):
    _fields_ = [("block_threads", C.c_int32), ("arena_kb", C.c_int32),
                ("us_per_iteration", C.c_double)]


class Ldu(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("diag", DP), ("upper", DP),
                ("lower", DP), ("source", DP), ("owner", IP), ("neighbour", IP)]


# every exported symbol of include/rq_b200.h with its argument types
SIGNATURES = {
    "rq_last_error": ([], C.c_char_p),
    "rq_version": ([], C.c_int),
    "rq_default_settings": ([C.POINTER(Settings)], C.c_int),
    "rq_problem_create": ([C.POINTER(MeshDesc), C.POINTER(BcDesc), C.c_double,
                           C.POINTER(Settings), C.POINTER(ObsDesc), DP, IP, C.c_int32, DP,
                           C.POINTER(C.c_void_p)], C.c_int),
    "rq_problem_destroy": ([C.c_void_p], C.c_int),
    "rq_problem_info": ([C.c_void_p, IP, IP, IP, IP], C.c_int),
    "rq_problem_workspace_bytes": ([C.c_void_p, C.POINTER(C.c_uint64)], C.c_int),
    "rq_problem_tune": ([C.c_void_p, DP, C.c_int32, C.POINTER(LaunchShape), C.c_int32,
                         C.POINTER(LaunchShape), C.POINTER(LaunchShape)], C.c_int),
    "rq_problem_set_launch": ([C.c_void_p, C.POINTER(LaunchShape)], C.c_int),
    "rq_problem_get_launch": ([C.c_void_p, C.POINTER(LaunchShape)], C.c_int),
    "rq_evaluate_batch": ([C.c_void_p, DP, C.c_int64, C.POINTER(RowOut), DP, DP, DP, C.c_int32],
                          C.c_int),
    "rq_evaluate_multi": ([C.POINTER(C.c_void_p), C.c_int32, IP, DP, C.c_int32, C.c_int64,
                           C.POINTER(RowOut), DP, C.c_int32], C.c_int),
    "rq_evaluate_multi_device": ([C.POINTER(C.c_void_p), C.c_int32, IP, C.c_void_p, C.c_int32,
                                  C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                  C.c_void_p], C.c_int),
    "rq_solve": ([C.c_void_p, DP, C.POINTER(RowOut), DP, DP, DP, C.c_int32], C.c_int),
    "rq_mesh_geometry": ([C.POINTER(MeshDesc), IP, DP], C.c_int),
    "rq_mesh_save_binary": ([C.POINTER(MeshDesc), C.c_char_p], C.c_int),
    "rq_linear_solve": ([C.POINTER(Ldu), DP, C.c_int32, C.c_double, C.c_int32,
                         C.POINTER(SolverResult)], C.c_int),
    "rq_linear_solve_batch": ([C.POINTER(Ldu), C.c_int32, C.POINTER(DP), C.c_int32, C.c_double,
                               C.c_int32, C.c_int32, C.POINTER(SolverResult)], C.c_int),
    "rq_linsys_create": ([C.POINTER(Ldu), C.c_int32, C.c_int32, C.c_int32,
                          C.POINTER(C.c_void_p)], C.c_int),
    "rq_linsys_solve": ([C.c_void_p, C.c_int32, C.c_double, C.POINTER(DP),
                         C.POINTER(SolverResult)], C.c_int),
    "rq_linsys_solve_device": ([C.c_void_p, C.c_int32, C.c_double, C.c_void_p], C.c_int),
    "rq_linsys_results": ([C.c_void_p, C.POINTER(SolverResult), C.POINTER(DP)], C.c_int),
    "rq_linsys_info": ([C.c_void_p, IP, C.POINTER(C.c_int64), C.POINTER(C.c_int64), IP],
                       C.c_int),
    "rq_linsys_destroy": ([C.c_void_p], C.c_int),
    "rq_evaluate_noalloc": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
                            C.c_int),
    "rq_posterior_weights": ([DP, DP, C.c_int64, DP, DP], C.c_int),
    "rq_posterior_weights_parts": ([DP, DP, C.c_int64, DP, DP, DP], C.c_int),
    "rq_posterior_weights_device": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                     C.c_void_p], C.c_int),
    "rq_server_create": ([C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_double, C.c_int32,
                          C.POINTER(C.c_void_p)], C.c_int),
    "rq_server_create_pooled": ([C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.c_double,
                                 C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)], C.c_int),
    "rq_server_memory": ([C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                          C.POINTER(C.c_int64), IP], C.c_int),
    "rq_server_submit": ([C.c_void_p, C.c_int32, DP, C.POINTER(C.c_int64)], C.c_int),
    "rq_server_poll": ([C.c_void_p, C.c_int64, IP, C.POINTER(RowOut), DP,
                        C.POINTER(C.c_int64)], C.c_int),
    "rq_server_wait": ([C.c_void_p, C.c_double, C.POINTER(C.c_int64)], C.c_int),
    "rq_server_close": ([C.c_void_p], C.c_int),
    "rq_server_info": ([C.c_void_p, IP, C.POINTER(C.c_int64), C.POINTER(C.c_int64), IP],
                       C.c_int),
    "rq_server_destroy": ([C.c_void_p], C.c_int),
    "rq_resample_indices": ([DP, C.c_int64, DP, C.c_int64, C.POINTER(C.c_int64)], C.c_int),
    "rq_predictive_moments": ([DP, C.c_int64, C.c_int32, DP, DP], C.c_int),
    "rq_conformal_quantile": ([DP, C.c_int64, C.c_double, DP], C.c_int),
    "rq_split_conformal": ([DP, DP, C.c_int64, DP, C.c_int64, C.c_double, DP, DP], C.c_int),
    "rq_warm_cache_create": ([C.c_void_p, C.c_int32, C.c_double, C.c_uint64,
                              C.POINTER(C.c_void_p)], C.c_int),
    "rq_warm_cache_destroy": ([C.c_void_p], C.c_int),
    "rq_warm_cache_info": ([C.c_void_p, IP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
                           C.c_int),
    "rq_warm_cache_clear": ([C.c_void_p], C.c_int),
    "rq_warm_cache_set_byte_budget": ([C.c_void_p, C.c_uint64], C.c_int),
    "rq_evaluate_cached": ([C.c_void_p, DP, C.POINTER(RowOut), DP, DP, DP, DP, IP, IP],
                           C.c_int),
}

_lib = None


class NativeError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[rq {code}] {message}")
        self.code = code


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` "
                              "(there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes, fn.restype = args, res
        _lib = L
    return _lib


def call(name: str, *args) -> None:
    rc = getattr(lib(), name)(*args)
    if rc != RQ_OK:
        msg = lib().rq_last_error().decode(errors="replace")
        if rc == RQ_E_INVALID:
            raise ValueError(msg)
        if rc == RQ_E_OOM:
            raise MemoryError(msg)
        if rc == RQ_E_UNSUPPORTED:
            raise NotImplementedError(msg)
        raise NativeError(rc, msg)


def dptr(a):
    return a.ctypes.data_as(DP) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(IP) if a is not None else None
