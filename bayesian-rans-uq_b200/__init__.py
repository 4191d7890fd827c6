"""B200-native forward model for Bayesian calibration of k-omega SST closure
coefficients: the SIMPLE + SST steady solve of the reference's ForwardModel /
ForwardBatch, run by hand-written sm_100a CUDA kernels behind a C ABI
(include/rq_b200.h). Import it as ``rans_uq_b200`` (the repository-root shim).
"""
from . import _native
from .core import (EvaluationResult, EvaluationStatus, FlowBoundaryConditions, ForwardBatch,
                   ForwardBatchResult, ForwardBatchRow, ForwardEvaluationResult, ForwardModel,
                   ForwardServer, InferenceParameterSet, Mesh, ObservationOperator,
                   SST_DEFAULTS, SST_NAMES, ServedResult, SolverSettings, Vec3, WarmStartCache,
                   evaluate_multi, evaluate_multi_device, rows_from_device_bytes)

__all__ = ["EvaluationResult", "EvaluationStatus", "FlowBoundaryConditions", "ForwardBatch",
           "ForwardBatchResult", "ForwardBatchRow", "ForwardEvaluationResult", "ForwardModel",
           "ForwardServer", "InferenceParameterSet", "ServedResult", "Mesh", "ObservationOperator", "SST_DEFAULTS", "SST_NAMES",
           "SolverSettings", "Vec3", "WarmStartCache", "evaluate_multi", "evaluate_multi_device",
           "rows_from_device_bytes", "lib"]


def lib():
    """The loaded CUDA library (raises if it is not built)."""
    return _native.lib()
