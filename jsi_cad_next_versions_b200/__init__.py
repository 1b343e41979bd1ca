"""B200-native NURBS minimum-distance and surface-surface-intersection query
path (the query path of JSI_CAD_NEXT VERSION5), behind a C ABI.

The compute lives in ``libjsi_b200.so`` (sm_100a CUDA kernels + C++ host
orchestration, include/jsi_b200.h); this package is its Python host mirror.
"""
from .api import (  # noqa: F401
    Context,
    curvature_bounds,
    DistanceBatch,
    DistanceResult,
    EvalAndConstructTask,
    IntersectionResult,
    JsiError,
    ONE_UV_SIZE,
    default_global_dist_nuv,
    default_global_intersect_nuv,
    deinit_cad,
    evalWithCuda,
    init_cad,
    intersection,
    minimum_distance,
    SurfaceBatch,
    TaskBatch,
)
from . import synth  # noqa: F401

__all__ = [
    "Context", "DistanceBatch", "DistanceResult", "SurfaceBatch", "TaskBatch", "EvalAndConstructTask", "IntersectionResult", "JsiError", "ONE_UV_SIZE",
    "curvature_bounds", "default_global_dist_nuv", "default_global_intersect_nuv", "deinit_cad", "evalWithCuda", "init_cad",
    "intersection", "minimum_distance", "synth",
]
