"""B200-native CLUE clustering: the reference's make_clusters path on hand-written sm_100a kernels.

The compute path is libclue_b200.so (include/clue_b200.h), reached through ``capi``.
There is no CPU fallback: importing the package fails if the library is not built.
"""
from . import capi  # noqa: F401  (loads libclue_b200.so; raises ImportError when missing)
from .capi import (Context, ExponentialKernel, FlatKernel, GaussianKernel, Metric, Params,  # noqa: F401
                   RunInfo, Result)

__all__ = ["capi", "Context", "FlatKernel", "ExponentialKernel", "GaussianKernel", "Metric", "Params",
           "RunInfo", "Result"]
