"""B200-native CLUE clustering: the reference's make_clusters path on hand-written sm_100a kernels.

The compute path is libclue_b200.so (include/clue_b200.h), reached through ``capi``.
There is no CPU fallback: using ``capi`` (or any name re-exported from it here) fails with
ImportError if the library is not built.  The library is loaded on first use, so that the
workload generators (``synthetic``), the byte model and the sharding helpers can be imported
by processes that never touch the GPU.
"""
import importlib

_FROM_CAPI = ("Context", "ExponentialKernel", "FlatKernel", "GaussianKernel", "Metric", "Params",
              "RunInfo", "Result")

__all__ = ["capi", *_FROM_CAPI]


def __getattr__(name):
    if name == "capi":
        return importlib.import_module(".capi", __name__)
    if name in _FROM_CAPI:
        return getattr(importlib.import_module(".capi", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
