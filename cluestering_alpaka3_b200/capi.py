"""ctypes binding of the C ABI in include/clue_b200.h (libclue_b200.so, built in-tree).

The library is the product: there is no Python or CPU fallback.  Importing this module
raises if the shared library is missing; calls raise ``ClueError`` subclasses that mirror
the reference's host exceptions (std::invalid_argument -> ValueError,
std::out_of_range -> IndexError, std::runtime_error -> RuntimeError).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
# CLUE_B200_LIB names another build of the library to load, e.g. libclue_b200_checked.so (the
# build with device bounds checks); by default the in-tree libclue_b200.so.
LIB_PATH = os.environ.get("CLUE_B200_LIB") or os.path.join(_PKG, "libclue_b200.so")
MAX_DIM = 10

OK, ERR_INVALID_ARG, ERR_OOM, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_NOT_SUPPORTED, \
    ERR_NONFINITE, ERR_OUT_OF_RANGE = range(9)

KERNEL_FLAT, KERNEL_EXPONENTIAL, KERNEL_GAUSSIAN = 0, 1, 2
METRIC_EUCLIDEAN, METRIC_WEIGHTED_EUCLIDEAN, METRIC_PERIODIC_EUCLIDEAN, METRIC_MANHATTAN, \
    METRIC_CHEBYSHEV, METRIC_WEIGHTED_CHEBYSHEV = range(6)
TIE_REFERENCE, TIE_RHO_INDEX = 0, 1
MEM_DEVICE, MEM_HOST = 0, 1
FLAG_REFERENCE_ORDER, FLAG_SPATIAL_DENSITY, FLAG_NEAR_TIES = 1, 2, 4
NEAR_TOL = 1e-5

# Every symbol declared in include/clue_b200.h.
EXPORTED = [
    "clue_abi_version", "clue_last_error", "clue_status_string", "clue_check_params",
    "clue_check_kernel", "clue_check_metric", "clue_grid_shape", "clue_metric_eval",
    "clue_kernel_eval", "clue_device_count", "clue_device_alloc", "clue_device_free",
    "clue_host_alloc_pinned", "clue_host_free_pinned", "clue_memcpy_htod", "clue_memcpy_dtoh",
    "clue_memcpy_dtod", "clue_stream_create", "clue_stream_destroy", "clue_stream_synchronize",
    "clue_context_create", "clue_context_destroy", "clue_context_reserve",
    "clue_context_workspace_bytes", "clue_make_clusters", "clue_make_clusters_async",
    "clue_context_read_info", "clue_get_clusters", "clue_context_set_timing",
    "clue_context_stage_times", "clue_context_kernel_launches", "clue_make_clusters_noalloc",
    "clue_batch_make_clusters", "clue_batch_make_clusters_async", "clue_graph_capture_batch",
    "clue_graph_launch", "clue_graph_destroy", "clue_events_loop", "clue_context_reserve_batch",
    "clue_server_create", "clue_server_destroy", "clue_server_submit", "clue_server_wait",
    "clue_server_stats_read", "clue_server_replay", "clue_tuning_defaults", "clue_context_set_tuning",
    "clue_context_get_tuning", "clue_autotune_batch", "clue_silhouette", "clue_context_read_near_counts",
    "clue_cluster_centroids",
]


class ClueError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class ClueInvalidArgument(ClueError, ValueError):
    pass


class ClueOutOfRange(ClueError, IndexError):
    pass


class _Kernel(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("par", ctypes.c_float * 3)]


class _Metric(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("par", ctypes.c_float * MAX_DIM)]


class _Params(ctypes.Structure):
    _fields_ = [("dc", ctypes.c_float), ("rhoc", ctypes.c_float), ("dm", ctypes.c_float),
                ("seed_dc", ctypes.c_float), ("points_per_tile", ctypes.c_int32),
                ("wrapped", ctypes.c_uint8 * MAX_DIM), ("seed_capacity", ctypes.c_int64),
                ("tiebreak", ctypes.c_int32), ("flags", ctypes.c_int32)]


class _Outputs(ctypes.Structure):
    _fields_ = [("cluster_index", ctypes.c_void_p), ("is_seed", ctypes.c_void_p),
                ("rho", ctypes.c_void_p), ("nearest_higher", ctypes.c_void_p),
                ("delta", ctypes.c_void_p)]


class _RunInfo(ctypes.Structure):
    _fields_ = [("n_seeds", ctypes.c_int64), ("n_clusters", ctypes.c_int64),
                ("dropped_seeds", ctypes.c_int64), ("seed_capacity_used", ctypes.c_int64),
                ("n_tiles", ctypes.c_int64), ("n_per_dim", ctypes.c_int64),
                ("label_rounds", ctypes.c_int64)]


class _NearCounts(ctypes.Structure):
    _fields_ = [("rho_near_rhoc", ctypes.c_int64), ("delta_near_seed_dc", ctypes.c_int64),
                ("delta_near_dm", ctypes.c_int64), ("nh_near_ties", ctypes.c_int64)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("ndim", ctypes.c_int32), ("n_slots", ctypes.c_int32),
                ("max_batch_events", ctypes.c_int32), ("max_event_points", ctypes.c_int32),
                ("max_pending", ctypes.c_int32), ("device_budget_bytes", ctypes.c_int64)]


class _RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("n_clusters", ctypes.c_int32), ("batch_events", ctypes.c_int32),
                ("slot", ctypes.c_int32), ("submit_s", ctypes.c_double), ("start_s", ctypes.c_double),
                ("done_s", ctypes.c_double)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("rejected", ctypes.c_int64),
                ("failed", ctypes.c_int64), ("batches", ctypes.c_int64), ("batched_points", ctypes.c_int64),
                ("slot_points", ctypes.c_int64), ("slot_events", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("max_batch_seen", ctypes.c_int32), ("max_in_flight", ctypes.c_int32)]


class _Tuning(ctypes.Structure):
    _fields_ = [("symmetric_density", ctypes.c_int32), ("nh_split_lanes", ctypes.c_int32),
                ("overlap_chunk_points", ctypes.c_int64), ("density_gate", ctypes.c_int32),
                ("density_exp2", ctypes.c_int32), ("labels_bfs", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libclue_b200.so is not built ({LIB_PATH}); run `make -C {_PKG}`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, f32, sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_size_t
    sig = {
        "clue_abi_version": ([], i32),
        "clue_last_error": ([], ctypes.c_char_p),
        "clue_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "clue_check_params": ([ctypes.POINTER(_Params)], ctypes.c_int),
        "clue_check_kernel": ([ctypes.POINTER(_Kernel)], ctypes.c_int),
        "clue_check_metric": ([ctypes.POINTER(_Metric), i32], ctypes.c_int),
        "clue_grid_shape": ([i32, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)], ctypes.c_int),
        "clue_metric_eval": ([ctypes.POINTER(_Metric), i32, vp, vp], f32),
        "clue_kernel_eval": ([ctypes.POINTER(_Kernel), f32, i32, i32], f32),
        "clue_device_count": ([ctypes.POINTER(i32)], ctypes.c_int),
        "clue_device_alloc": ([i32, sz, ctypes.POINTER(vp)], ctypes.c_int),
        "clue_device_free": ([vp], ctypes.c_int),
        "clue_host_alloc_pinned": ([sz, ctypes.POINTER(vp)], ctypes.c_int),
        "clue_host_free_pinned": ([vp], ctypes.c_int),
        "clue_memcpy_htod": ([vp, vp, sz, vp], ctypes.c_int),
        "clue_memcpy_dtoh": ([vp, vp, sz, vp], ctypes.c_int),
        "clue_memcpy_dtod": ([vp, vp, sz, vp], ctypes.c_int),
        "clue_stream_create": ([i32, ctypes.POINTER(vp)], ctypes.c_int),
        "clue_stream_destroy": ([vp], ctypes.c_int),
        "clue_stream_synchronize": ([vp], ctypes.c_int),
        "clue_context_create": ([i32, ctypes.POINTER(vp)], ctypes.c_int),
        "clue_context_destroy": ([vp], ctypes.c_int),
        "clue_context_reserve": ([vp, i32, i32, i32], ctypes.c_int),
        "clue_context_workspace_bytes": ([vp], sz),
        "clue_make_clusters": ([vp, ctypes.POINTER(_Params), ctypes.POINTER(_Kernel),
                                ctypes.POINTER(_Metric), i32, i32, vp, vp, ctypes.POINTER(_Outputs),
                                i32, vp, ctypes.POINTER(_RunInfo)], ctypes.c_int),
        "clue_make_clusters_async": ([vp, ctypes.POINTER(_Params), ctypes.POINTER(_Kernel),
                                      ctypes.POINTER(_Metric), i32, i32, vp, vp,
                                      ctypes.POINTER(_Outputs), vp], ctypes.c_int),
        "clue_context_read_info": ([vp, vp, ctypes.POINTER(_RunInfo)], ctypes.c_int),
        "clue_context_read_near_counts": ([vp, vp, ctypes.POINTER(_NearCounts)], ctypes.c_int),
        "clue_context_set_timing": ([vp, i32], ctypes.c_int),
        "clue_context_stage_times": ([vp, ctypes.POINTER(f32), i32], ctypes.c_int),
        "clue_context_kernel_launches": ([vp], ctypes.c_uint64),
        "clue_make_clusters_noalloc": ([ctypes.POINTER(_Params), ctypes.POINTER(_Kernel),
                                        ctypes.POINTER(_Metric), i32, i32, vp, vp,
                                        ctypes.POINTER(_Outputs), vp, ctypes.POINTER(_RunInfo)],
                                       ctypes.c_int),
        "clue_get_clusters": ([vp, i32, vp, vp, vp, ctypes.POINTER(i32), ctypes.POINTER(i32), vp],
                              ctypes.c_int),
    }
    batch_args = [vp, ctypes.POINTER(_Params), ctypes.POINTER(_Kernel), ctypes.POINTER(_Metric), i32, i32, vp,
                  vp, vp, ctypes.POINTER(_Outputs), vp]
    sig["clue_batch_make_clusters"] = (batch_args + [i32, vp, ctypes.POINTER(_RunInfo)], ctypes.c_int)
    sig["clue_batch_make_clusters_async"] = (batch_args + [vp], ctypes.c_int)
    sig["clue_graph_capture_batch"] = (batch_args + [vp, ctypes.POINTER(vp)], ctypes.c_int)
    sig["clue_graph_launch"] = ([vp, vp], ctypes.c_int)
    sig["clue_events_loop"] = (batch_args[:-1] + [vp, vp], ctypes.c_int)
    sig["clue_graph_destroy"] = ([vp], ctypes.c_int)
    sig["clue_context_reserve_batch"] = ([vp, i32, i64, i64, i32], ctypes.c_int)
    sig["clue_server_create"] = ([ctypes.POINTER(_ServerConfig), ctypes.POINTER(_Params), ctypes.POINTER(_Kernel),
                                  ctypes.POINTER(_Metric), ctypes.POINTER(vp)], ctypes.c_int)
    sig["clue_server_destroy"] = ([vp], ctypes.c_int)
    sig["clue_server_submit"] = ([vp, i32, vp, i64, vp, ctypes.POINTER(_Outputs), ctypes.POINTER(i64)], ctypes.c_int)
    sig["clue_server_wait"] = ([vp, i64, i32, ctypes.POINTER(_RequestInfo)], ctypes.c_int)
    sig["clue_server_stats_read"] = ([vp, ctypes.POINTER(_ServerStats)], ctypes.c_int)
    sig["clue_server_replay"] = ([vp, i32, vp, vp, vp, vp, vp, ctypes.POINTER(_Outputs), vp, ctypes.POINTER(i32)],
                                 ctypes.c_int)
    sig["clue_silhouette"] = ([vp, i32, i32, vp, vp, vp, ctypes.POINTER(f32), vp], ctypes.c_int)
    sig["clue_cluster_centroids"] = ([vp, i32, i32, vp, vp, i32, vp, vp, ctypes.POINTER(i32), vp], ctypes.c_int)
    sig["clue_tuning_defaults"] = ([ctypes.POINTER(_Tuning)], None)
    sig["clue_context_set_tuning"] = ([vp, ctypes.POINTER(_Tuning)], ctypes.c_int)
    sig["clue_context_get_tuning"] = ([vp, ctypes.POINTER(_Tuning)], ctypes.c_int)
    sig["clue_autotune_batch"] = (batch_args[:-2] + [vp, ctypes.c_char_p, ctypes.POINTER(_Tuning)], ctypes.c_int)
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    return lib


lib = _load()


def last_error() -> str:
    msg = lib.clue_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    if status == OK:
        return
    msg = last_error()
    if status == ERR_INVALID_ARG or status == ERR_NONFINITE:
        raise ClueInvalidArgument(status, msg)
    if status == ERR_OUT_OF_RANGE:
        raise ClueOutOfRange(status, msg)
    raise ClueError(status, msg)


@dataclass
class Kernel:
    """A convolutional kernel plugin: FlatKernel / ExponentialKernel / GaussianKernel."""
    type: int
    par: tuple

    def struct(self) -> _Kernel:
        k = _Kernel()
        k.type = self.type
        for i, v in enumerate(self.par):
            k.par[i] = v
        check(lib.clue_check_kernel(ctypes.byref(k)))
        return k


def FlatKernel(flat: float) -> Kernel:
    return Kernel(KERNEL_FLAT, (flat,))


def ExponentialKernel(avg: float, amplitude: float) -> Kernel:
    return Kernel(KERNEL_EXPONENTIAL, (avg, amplitude))


def GaussianKernel(avg: float, std: float, amplitude: float) -> Kernel:
    return Kernel(KERNEL_GAUSSIAN, (avg, std, amplitude))


@dataclass
class Metric:
    type: int = METRIC_EUCLIDEAN
    par: tuple = ()

    def struct(self, ndim: int) -> _Metric:
        m = _Metric()
        m.type = self.type
        for i, v in enumerate(self.par):
            m.par[i] = v
        check(lib.clue_check_metric(ctypes.byref(m), ndim))
        return m


@dataclass
class Params:
    dc: float
    rhoc: float
    dm: float | None = None
    seed_dc: float | None = None
    points_per_tile: int = 128
    wrapped: tuple = ()
    seed_capacity: int = 0       # reference SeedArray policy; < 0 keeps every seed
    tiebreak: int = TIE_REFERENCE
    flags: int = 0               # FLAG_REFERENCE_ORDER / FLAG_SPATIAL_DENSITY / FLAG_NEAR_TIES

    def struct(self) -> _Params:
        p = _Params()
        p.dc = self.dc
        p.rhoc = self.rhoc
        p.dm = self.dc if self.dm is None else self.dm
        p.seed_dc = self.dc if self.seed_dc is None else self.seed_dc
        p.points_per_tile = self.points_per_tile
        for d, w in enumerate(self.wrapped):
            p.wrapped[d] = 1 if w else 0
        p.seed_capacity = self.seed_capacity
        p.tiebreak = self.tiebreak
        p.flags = self.flags
        check(lib.clue_check_params(ctypes.byref(p)))
        return p


@dataclass
class RunInfo:
    n_seeds: int = 0
    n_clusters: int = 0
    dropped_seeds: int = 0
    seed_capacity_used: int = 0
    n_tiles: int = 0
    n_per_dim: int = 0
    label_rounds: int = 0


@dataclass
class Result:
    cluster_index: object
    is_seed: object = None
    rho: object = None
    nearest_higher: object = None
    delta: object = None
    info: RunInfo = field(default_factory=RunInfo)


def grid_shape(n: int, points_per_tile: int, ndim: int) -> tuple[int, int]:
    npd, nt = ctypes.c_int32(), ctypes.c_int32()
    check(lib.clue_grid_shape(n, points_per_tile, ndim, ctypes.byref(npd), ctypes.byref(nt)))
    return npd.value, nt.value


def metric_eval(metric: Metric, a, b) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    m = metric.struct(a.shape[0])
    return lib.clue_metric_eval(ctypes.byref(m), a.shape[0], a.ctypes.data, b.ctypes.data)


def kernel_eval(kernel: Kernel, dist: float, i: int, j: int) -> float:
    return lib.clue_kernel_eval(ctypes.byref(kernel.struct()), dist, i, j)


def device_count() -> int:
    c = ctypes.c_int32()
    st = lib.clue_device_count(ctypes.byref(c))
    return c.value if st == OK else 0


class Context:
    """Reusable device workspace on one GPU (the Clusterer's tiles/seeds/followers)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(lib.clue_context_create(device, ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib.clue_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, ndim: int, n: int, points_per_tile: int = 128):
        check(lib.clue_context_reserve(self.handle, ndim, n, points_per_tile))

    @property
    def workspace_bytes(self) -> int:
        return lib.clue_context_workspace_bytes(self.handle)

    def make_clusters_host(self, coords: np.ndarray, weight: np.ndarray, params: Params,
                           kernel: Kernel | None = None, metric: Metric | None = None,
                           outputs: tuple = ("cluster_index", "is_seed", "rho", "nearest_higher",
                                             "delta"), stream: int = 0) -> Result:
        """Host (numpy) inputs and outputs; the library stages them through the device."""
        c = np.ascontiguousarray(coords, dtype=np.float32)
        if c.ndim == 1:
            c = c[None, :]
        ndim, n = c.shape
        w = np.ascontiguousarray(weight, dtype=np.float32)
        if w.shape != (n,):
            raise ValueError("weight must have one entry per point")
        res = Result(np.empty(n, np.int32))
        out = _Outputs()
        out.cluster_index = res.cluster_index.ctypes.data
        for name, dt in (("is_seed", np.int32), ("rho", np.float32), ("nearest_higher", np.int32),
                         ("delta", np.float32)):
            if name in outputs:
                arr = np.empty(n, dt)
                setattr(res, name, arr)
                setattr(out, name, arr.ctypes.data)
        info = _RunInfo()
        k = (kernel or FlatKernel(0.5)).struct()
        m = (metric or Metric()).struct(ndim)
        p = params.struct()
        check(lib.clue_make_clusters(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m),
                                     ndim, n, c.ctypes.data, w.ctypes.data, ctypes.byref(out),
                                     MEM_HOST, ctypes.c_void_p(stream), ctypes.byref(info)))
        res.info = RunInfo(**{f: getattr(info, f) for f, _ in _RunInfo._fields_})
        return res

    def make_clusters_device(self, coords_ptr: int, weight_ptr: int, ndim: int, n: int,
                             out_ptrs: dict, params: Params, kernel: Kernel | None = None,
                             metric: Metric | None = None, stream: int = 0,
                             blocking: bool = True) -> RunInfo | None:
        """Device pointers in and out (e.g. torch CUDA tensors' data_ptr())."""
        out = _Outputs()
        for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):
            setattr(out, name, out_ptrs.get(name) or None)
        k = (kernel or FlatKernel(0.5)).struct()
        m = (metric or Metric()).struct(ndim)
        p = params.struct()
        if blocking:
            info = _RunInfo()
            check(lib.clue_make_clusters(self.handle, ctypes.byref(p), ctypes.byref(k),
                                         ctypes.byref(m), ndim, n, ctypes.c_void_p(coords_ptr),
                                         ctypes.c_void_p(weight_ptr), ctypes.byref(out), MEM_DEVICE,
                                         ctypes.c_void_p(stream), ctypes.byref(info)))
            return RunInfo(**{f: getattr(info, f) for f, _ in _RunInfo._fields_})
        check(lib.clue_make_clusters_async(self.handle, ctypes.byref(p), ctypes.byref(k),
                                           ctypes.byref(m), ndim, n, ctypes.c_void_p(coords_ptr),
                                           ctypes.c_void_p(weight_ptr), ctypes.byref(out),
                                           ctypes.c_void_p(stream)))
        return None

    def set_tuning(self, symmetric_density: int | None = None, nh_split_lanes: int | None = None,
                   overlap_chunk_points: int | None = None, density_gate: int | None = None,
                   density_exp2: int | None = None, labels_bfs: int | None = None):
        """Set the runtime choices (clue_context_set_tuning); None keeps the current value."""
        t = _Tuning()
        check(lib.clue_context_get_tuning(self.handle, ctypes.byref(t)))
        if labels_bfs is not None:
            t.labels_bfs = labels_bfs
        if density_gate is not None:
            t.density_gate = density_gate
        if density_exp2 is not None:
            t.density_exp2 = density_exp2
        if symmetric_density is not None:
            t.symmetric_density = symmetric_density
        if nh_split_lanes is not None:
            t.nh_split_lanes = nh_split_lanes
        if overlap_chunk_points is not None:
            t.overlap_chunk_points = overlap_chunk_points
        check(lib.clue_context_set_tuning(self.handle, ctypes.byref(t)))

    def reset_tuning(self):
        check(lib.clue_context_set_tuning(self.handle, None))

    def tuning(self) -> dict:
        t = _Tuning()
        check(lib.clue_context_get_tuning(self.handle, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in _Tuning._fields_}

    def autotune_batch(self, coords_ptr: int, weight_ptr: int, ndim: int, event_offsets, params: Params,
                       kernel: Kernel | None = None, metric: Metric | None = None, stream: int = 0,
                       cache_path: str | None = None) -> dict:
        """Time the runtime choices on a device-resident batch and keep the fastest
        (clue_autotune_batch); with cache_path, reuse or extend an on-disk cache."""
        p, k, m, off = self._batch_structs(ndim, params, kernel, metric, event_offsets)
        t = _Tuning()
        check(lib.clue_autotune_batch(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m), ndim,
                                      len(off) - 1, off.ctypes.data, ctypes.c_void_p(coords_ptr),
                                      ctypes.c_void_p(weight_ptr), ctypes.c_void_p(stream),
                                      cache_path.encode() if cache_path else None, ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in _Tuning._fields_}

    def silhouette_device(self, coords_ptr: int, labels_ptr: int, ndim: int, n: int, per_point_ptr: int = 0,
                          stream: int = 0) -> float:
        """Silhouette score on the GPU (clue_silhouette) of device coordinates (SoA) and labels;
        per_point_ptr (device, n floats) optionally receives every point's score."""
        mean = ctypes.c_float(0.0)
        check(lib.clue_silhouette(self.handle, ndim, n, ctypes.c_void_p(coords_ptr), ctypes.c_void_p(labels_ptr),
                                  ctypes.c_void_p(per_point_ptr or None), ctypes.byref(mean),
                                  ctypes.c_void_p(stream)))
        return float(mean.value)

    def cluster_centroids_device(self, coords_ptr: int, labels_ptr: int, ndim: int, n: int, capacity: int,
                                 centroids_ptr: int, sizes_ptr: int = 0, stream: int = 0) -> int:
        """Cluster centroids on the GPU (clue_cluster_centroids) into a device buffer of
        capacity x ndim floats (and optionally the sizes); returns the number of clusters."""
        ncl = ctypes.c_int32(0)
        check(lib.clue_cluster_centroids(self.handle, ndim, n, ctypes.c_void_p(coords_ptr), ctypes.c_void_p(labels_ptr),
                                         capacity, ctypes.c_void_p(centroids_ptr), ctypes.c_void_p(sizes_ptr or None),
                                         ctypes.byref(ncl), ctypes.c_void_p(stream)))
        return int(ncl.value)

    def cluster_centroids(self, coords: np.ndarray, labels: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """Host arrays in, (centroids (n_clusters, ndim) float32, sizes) out, computed on the GPU."""
        c = np.ascontiguousarray(coords, dtype=np.float32)
        if c.ndim == 1:
            c = c[None, :]
        ndim, n = c.shape
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        cap = int(lab.max(initial=-1)) + 1
        bufs = []
        try:
            def dev(nbytes):
                p = ctypes.c_void_p()
                check(lib.clue_device_alloc(self.device, max(nbytes, 4), ctypes.byref(p)))
                bufs.append(p)
                return p
            dc, dl = dev(c.nbytes), dev(lab.nbytes)
            dcen, dsz = dev(cap * ndim * 4), dev(cap * 4)
            check(lib.clue_memcpy_htod(dc, c.ctypes.data, c.nbytes, None))
            check(lib.clue_memcpy_htod(dl, lab.ctypes.data, lab.nbytes, None))
            ncl = self.cluster_centroids_device(dc.value, dl.value, ndim, n, cap, dcen.value, dsz.value)
            cen = np.empty((ncl, ndim), np.float32)
            sz = np.empty(ncl, np.int32)
            if ncl:
                check(lib.clue_memcpy_dtoh(cen.ctypes.data, dcen, cen.nbytes, None))
                check(lib.clue_memcpy_dtoh(sz.ctypes.data, dsz, sz.nbytes, None))
            return cen, sz
        finally:
            for p in bufs:
                lib.clue_device_free(p)

    def set_timing(self, enable: bool = True):
        check(lib.clue_context_set_timing(self.handle, 1 if enable else 0))

    def stage_times(self) -> list[float]:
        """Milliseconds of (tile build, density, nearest higher, seeds+labels) of the last run."""
        arr = (ctypes.c_float * 4)()
        check(lib.clue_context_stage_times(self.handle, arr, 4))
        return list(arr)

    @property
    def kernel_launches(self) -> int:
        return lib.clue_context_kernel_launches(self.handle)

    def _batch_structs(self, ndim, params, kernel, metric, event_offsets):
        off = np.ascontiguousarray(event_offsets, dtype=np.int32)
        return (params.struct(), (kernel or FlatKernel(0.5)).struct(), (metric or Metric()).struct(ndim), off)

    def batch_host(self, coords: np.ndarray, weight: np.ndarray, event_offsets, params: Params,
                   kernel: Kernel | None = None, metric: Metric | None = None, stream: int = 0,
                   out: dict | None = None, ncl: np.ndarray | None = None):
        """Cluster concatenated events (host arrays); returns (Result, n_clusters per event).
        `out` may hold preallocated host arrays (e.g. pinned) for some of cluster_index, is_seed,
        rho, nearest_higher, delta: then only those are copied back (the others are None)."""
        c = np.ascontiguousarray(coords, dtype=np.float32)
        if c.ndim == 1:
            c = c[None, :]
        ndim, n = c.shape
        w = np.ascontiguousarray(weight, dtype=np.float32)
        p, k, m, off = self._batch_structs(ndim, params, kernel, metric, event_offsets)
        E = len(off) - 1
        names = ("cluster_index", "is_seed", "rho", "nearest_higher", "delta")
        if out is None:
            res = Result(np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32),
                         np.empty(n, np.int32), np.empty(n, np.float32))
        else:
            res = Result(*(out.get(name) for name in names))
        out = _Outputs()
        for name in names:
            a = getattr(res, name)
            setattr(out, name, a.ctypes.data if a is not None else None)
        if ncl is None:
            ncl = np.empty(E, np.int32)
        info = _RunInfo()
        check(lib.clue_batch_make_clusters(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m), ndim,
                                           E, off.ctypes.data, c.ctypes.data, w.ctypes.data, ctypes.byref(out),
                                           ncl.ctypes.data, MEM_HOST, ctypes.c_void_p(stream),
                                           ctypes.byref(info)))
        res.info = RunInfo(**{f: getattr(info, f) for f, _ in _RunInfo._fields_})
        return res, ncl

    def batch_device(self, coords_ptr: int, weight_ptr: int, ndim: int, event_offsets, out_ptrs: dict,
                     params: Params, kernel: Kernel | None = None, metric: Metric | None = None,
                     ncl_ptr: int = 0, stream: int = 0, blocking: bool = True):
        p, k, m, off = self._batch_structs(ndim, params, kernel, metric, event_offsets)
        E = len(off) - 1
        out = _Outputs()
        for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):
            setattr(out, name, out_ptrs.get(name) or None)
        if blocking:
            info = _RunInfo()
            check(lib.clue_batch_make_clusters(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m),
                                               ndim, E, off.ctypes.data, ctypes.c_void_p(coords_ptr),
                                               ctypes.c_void_p(weight_ptr), ctypes.byref(out),
                                               ctypes.c_void_p(ncl_ptr or None), MEM_DEVICE,
                                               ctypes.c_void_p(stream), ctypes.byref(info)))
            return RunInfo(**{f: getattr(info, f) for f, _ in _RunInfo._fields_})
        check(lib.clue_batch_make_clusters_async(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m),
                                                 ndim, E, off.ctypes.data, ctypes.c_void_p(coords_ptr),
                                                 ctypes.c_void_p(weight_ptr), ctypes.byref(out),
                                                 ctypes.c_void_p(ncl_ptr or None), ctypes.c_void_p(stream)))
        return None

    def capture_batch(self, coords_ptr: int, weight_ptr: int, ndim: int, event_offsets, out_ptrs: dict,
                      params: Params, kernel: Kernel | None = None, metric: Metric | None = None,
                      ncl_ptr: int = 0, stream: int = 0) -> "Graph":
        """Capture the batched pipeline into a CUDA graph (stream must not be the default stream)."""
        p, k, m, off = self._batch_structs(ndim, params, kernel, metric, event_offsets)
        E = len(off) - 1
        out = _Outputs()
        for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):
            setattr(out, name, out_ptrs.get(name) or None)
        h = ctypes.c_void_p()
        check(lib.clue_graph_capture_batch(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m), ndim,
                                           E, off.ctypes.data, ctypes.c_void_p(coords_ptr),
                                           ctypes.c_void_p(weight_ptr), ctypes.byref(out),
                                           ctypes.c_void_p(ncl_ptr or None), ctypes.c_void_p(stream),
                                           ctypes.byref(h)))
        return Graph(h)

    def events_loop(self, coords_ptr: int, weight_ptr: int, ndim: int, event_offsets, out_ptrs: dict,
                    params: Params, kernel: Kernel | None = None, metric: Metric | None = None,
                    stream: int = 0, event_times: bool = False):
        """The plain pipeline once per event (clue_events_loop); returns per-event ms if asked."""
        p, k, m, off = self._batch_structs(ndim, params, kernel, metric, event_offsets)
        E = len(off) - 1
        out = _Outputs()
        for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):
            setattr(out, name, out_ptrs.get(name) or None)
        ms = np.zeros(E, np.float32) if event_times else None
        check(lib.clue_events_loop(self.handle, ctypes.byref(p), ctypes.byref(k), ctypes.byref(m), ndim, E,
                                   off.ctypes.data, ctypes.c_void_p(coords_ptr), ctypes.c_void_p(weight_ptr),
                                   ctypes.byref(out), ctypes.c_void_p(stream),
                                   ms.ctypes.data if ms is not None else None))
        return ms

    def get_clusters(self, labels_ptr: int, n: int, offsets_ptr: int, points_ptr: int,
                     stream: int = 0) -> tuple[int, int]:
        """Cluster -> points CSR of n device labels (clue_get_clusters).  offsets_ptr must hold
        n + 1 int32 and points_ptr n int32 (device).  Returns (n_clusters, n_clustered)."""
        nc, ncl = ctypes.c_int32(0), ctypes.c_int32(0)
        check(lib.clue_get_clusters(self.handle, n, ctypes.c_void_p(labels_ptr), ctypes.c_void_p(offsets_ptr),
                                    ctypes.c_void_p(points_ptr), ctypes.byref(nc), ctypes.byref(ncl),
                                    ctypes.c_void_p(stream)))
        return nc.value, ncl.value

    def read_info(self, stream: int = 0) -> RunInfo:
        info = _RunInfo()
        check(lib.clue_context_read_info(self.handle, ctypes.c_void_p(stream), ctypes.byref(info)))
        return RunInfo(**{f: getattr(info, f) for f, _ in _RunInfo._fields_})

    def near_counts(self, stream: int = 0) -> dict:
        """Near-threshold decisions of the last run (relative tolerance NEAR_TOL): densities near
        rhoc, nearest-higher distances near seed_dc and dm, and (runs with FLAG_NEAR_TIES, else -1)
        points whose nearest-higher choice compares densities within the tolerance."""
        c = _NearCounts()
        check(lib.clue_context_read_near_counts(self.handle, ctypes.c_void_p(stream), ctypes.byref(c)))
        return {f: int(getattr(c, f)) for f, _ in _NearCounts._fields_}


class Graph:
    """An executable CUDA graph of the batched pipeline (clue_graph_capture_batch)."""

    def __init__(self, handle):
        self.handle = handle

    def launch(self, stream: int = 0):
        check(lib.clue_graph_launch(self.handle, ctypes.c_void_p(stream)))

    def close(self):
        if self.handle:
            lib.clue_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ServerConfig:
    ndim: int
    device: int = 0
    n_slots: int = 3
    max_batch_events: int = 1024
    max_event_points: int = 200000
    max_pending: int = 1 << 16
    device_budget_bytes: int = 8 << 30

    def struct(self) -> _ServerConfig:
        c = _ServerConfig()
        for f, _ in _ServerConfig._fields_:
            setattr(c, f, getattr(self, f))
        return c


@dataclass
class EventResult:
    cluster_index: np.ndarray
    is_seed: np.ndarray
    rho: np.ndarray
    nearest_higher: np.ndarray
    delta: np.ndarray
    info: dict


class Server:
    """Continuous-batching request loop on one GPU (clue_server_*): submit events from host
    memory, wait for their results; or replay a whole arrival trace natively."""

    def __init__(self, config: ServerConfig, params: Params, kernel: Kernel, metric: Metric | None = None):
        metric = metric or Metric()
        self.ndim = config.ndim
        h = ctypes.c_void_p()
        cfg = config.struct()
        check(lib.clue_server_create(ctypes.byref(cfg), ctypes.byref(params.struct()), ctypes.byref(kernel.struct()),
                                     ctypes.byref(metric.struct(config.ndim)), ctypes.byref(h)))
        self.handle = h
        self._live = {}  # ticket -> arrays the server reads / writes until the request is waited

    def submit(self, coords: np.ndarray, weight: np.ndarray) -> int:
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        weight = np.ascontiguousarray(weight, dtype=np.float32)
        n = weight.shape[0]
        res = EventResult(np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32),
                          np.empty(n, np.int32), np.empty(n, np.float32), {})
        out = _Outputs(res.cluster_index.ctypes.data, res.is_seed.ctypes.data, res.rho.ctypes.data,
                       res.nearest_higher.ctypes.data, res.delta.ctypes.data)
        t = ctypes.c_int64()
        check(lib.clue_server_submit(self.handle, n, coords.ctypes.data, coords.shape[1], weight.ctypes.data,
                                     ctypes.byref(out), ctypes.byref(t)))
        self._live[t.value] = (coords, weight, res)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> EventResult:
        info = _RequestInfo()
        st = lib.clue_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(info))
        if st == ERR_TIMEOUT:
            check(st)
        _, _, res = self._live.pop(ticket)
        check(st)
        res.info = {f: getattr(info, f) for f, _ in _RequestInfo._fields_}
        return res

    def stats(self) -> dict:
        s = _ServerStats()
        check(lib.clue_server_stats_read(self.handle, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _ServerStats._fields_}

    def replay(self, coords: np.ndarray, weight: np.ndarray, event_offsets, arrival_s, event_ids=None,
               outputs: bool = True):
        """Submits trace event e (pool event event_ids[e], or e) at arrival_s[e] seconds, open loop,
        from a native thread.  Returns (outputs dict of concatenated arrays or None,
        latency_s per event (-1 = refused), n_refused)."""
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        weight = np.ascontiguousarray(weight, dtype=np.float32)
        off = np.ascontiguousarray(event_offsets, dtype=np.int32)
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        ids = None if event_ids is None else np.ascontiguousarray(event_ids, dtype=np.int32)
        E = arr.shape[0]
        res, outp = None, None
        if outputs:
            if ids is not None:
                raise ValueError("outputs need one trace event per pool event (event_ids=None)")
            n = weight.shape[0]
            res = {"cluster_index": np.empty(n, np.int32), "is_seed": np.empty(n, np.int32),
                   "rho": np.empty(n, np.float32), "nearest_higher": np.empty(n, np.int32),
                   "delta": np.empty(n, np.float32)}
            outp = ctypes.byref(_Outputs(*(res[k].ctypes.data for k in
                                           ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"))))
        lat = np.empty(E, np.float64)
        rej = ctypes.c_int32()
        check(lib.clue_server_replay(self.handle, E, None if ids is None else ids.ctypes.data, off.ctypes.data,
                                     arr.ctypes.data, coords.ctypes.data, weight.ctypes.data, outp, lat.ctypes.data,
                                     ctypes.byref(rej)))
        return res, lat, rej.value

    def close(self):
        if getattr(self, "handle", None):
            lib.clue_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
