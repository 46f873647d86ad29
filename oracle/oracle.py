"""ctypes front-end of the CPU restatement in ``clue_oracle.c``.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference leg as the checker.  The product never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
MAX_DIM = 10


def _cpu_tag() -> str:
    """Short tag of this host's CPU: the library is built with -march=native, so each CPU
    model (and instruction-set flag list) gets its own build directory."""
    import hashlib
    import platform
    model, flags = platform.processor(), ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model in ("", platform.processor()):
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags"):
                    flags = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return hashlib.sha1((model + "|" + flags).encode()).hexdigest()[:12]


_BUILD_DIR = os.path.join(_HERE, "_build", _cpu_tag())
_LIB_PATH = os.path.join(_BUILD_DIR, "libclue_oracle.so")

KERNELS = {"flat": 0, "exp": 1, "gaus": 2}
METRICS = {"euclidean": 0, "weighted_euclidean": 1, "periodic_euclidean": 2,
           "manhattan": 3, "chebyshev": 4, "weighted_chebyshev": 5}
TIEBREAKS = {"reference": 0, "rho_index": 1}


class _Params(ctypes.Structure):
    _fields_ = [("dc", ctypes.c_float), ("rhoc", ctypes.c_float), ("dm", ctypes.c_float),
                ("seed_dc", ctypes.c_float), ("ppbin", ctypes.c_int32), ("ndim", ctypes.c_int32),
                ("wrapped", ctypes.c_uint8 * MAX_DIM), ("kernel_type", ctypes.c_int32),
                ("kernel_par", ctypes.c_float * 3), ("metric_type", ctypes.c_int32),
                ("metric_par", ctypes.c_float * MAX_DIM), ("seed_capacity", ctypes.c_int64),
                ("tiebreak", ctypes.c_int32), ("nthreads", ctypes.c_int32)]


class _Out(ctypes.Structure):
    _fields_ = [("cluster_index", ctypes.c_void_p), ("is_seed", ctypes.c_void_p),
                ("rho", ctypes.c_void_p), ("nearest_higher", ctypes.c_void_p),
                ("delta", ctypes.c_void_p),
                ("n_seeds", ctypes.c_int64), ("n_clusters", ctypes.c_int64),
                ("dropped_seeds", ctypes.c_int64), ("seed_capacity_used", ctypes.c_int64),
                ("max_dfs_stack", ctypes.c_int64), ("candidates_rho", ctypes.c_int64),
                ("candidates_nh", ctypes.c_int64), ("nh_distance_ties", ctypes.c_int64)]


class _Grid(ctypes.Structure):
    _fields_ = [("nperdim", ctypes.c_int32), ("ntiles", ctypes.c_int32),
                ("minmax", ctypes.c_float * (2 * MAX_DIM)), ("tilesize", ctypes.c_float * MAX_DIM)]


def build() -> str:
    """Compile the restatement with its Makefile (gcc -O2 -march=native, -ffp-contract=off) into
    this CPU's build directory."""
    subprocess.run(["make", "-s", "-C", _HERE, "OUT=" + os.path.relpath(_BUILD_DIR, _HERE)], check=True)
    return _LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        lib.oracle_run.argtypes = [ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.POINTER(_Out)]
        lib.oracle_run.restype = ctypes.c_int
        lib.oracle_tiles.argtypes = [ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p,
                                     ctypes.POINTER(_Grid), ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_tiles.restype = ctypes.c_int
        lib.oracle_rho_f64.argtypes = [ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
        lib.oracle_rho_f64.restype = ctypes.c_int
        lib.oracle_nearest_higher.argtypes = [ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_int64)]
        lib.oracle_nearest_higher.restype = ctypes.c_int
        lib.oracle_silhouette.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
        lib.oracle_silhouette.restype = ctypes.c_int
        lib.oracle_metric.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_metric.restype = ctypes.c_float
        lib.oracle_kernel.argtypes = [ctypes.POINTER(_Params), ctypes.c_float, ctypes.c_int32,
                                      ctypes.c_int32]
        lib.oracle_kernel.restype = ctypes.c_float
        lib.oracle_run_events.argtypes = [ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_Out), ctypes.c_void_p]
        lib.oracle_run_events.restype = ctypes.c_int
        lib.oracle_near_flags.argtypes = [ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_double)]
        lib.oracle_near_flags.restype = ctypes.c_int
        lib.oracle_events_aux.argtypes = [ctypes.c_int, ctypes.POINTER(_Params), ctypes.c_int32, ctypes.c_void_p,
                                          ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_double)]
        lib.oracle_events_aux.restype = ctypes.c_int
        _lib = lib
    return _lib


@dataclass
class Config:
    """CLUE parameters, named as in the reference's Clusterer constructor."""
    dc: float
    rhoc: float
    dm: float | None = None
    seed_dc: float | None = None
    ppbin: int = 128
    kernel: str = "flat"
    kernel_par: tuple = (0.5,)
    metric: str = "euclidean"
    metric_par: tuple = ()
    wrapped: tuple = ()
    seed_capacity: int = 0       # reference SeedArray policy by default; <0 keeps all seeds
    tiebreak: str = "reference"
    nthreads: int = 1

    def to_struct(self, ndim: int) -> _Params:
        p = _Params()
        p.dc = self.dc
        p.rhoc = self.rhoc
        p.dm = self.dc if self.dm is None else self.dm
        p.seed_dc = self.dc if self.seed_dc is None else self.seed_dc
        p.ppbin = self.ppbin
        p.ndim = ndim
        for d, w in enumerate(self.wrapped):
            p.wrapped[d] = int(w)
        p.kernel_type = KERNELS[self.kernel]
        for k, v in enumerate(self.kernel_par):
            p.kernel_par[k] = v
        p.metric_type = METRICS[self.metric]
        for k, v in enumerate(self.metric_par):
            p.metric_par[k] = v
        p.seed_capacity = self.seed_capacity
        p.tiebreak = TIEBREAKS[self.tiebreak]
        p.nthreads = self.nthreads
        return p


@dataclass
class Result:
    cluster_index: np.ndarray
    is_seed: np.ndarray
    rho: np.ndarray
    nearest_higher: np.ndarray
    delta: np.ndarray
    stats: dict = field(default_factory=dict)


def _soa(coords: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(coords, dtype=np.float32)
    if c.ndim == 1:
        c = c[None, :]
    return c


def run(coords: np.ndarray, weight: np.ndarray, cfg: Config) -> Result:
    """Run the full restated pipeline. ``coords`` is SoA with shape (ndim, n)."""
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    w = np.ascontiguousarray(weight, dtype=np.float32)
    assert w.shape == (n,)
    res = Result(np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32),
                 np.empty(n, np.int32), np.empty(n, np.float32))
    out = _Out()
    out.cluster_index = res.cluster_index.ctypes.data
    out.is_seed = res.is_seed.ctypes.data
    out.rho = res.rho.ctypes.data
    out.nearest_higher = res.nearest_higher.ctypes.data
    out.delta = res.delta.ctypes.data
    p = cfg.to_struct(ndim)
    rc = lib.oracle_run(ctypes.byref(p), n, c.ctypes.data, w.ctypes.data, ctypes.byref(out))
    if rc != 0:
        raise ValueError(f"oracle_run failed ({rc})")
    res.stats = {k: getattr(out, k) for k in ("n_seeds", "n_clusters", "dropped_seeds",
                                               "seed_capacity_used", "max_dfs_stack",
                                               "candidates_rho", "candidates_nh",
                                               "nh_distance_ties")}
    return res


def nearest_higher(coords: np.ndarray, rho: np.ndarray, cfg: Config):
    """Nearest-higher stage alone on the given densities: (nearest_higher, delta, distance ties).

    Same grid, candidate order and tie-break as ``run`` (ClusteringKernels.hpp:109-212); used to
    check an implementation's nearest-higher search on its own densities."""
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    r = np.ascontiguousarray(rho, dtype=np.float32)
    assert r.shape == (n,)
    nh = np.empty(n, np.int32)
    delta = np.empty(n, np.float32)
    ties = ctypes.c_int64(0)
    p = cfg.to_struct(ndim)
    rc = lib.oracle_nearest_higher(ctypes.byref(p), n, c.ctypes.data, r.ctypes.data, nh.ctypes.data,
                                   delta.ctypes.data, ctypes.byref(ties))
    if rc != 0:
        raise ValueError(f"oracle_nearest_higher failed ({rc})")
    return nh, delta, int(ties.value)


def silhouette(coords: np.ndarray, labels: np.ndarray):
    """Silhouette score of labelled points: (per-point scores with NaN where not scored, mean).

    Restates include/CLUEstering/utils/detail/scores.hpp:17-99 with separately rounded FP32."""
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    per = np.empty(n, np.float32)
    mean = ctypes.c_float(0.0)
    rc = lib.oracle_silhouette(ndim, n, c.ctypes.data, lab.ctypes.data, per.ctypes.data, ctypes.byref(mean))
    if rc != 0:
        raise ValueError(f"oracle_silhouette failed ({rc})")
    return per, float(mean.value)


def tiles(coords: np.ndarray, cfg: Config):
    """Reference tile grid and tile CSR: (grid dict, offsets, indexes)."""
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    p = cfg.to_struct(ndim)
    g = _Grid()
    rc = lib.oracle_tiles(ctypes.byref(p), n, c.ctypes.data, ctypes.byref(g), None, None)
    if rc != 0:
        raise ValueError(f"oracle_tiles failed ({rc})")
    off = np.empty(g.ntiles + 1, np.int32)
    idx = np.empty(n, np.int32)
    lib.oracle_tiles(ctypes.byref(p), n, c.ctypes.data, ctypes.byref(g), off.ctypes.data,
                     idx.ctypes.data)
    grid = {"nperdim": g.nperdim, "ntiles": g.ntiles,
            "min": np.array([g.minmax[2 * d] for d in range(ndim)], np.float32),
            "max": np.array([g.minmax[2 * d + 1] for d in range(ndim)], np.float32),
            "tilesize": np.array([g.tilesize[d] for d in range(ndim)], np.float32)}
    return grid, off, idx


def rho_f64(coords: np.ndarray, weight: np.ndarray, cfg: Config, rel_tol: float = 1e-5,
            with_near: bool = False):
    """FP64 densities; with_near also returns the near-dc flags (see clue_oracle.h)."""
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    w = np.ascontiguousarray(weight, dtype=np.float32)
    out = np.empty(n, np.float64)
    near = np.zeros(n, np.uint8)
    p = cfg.to_struct(ndim)
    rc = lib.oracle_rho_f64(ctypes.byref(p), n, c.ctypes.data, w.ctypes.data, out.ctypes.data,
                            near.ctypes.data, rel_tol)
    if rc != 0:
        raise ValueError(f"oracle_rho_f64 failed ({rc})")
    return (out, near.astype(bool)) if with_near else out


def metric(a, b, cfg: Config) -> float:
    lib = _load()
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    p = cfg.to_struct(a.shape[0])
    return lib.oracle_metric(ctypes.byref(p), a.ctypes.data, b.ctypes.data)


def kernel(dist: float, i: int, j: int, cfg: Config, ndim: int = 1) -> float:
    lib = _load()
    p = cfg.to_struct(ndim)
    return lib.oracle_kernel(ctypes.byref(p), dist, i, j)


def canonicalize(labels: np.ndarray, outlier: int = -1) -> np.ndarray:
    """Renumber clusters by first appearance (the reference's CLUEstering.py:65-78)."""
    labels = np.asarray(labels)
    out = labels.copy()
    mask = labels != outlier
    vals = labels[mask]
    if vals.size == 0:
        return out
    uniq, first = np.unique(vals, return_index=True)
    rank = np.empty(len(uniq), dtype=labels.dtype)
    rank[np.argsort(first)] = np.arange(len(uniq), dtype=labels.dtype)
    out[mask] = rank[np.searchsorted(uniq, vals)]
    return out


# ---- batches of independent events and near-threshold classification ----------------------

NEAR_RHOC, NEAR_FLIP, NEAR_TIE, NEAR_SEED_DC, NEAR_DM = 1, 2, 4, 8, 16


def _ptr(a):
    return None if a is None else a.ctypes.data


def run_events(coords: np.ndarray, weight: np.ndarray, offsets: np.ndarray, cfg: Config) -> Result:
    """Every event of a batch clustered alone (as ``run``), one event per OpenMP thread
    (``cfg.nthreads`` threads).  Nearest highers are batch-global; stats are summed and
    ``stats["ev_n_clusters"]`` holds each event's clusters."""
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    w = np.ascontiguousarray(weight, dtype=np.float32)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    E = len(off) - 1
    res = Result(np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32),
                 np.empty(n, np.int32), np.empty(n, np.float32))
    out = _Out()
    out.cluster_index = res.cluster_index.ctypes.data
    out.is_seed = res.is_seed.ctypes.data
    out.rho = res.rho.ctypes.data
    out.nearest_higher = res.nearest_higher.ctypes.data
    out.delta = res.delta.ctypes.data
    evc = np.zeros(E, np.int64)
    p = cfg.to_struct(ndim)
    rc = lib.oracle_run_events(ctypes.byref(p), E, off.ctypes.data, n, c.ctypes.data, w.ctypes.data,
                               ctypes.byref(out), evc.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle_run_events failed ({rc})")
    res.stats = {k: getattr(out, k) for k in ("n_seeds", "n_clusters", "dropped_seeds", "max_dfs_stack",
                                               "candidates_rho", "candidates_nh", "nh_distance_ties")}
    res.stats["ev_n_clusters"] = evc
    return res


def _events_aux(kind, coords, offsets, cfg, weight=None, rho_a=None, rho_b=None, delta_a=None, tol=1e-5,
                want_rho64=False, want_flags=False, want_nh=False):
    lib = _load()
    c = _soa(coords)
    ndim, n = c.shape
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    conv = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    w, ra, rb, da = conv(weight), conv(rho_a), conv(rho_b), conv(delta_a)
    rho64 = np.empty(n, np.float64) if want_rho64 else None
    flags = np.zeros(n, np.uint8) if want_flags else None
    nh = np.empty(n, np.int32) if want_nh else None
    delta = np.empty(n, np.float32) if want_nh else None
    worst = ctypes.c_double(0.0)
    p = cfg.to_struct(ndim)
    rc = lib.oracle_events_aux(kind, ctypes.byref(p), len(off) - 1, off.ctypes.data, n, c.ctypes.data, _ptr(w),
                               _ptr(ra), _ptr(rb), _ptr(da), tol, _ptr(rho64), _ptr(flags), _ptr(nh), _ptr(delta),
                               ctypes.byref(worst))
    if rc != 0:
        raise ValueError(f"oracle_events_aux({kind}) failed ({rc})")
    return rho64, flags, nh, delta, float(worst.value)


def rho_f64_events(coords, weight, offsets, cfg: Config, rel_tol: float = 1e-5):
    """FP64 densities of every event alone, with the near-dc flags: (rho64, near_dc)."""
    rho64, near, _, _, _ = _events_aux(0, coords, offsets, cfg, weight=weight, tol=rel_tol, want_rho64=True,
                                       want_flags=True)
    return rho64, near.astype(bool)


def nearest_higher_events(coords, rho, offsets, cfg: Config):
    """Nearest-higher stage of every event alone on the given densities: (nearest_higher
    batch-global, delta)."""
    _, _, nh, delta, _ = _events_aux(1, coords, offsets, cfg, rho_a=rho, want_nh=True)
    return nh, delta


def near_flags(coords, rho_a, rho_b, delta_a, cfg: Config, tol: float = 1e-5, offsets=None):
    """Near-threshold decision points of two density vectors (NEAR_* bits per point) and the
    largest relative density gap over the pairs whose higher-relation flipped."""
    if offsets is None:
        offsets = np.array([0, _soa(coords).shape[1]], np.int32)
    _, flags, _, _, worst = _events_aux(2, coords, offsets, cfg, rho_a=rho_a, rho_b=rho_b, delta_a=delta_a,
                                        tol=tol, want_flags=True)
    return flags, worst
