"""Python front end with the reference's `clusterer` interface (CLUEstering/CLUEstering.py:272-1260
in the reference), running on libclue_b200 through the backend module CLUE_GPU_B200.

The class keeps the reference's constructor, set_params, read_data (DataFrame, CSV path, dict,
list/array of coordinate rows plus a weight row), set_wrapped, choose_kernel, run_clue, fit,
fit_predict, the result properties (n_clusters, cluster_ids, labels, cluster_points,
points_per_cluster, output_df), cluster_centroid(s), to_csv and import_clusterer.  Backends:
"gpu b200" (default) and "gpu cuda", both served by the B200 library; the reference's CPU
backends are not part of this package.  Plotting (input_plotter / cluster_plotter) is left out.
"""
from __future__ import annotations

import os
import sys
import time
from dataclasses import dataclass
from typing import Union

import numpy as np
import pandas as pd

_PYDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "python")
if _PYDIR not in sys.path:
    sys.path.insert(0, _PYDIR)

try:
    import CLUE_Convolutional_Kernels as clue_kernels  # noqa: E402
    import CLUE_GPU_B200 as gpu_b200  # noqa: E402
except ImportError as e:  # the modules are built by `make -C cluestering_alpaka3_b200`
    raise ImportError(f"CLUE_GPU_B200 / CLUE_Convolutional_Kernels not built ({e}); "
                      "run `make -C cluestering_alpaka3_b200`") from e

BACKENDS = ("gpu b200", "gpu cuda")


def all_backends():
    return list(BACKENDS)


def canonicalize(labels, outlier=-1):
    """Renumbers labels by first appearance (outliers unchanged), so that two clusterings can be
    compared independently of label numbering (reference: CLUEstering.py:65-77)."""
    labels = np.asarray(labels)
    out = labels.copy()
    keep = labels != outlier
    if not keep.any():
        return out
    uniq, first = np.unique(labels[keep], return_index=True)
    rank = np.empty(uniq.size, np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(uniq.size)
    out[keep] = rank[np.searchsorted(uniq, labels[keep])]
    return out


@dataclass
class ClusteringDataSoA:
    """coords: (n_dim + 1) x n float32, coordinates then weights; results: n int32 cluster ids."""
    coords: np.ndarray = None
    results: np.ndarray = None
    n_dim: int = None
    n_points: int = None


@dataclass
class cluster_properties:
    n_clusters: int
    cluster_ids: np.ndarray
    cluster_points: np.ndarray
    points_per_cluster: np.ndarray
    output_df: pd.DataFrame


class clusterer:
    """CLUE clustering with the reference's Python interface, on B200 GPUs."""

    def __init__(self, dc=None, rhoc=None, dm=None, seed_dc=None, ppbin: int = 128, args=None):
        if args is not None:
            dc, rhoc, dm = args.dc, args.rhoc, args.dm
        self._dc = dc
        self._rhoc = rhoc
        self._dm = dc if dm is None else dm
        self._seed_dc = dc if seed_dc is None else seed_dc
        self._ppbin = ppbin
        self.clust_data = None
        self._kernel = clue_kernels.FlatKernel(0.5)
        self.wrapped = None
        self.clust_prop = None
        self._elapsed_time = 0.0

    def set_params(self, dc: float, rhoc: float, dm=None, seed_dc=None, ppbin: int = 128) -> None:
        self._dc = dc
        self._rhoc = rhoc
        self._dm = dc if dm is None else dm
        self._seed_dc = dc if seed_dc is None else seed_dc
        self._ppbin = ppbin

    # ---- input --------------------------------------------------------------------------
    def _read_array(self, input_data) -> None:
        if len(input_data) < 2 or len(input_data) > 11:
            raise ValueError("Inadequate data. The supported dimensions are between 1 and 10.")
        npoints = len(input_data[-1])
        ndim = len(input_data) - 1
        coords = np.ascontiguousarray(np.vstack([np.asarray(r, dtype=np.float32) for r in input_data]),
                                      dtype=np.float32)
        self.clust_data = ClusteringDataSoA(coords, np.zeros(npoints, np.int32), ndim, npoints)

    def _handle_dataframe(self, df_: pd.DataFrame) -> None:
        if len(df_.columns) < 2:
            raise ValueError("Inadequate data. The data must contain at least one coordinate and the weight.")
        if len(df_.columns) > 11:
            raise ValueError("Inadequate data. The maximum number of dimensions supported is 10.")
        arr = df_.to_numpy(dtype=np.float32)
        coords = np.ascontiguousarray(arr.T, dtype=np.float32)
        self.clust_data = ClusteringDataSoA(coords, np.zeros(len(df_.index), np.int32), arr.shape[1] - 1,
                                            len(df_.index))

    def read_data(self, input_data: Union[pd.DataFrame, str, dict, list, np.ndarray], wrapped_coords=None) -> None:
        if isinstance(input_data, (list, np.ndarray)):
            self._read_array(input_data)
        elif isinstance(input_data, str):
            if not input_data.endswith(".csv"):
                raise ValueError("Wrong type of file. The file is not a csv file.")
            self._handle_dataframe(pd.read_csv(input_data, dtype=np.float32))
        elif isinstance(input_data, (dict, pd.DataFrame)):
            self._handle_dataframe(pd.DataFrame(input_data, copy=False, dtype=np.float32))
        else:
            raise ValueError("Unsupported input type.")
        self.wrapped = list(wrapped_coords) if wrapped_coords is not None else [0] * self.clust_data.n_dim

    def set_wrapped(self, wrapped_coords) -> None:
        self.wrapped = list(wrapped_coords)

    def choose_kernel(self, choice: str, parameters=None, function=lambda: 0) -> None:
        parameters = [] if parameters is None else list(parameters)
        expected = {"flat": 1, "exp": 2, "gaus": 3}
        if choice not in expected:
            raise ValueError("Invalid kernel. Allowed choices are: flat, exp, gaus.")
        if len(parameters) != expected[choice]:
            raise ValueError(f"Wrong number of parameters. The {choice} kernel requires "
                             f"{expected[choice]} parameter(s).")
        cls = {"flat": clue_kernels.FlatKernel, "exp": clue_kernels.ExponentialKernel,
               "gaus": clue_kernels.GaussianKernel}[choice]
        self._kernel = cls(*parameters)

    @property
    def coords(self) -> np.ndarray:
        return self.clust_data.coords[:-1]

    @property
    def weight(self) -> np.ndarray:
        return self.clust_data.coords[-1]

    @property
    def n_dim(self) -> int:
        return self.clust_data.n_dim

    @property
    def n_points(self) -> int:
        return self.clust_data.n_points

    def list_devices(self, backend: str = "all") -> None:
        if backend not in ("all",) + BACKENDS:
            raise ValueError(f"Invalid backend. Allowed choices are: all, {', '.join(BACKENDS)}.")
        gpu_b200.listDevices(backend if backend != "all" else "gpu b200")

    # ---- run ----------------------------------------------------------------------------
    def run_clue(self, backend: str = "gpu b200", block_size: int = 1024, device_id: int = 0, verbose: bool = False,
                 dimensions=None) -> None:
        if backend not in BACKENDS:
            raise ValueError(f"Invalid backend '{backend}'. Allowed choices are: {', '.join(BACKENDS)}.")
        data = self.clust_data
        if dimensions is not None:
            rows = [data.coords[d] for d in dimensions] + [data.coords[-1]]
            data = ClusteringDataSoA(np.ascontiguousarray(np.vstack(rows), dtype=np.float32),
                                     np.zeros(data.n_points, np.int32), len(dimensions), data.n_points)
        wrapped = [int(w) for w in (self.wrapped or [])]
        if dimensions is not None:
            wrapped = [wrapped[d] if d < len(wrapped) else 0 for d in dimensions]
        start = time.time_ns()
        gpu_b200.mainRun(self._dc, self._rhoc, self._dm, self._seed_dc, self._ppbin, wrapped, data.coords,
                         data.results, self._kernel, data.n_dim, data.n_points, block_size, device_id)
        finish = time.time_ns()
        ids = data.results.copy()
        self.clust_prop = self._properties(ids, pd.DataFrame({"cluster_ids": ids}))
        self._elapsed_time = (finish - start) / 1e6
        if verbose:
            print(f"CLUE executed in {self._elapsed_time} ms")
            print(f"Number of clusters found: {self.clust_prop.n_clusters}")

    @staticmethod
    def _properties(ids: np.ndarray, df_: pd.DataFrame) -> cluster_properties:
        n_clusters = int(ids.max()) + 1 if ids.size else 0
        keep = ids >= 0
        members = np.nonzero(keep)[0][np.argsort(ids[keep], kind="stable")]
        counts = np.bincount(ids[keep], minlength=n_clusters) if n_clusters > 0 else np.zeros(0, np.int64)
        splits = np.cumsum(counts)[:-1] if n_clusters > 0 else []
        points = np.empty(n_clusters, dtype=object)
        for c, part in enumerate(np.split(members, splits) if n_clusters > 0 else []):
            points[c] = part.tolist()
        return cluster_properties(n_clusters, ids, points, counts, df_)

    def run_clue_from_args(self, args):
        return self.run_clue(backend=args.backend, block_size=args.block_size, device_id=args.device_id,
                             verbose=args.verbose, dimensions=args.dimension)

    def fit(self, data, backend: str = "gpu b200", block_size: int = 1024, device_id: int = 0, verbose: bool = False,
            dimensions=None) -> "clusterer":
        self.read_data(data)
        self.run_clue(backend, block_size, device_id, verbose, dimensions)
        return self

    def fit_predict(self, data, backend: str = "gpu b200", block_size: int = 1024, device_id: int = 0,
                    verbose: bool = False, dimensions=None) -> np.ndarray:
        self.read_data(data)
        self.run_clue(backend, block_size, device_id, verbose, dimensions)
        return self.cluster_ids

    # ---- results ------------------------------------------------------------------------
    @property
    def n_clusters(self) -> int:
        return self.clust_prop.n_clusters

    @property
    def cluster_ids(self) -> np.ndarray:
        return self.clust_prop.cluster_ids

    @property
    def labels(self) -> np.ndarray:
        return self.clust_prop.cluster_ids

    @property
    def cluster_points(self) -> np.ndarray:
        return self.clust_prop.cluster_points

    @property
    def points_per_cluster(self) -> np.ndarray:
        return self.clust_prop.points_per_cluster

    @property
    def output_df(self) -> pd.DataFrame:
        return self.clust_prop.output_df

    def cluster_centroid(self, cluster_index: int) -> np.ndarray:
        sel = self.clust_prop.cluster_ids == cluster_index
        if not sel.any():
            raise ValueError(f"No cluster with index {cluster_index}.")
        return self.clust_data.coords[:-1, sel].astype(np.float64).mean(axis=1)

    def cluster_centroids(self) -> np.ndarray:
        ids = self.clust_prop.cluster_ids
        keep = ids >= 0
        sums = np.zeros((self.clust_prop.n_clusters, self.clust_data.n_dim))
        np.add.at(sums, ids[keep], self.clust_data.coords[:-1, keep].T.astype(np.float64))
        return sums / self.clust_prop.points_per_cluster.reshape(-1, 1)

    def to_csv(self, output_folder: str, file_name: str) -> None:
        if not output_folder.endswith("/"):
            output_folder += "/"
        if not file_name.endswith(".csv"):
            file_name += ".csv"
        data = {f"x{i}": self.clust_data.coords[i] for i in range(self.clust_data.n_dim)}
        data["weight"] = self.clust_data.coords[-1]
        data["cluster_ids"] = self.clust_prop.cluster_ids
        pd.DataFrame(data).to_csv(output_folder + file_name, index=False)

    def import_clusterer(self, input_folder: str, file_name: str) -> None:
        df_ = pd.read_csv(os.path.join(input_folder, file_name))
        ids = np.asarray(df_["cluster_ids"], dtype=np.int32)
        cols = [c for c in df_.columns if c.startswith("x")] + ["weight"]
        self._handle_dataframe(df_[cols].astype(np.float32))
        self.clust_data.results[:] = ids
        self.clust_prop = self._properties(ids, df_)
