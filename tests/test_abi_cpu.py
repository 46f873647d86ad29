"""The C ABI library on the host (no GPU needed): symbols, validation, grid, plugins."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            syms |= set(re.findall(r"\b(clue_[a-z0-9_]+)\s*\(", txt))
    return syms


def test_library_exports_every_declared_symbol():
    from cluestering_alpaka3_b200 import capi
    syms = declared_symbols()
    assert "clue_make_clusters" in syms
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(capi.EXPORTED) >= syms


def test_abi_version():
    from cluestering_alpaka3_b200 import capi
    assert capi.lib.clue_abi_version() == 2


@pytest.mark.parametrize("dc,rhoc,dm,seed,ppbin", [(0.0, 1, 1, 1, 128), (-1, 1, 1, 1, 128), (1, -1, 1, 1, 128),
                                                    (1, 1, 0, 1, 128), (1, 1, 1, 0, 128), (1, 1, 1, 1, 0),
                                                    (float("nan"), 1, 1, 1, 128)])
def test_invalid_params_rejected(dc, rhoc, dm, seed, ppbin):
    # reference tests/test_clusterer.cpp:47-54 and core/detail/Clusterer.hpp:24-51
    from cluestering_alpaka3_b200 import capi
    with pytest.raises(ValueError):
        capi.Params(dc=dc, rhoc=rhoc, dm=dm, seed_dc=seed, points_per_tile=ppbin).struct()


def test_valid_params_accepted():
    from cluestering_alpaka3_b200 import capi
    capi.Params(dc=1.3, rhoc=0.0, dm=1.3).struct()


@pytest.mark.parametrize("k", [("flat", (0.0,)), ("flat", (-1.0,)), ("exp", (0.0, 1.0)), ("exp", (1.0, 0.0)),
                               ("exp", (-1.0, 1.0)), ("exp", (1.0, -1.0)), ("gaus", (1.0, 0.0, 1.0)),
                               ("gaus", (1.0, 1.0, 0.0)), ("gaus", (-1.0, 1.0, 1.0)), ("gaus", (1.0, -1.0, 1.0)),
                               ("gaus", (1.0, 1.0, -1.0))])
def test_kernel_throw_rules(k):
    # reference tests/test_convolutional_kernels.cpp:7-26 (Gaussian mean 0 is accepted here)
    from cluestering_alpaka3_b200 import capi
    from parity_util import KERNEL_NAMES
    with pytest.raises(ValueError):
        capi.Kernel(KERNEL_NAMES[k[0]], k[1]).struct()


def test_gaussian_mean_zero_accepted():
    from cluestering_alpaka3_b200 import capi
    capi.GaussianKernel(0.0, 0.5, 1.0).struct()


@pytest.mark.parametrize("n,ppbin,nd", [(1, 128, 2), (127, 128, 2), (129, 128, 2), (16384, 128, 2),
                                        (1 << 20, 128, 2), (1 << 22, 128, 3), (999, 7, 4), (10000, 128, 10),
                                        (5000, 1, 1)])
def test_grid_shape_matches_oracle(n, ppbin, nd):
    from cluestering_alpaka3_b200 import capi
    npd, nt = capi.grid_shape(n, ppbin, nd)
    c = np.zeros((nd, n), np.float32)
    g, off, idx = O.tiles(c, O.Config(1.0, 1.0, ppbin=ppbin))
    assert (npd, nt) == (g["nperdim"], g["ntiles"])


@pytest.mark.parametrize("metric,par", [("euclidean", ()), ("weighted_euclidean", (0.3, 2.0, 1.1)),
                                        ("periodic_euclidean", (6.0, 0.0, 10.0)), ("manhattan", ()),
                                        ("chebyshev", ()), ("weighted_chebyshev", (0.3, 2.0, 1.1))])
def test_metric_eval_bitexact_vs_oracle(metric, par):
    from cluestering_alpaka3_b200 import capi
    rng = np.random.default_rng(1)
    m = capi.Metric(list(O.METRICS).index(metric), par)
    cfg = O.Config(1, 1, metric=metric, metric_par=par)
    for _ in range(200):
        a = rng.normal(0, 10, 3).astype(np.float32)
        b = rng.normal(0, 10, 3).astype(np.float32)
        x, y = np.float32(capi.metric_eval(m, a, b)), np.float32(O.metric(a, b, cfg))
        assert x.view(np.uint32) == y.view(np.uint32)


def test_metric_sentinel_is_infinite():
    # distance to the FLT_MAX sentinel of PointsView::operator[](-1) exceeds any seed_dc
    from cluestering_alpaka3_b200 import capi
    a = np.array([1.0, 2.0], np.float32)
    s = np.full(2, np.finfo(np.float32).max, np.float32)
    for t in range(6):
        m = capi.Metric(t, (1.0, 1.0))
        assert capi.metric_eval(m, a, s) > 1e30


def test_kernel_eval_vs_oracle():
    from cluestering_alpaka3_b200 import capi
    for k, cfg in [(capi.FlatKernel(0.5), O.Config(1, 1)),
                   (capi.ExponentialKernel(1.0, 2.0), O.Config(1, 1, kernel="exp", kernel_par=(1.0, 2.0))),
                   (capi.GaussianKernel(0.5, 0.7, 1.5), O.Config(1, 1, kernel="gaus", kernel_par=(0.5, 0.7, 1.5)))]:
        for d in (0.0, 0.3, 1.0, 2.5):
            assert capi.kernel_eval(k, d, 1, 2) == O.kernel(d, 1, 2, cfg)
            assert capi.kernel_eval(k, d, 3, 3) == 1.0


def test_no_gpu_calls_fail_cleanly():
    from cluestering_alpaka3_b200 import capi
    if capi.device_count() > 0:
        pytest.skip("GPU present")
    with pytest.raises(capi.ClueError):
        capi.Context(0)


def test_tuning_defaults():
    import ctypes
    from cluestering_alpaka3_b200 import capi
    t = capi._Tuning()
    capi.lib.clue_tuning_defaults(ctypes.byref(t))
    assert (t.symmetric_density, t.nh_split_lanes, t.overlap_chunk_points) == (1, 8, 2200000)
