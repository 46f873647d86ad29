"""The Python entry of the reference: backend module mainRun (same signature as the reference's
CLUE_GPU_CUDA / CLUE_CPU_Serial modules, CLUEstering/BindingModules/serial/binding_cpu.cpp:34-47)
and the `clusterer` class (CLUEstering/CLUEstering.py:272-1260), running on libclue_b200.
Flat-kernel runs are compared with the oracle bit for bit."""
import os
import sys

import numpy as np
import pandas as pd
import pytest

from oracle import oracle as O
from parity_util import random_blobs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PYDIR = os.path.join(ROOT, "cluestering_alpaka3_b200", "python")


@pytest.fixture(scope="module")
def mods():
    if PYDIR not in sys.path:
        sys.path.insert(0, PYDIR)
    import CLUE_Convolutional_Kernels as K
    import CLUE_GPU_B200 as B
    import CLUE_GPU_CUDA as C
    return K, B, C


def soa(coords, weight):
    return np.ascontiguousarray(np.vstack([coords, weight[None, :]]), dtype=np.float32)


# ---- host-only ------------------------------------------------------------------------------
def test_kernel_module_validation(mods):
    K, _, _ = mods
    K.FlatKernel(0.5)
    K.ExponentialKernel(1.0, 1.0)
    K.GaussianKernel(0.0, 0.5, 1.0)  # mean 0 accepted
    for bad in [lambda: K.FlatKernel(0.0), lambda: K.FlatKernel(-1.0), lambda: K.ExponentialKernel(0.0, 1.0),
                lambda: K.ExponentialKernel(1.0, -1.0), lambda: K.GaussianKernel(1.0, 0.0, 1.0),
                lambda: K.GaussianKernel(1.0, 1.0, 0.0), lambda: K.GaussianKernel(-1.0, 1.0, 1.0)]:
        with pytest.raises(ValueError):
            bad()


def test_canonicalize():
    from cluestering_alpaka3_b200.clusterer import canonicalize
    np.testing.assert_array_equal(canonicalize([3, 3, -1, 0, 7, 0, -1, 3]), [0, 0, -1, 1, 2, 1, -1, 0])
    np.testing.assert_array_equal(canonicalize([-1, -1]), [-1, -1])


def test_read_data_forms(tmp_path):
    from cluestering_alpaka3_b200.clusterer import clusterer
    rng = np.random.default_rng(0)
    x, y, w = rng.random(50, dtype=np.float32), rng.random(50, dtype=np.float32), np.ones(50, np.float32)
    ref = np.vstack([x, y, w])
    forms = [[x, y, w], np.vstack([x, y, w]), {"x0": x, "x1": y, "weight": w},
             pd.DataFrame({"x0": x, "x1": y, "weight": w})]
    p = tmp_path / "d.csv"
    pd.DataFrame({"x0": x, "x1": y, "weight": w}).to_csv(p, index=False)
    forms.append(str(p))
    for f in forms:
        c = clusterer(1.0, 2.0)
        c.read_data(f)
        assert c.n_dim == 2 and c.n_points == 50 and c.wrapped == [0, 0]
        np.testing.assert_array_equal(c.clust_data.coords, ref)
        assert c.clust_data.coords.flags["C_CONTIGUOUS"] and c.clust_data.coords.dtype == np.float32
    c = clusterer(1.0, 2.0)
    with pytest.raises(ValueError):
        c.read_data([x])
    with pytest.raises(ValueError):
        c.read_data([x] * 12)
    with pytest.raises(ValueError):
        c.read_data(str(tmp_path / "d.txt"))
    with pytest.raises(ValueError):
        c.choose_kernel("flat", [1.0, 2.0])
    with pytest.raises(ValueError):
        c.choose_kernel("triangle", [1.0])
    c.read_data(forms[0])
    with pytest.raises(ValueError):
        c.run_clue(backend="cpu serial")
    assert clusterer(1.0, 2.0)._dm == 1.0 and clusterer(1.0, 2.0, 3.0, 4.0)._seed_dc == 4.0


# ---- GPU ------------------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("ndim", [1, 2, 3, 4])
def test_mainrun_flat_matches_oracle(gpu_context, mods, ndim):
    K, B, C = mods
    rng = np.random.default_rng(40 + ndim)
    c, w = random_blobs(rng, 20000, ndim, nblobs=10, extent=60.0)
    dc, rhoc, dm = 1.2, 5.0, 1.6
    ref = O.run(c, w, O.Config(dc=dc, rhoc=rhoc, dm=dm))
    for mod in (B, C):
        data = soa(c, w)
        res = np.full(c.shape[1], -7, np.int32)
        mod.mainRun(dc, rhoc, dm, dc, 128, [0] * ndim, data, res, K.FlatKernel(0.5), ndim, c.shape[1], 256, 0)
        np.testing.assert_array_equal(res, ref.cluster_index)


@pytest.mark.gpu
def test_mainrun_wrapped_and_params(gpu_context, mods):
    K, B, _ = mods
    rng = np.random.default_rng(3)
    c = np.vstack([rng.uniform(-np.pi, np.pi, 6000), rng.normal(0, 1.0, 6000)]).astype(np.float32)
    w = np.ones(6000, np.float32)
    ref = O.run(c, w, O.Config(dc=0.3, rhoc=3.0, dm=0.4, seed_dc=0.5, ppbin=64, wrapped=(1, 0)))
    res = np.zeros(6000, np.int32)
    B.mainRun(0.3, 3.0, 0.4, 0.5, 64, [1, 0], soa(c, w), res, K.FlatKernel(0.5), 2, 6000, 1024, 0)
    np.testing.assert_array_equal(res, ref.cluster_index)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [("exp", (1.0, 1.0)), ("gaus", (0.0, 0.5, 1.0))])
def test_mainrun_exp_gauss_labels(gpu_context, mods, kernel):
    K, B, _ = mods
    rng = np.random.default_rng(9)
    c, w = random_blobs(rng, 10000, 2, nblobs=12, extent=80.0, sigma=1.2)
    ref = O.run(c, w, O.Config(dc=2.0, rhoc=4.0, dm=3.0, kernel=kernel[0], kernel_par=kernel[1]))
    k = K.ExponentialKernel(*kernel[1]) if kernel[0] == "exp" else K.GaussianKernel(*kernel[1])
    res = np.zeros(10000, np.int32)
    B.mainRun(2.0, 4.0, 3.0, 2.0, 128, [0, 0], soa(c, w), res, k, 2, 10000, 256, 0)
    # mainRun returns labels only: they equal the C ABI run of the same pipeline, whose full
    # outputs meet the tolerance rule (rho within 1e-5 of FP64, later stages exact on the device's
    # densities, every label difference from the restatement caused by a near-threshold point)
    from parity_util import check_tolerant, gpu_args
    got = gpu_context.make_clusters_host(c, w, *gpu_args(dc=2.0, rhoc=4.0, dm=3.0, kernel=kernel))
    np.testing.assert_array_equal(res, got.cluster_index)
    cfg = O.Config(dc=2.0, rhoc=4.0, dm=3.0, kernel=kernel[0], kernel_par=kernel[1], nthreads=os.cpu_count() or 1)
    check_tolerant(c, w, cfg, got, ref=ref, tag="mainRun " + kernel[0])


@pytest.mark.gpu
def test_clusterer_known_answer_and_io(gpu_context, tmp_path):
    from cluestering_alpaka3_b200.clusterer import clusterer
    g = np.load(os.path.join(ROOT, "tests", "golden", "data_32768.npz"))
    df = pd.DataFrame({"x0": g["coords"][0], "x1": g["coords"][1], "weight": g["weight"]})
    cl = clusterer(1.3, 10.0, 1.3)
    labels = cl.fit_predict(df)
    ref = O.run(g["coords"], g["weight"], O.Config(dc=1.3, rhoc=10.0, dm=1.3))
    np.testing.assert_array_equal(labels, ref.cluster_index)
    assert cl.n_clusters == 20
    assert cl.points_per_cluster.sum() == (labels >= 0).sum()
    assert sorted(cl.cluster_points[3]) == list(np.nonzero(labels == 3)[0])
    cents = cl.cluster_centroids()
    np.testing.assert_allclose(cents[3], g["coords"][:, labels == 3].astype(np.float64).mean(axis=1), rtol=1e-6)
    np.testing.assert_allclose(cl.cluster_centroid(3), cents[3])
    cl.to_csv(str(tmp_path), "out")
    back = clusterer(1.3, 10.0, 1.3)
    back.import_clusterer(str(tmp_path) + "/", "out.csv")
    np.testing.assert_array_equal(back.cluster_ids, labels)
    assert back.n_clusters == 20
    # dimensions subset: cluster on x0 only equals a 1-D run
    one = clusterer(1.3, 10.0, 1.3)
    one.read_data(df)
    one.run_clue(dimensions=[0])
    ref1 = O.run(g["coords"][:1].copy(), g["weight"], O.Config(dc=1.3, rhoc=10.0, dm=1.3))
    np.testing.assert_array_equal(one.cluster_ids, ref1.cluster_index)
