"""The clue:: C++ API (include/CLUEstering) compiled against libclue_b200.

The CPU test builds tests/cpp/test_api.cpp and runs its host-only checks (kernels, metrics,
points containers, association maps, CSV I/O, cluster properties, centroids).  The GPU test
clusters golden inputs through every make_clusters overload and compares the result with the
oracle bit for bit, plus the reference's own checks on data_32768 (20 clusters, silhouette
>= 0.9, tests/test_clusterer.cpp and tests/test_host_points.cpp in the reference).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_api.cpp")


def build(tmp_path):
    from cluestering_alpaka3_b200 import capi
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    libdir = os.path.dirname(capi.LIB_PATH)
    exe = str(tmp_path / "test_api")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", libdir, "-lclue_b200", f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_api_host_parts(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe, "cpu", str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED" in r.stdout


def write_csv(path, coords, weight):
    with open(path, "w") as f:
        f.write("x0,x1,weight\n")
        for i in range(coords.shape[1]):
            f.write("%.9g,%.9g,%.9g\n" % (coords[0, i], coords[1, i], weight[i]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["data_32768", "data_4096", "sissa_1000", "toyDetector_1000"])
def test_cpp_api_clustering_matches_oracle(tmp_path, name, gpu_context):
    exe = build(tmp_path)
    g = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    coords, weight = g["coords"], g["weight"]
    dc, rhoc, dm = (float(v) for v in g["params"])
    src = str(tmp_path / "in.csv")
    out = str(tmp_path / "out.csv")
    write_csv(src, coords, weight)
    r = subprocess.run([exe, "gpu", src, repr(dc), repr(rhoc), repr(dm), out], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    res = np.loadtxt(out, delimiter=",", skiprows=1, dtype=np.float64)
    labels = res[:, 3].astype(np.int32)
    is_seed = res[:, 4].astype(np.int32)
    nh = res[:, 5].astype(np.int32)
    rho_bits = res[:, 6].astype(np.uint32)
    delta_bits = res[:, 7].astype(np.uint32)

    ref = O.run(coords, weight, O.Config(dc=np.float32(dc), rhoc=np.float32(rhoc), dm=np.float32(dm)))
    np.testing.assert_array_equal(labels, ref.cluster_index)
    np.testing.assert_array_equal(is_seed, ref.is_seed)
    np.testing.assert_array_equal(nh, ref.nearest_higher)
    np.testing.assert_array_equal(rho_bits, ref.rho.view(np.uint32))
    np.testing.assert_array_equal(delta_bits, ref.delta.view(np.uint32))

    summary = dict(kv.split("=") for kv in r.stdout.split("\n")[0].split())
    assert int(summary["n_clusters"]) == ref.stats["n_clusters"]
    if name == "data_32768":
        assert int(summary["n_clusters"]) == 20
        assert float(summary["silhouette"]) >= 0.9
