"""The CPU oracle pinned against the reference's own golden data (CPU only).

* known answer: data_32768 @ (dc, rhoc, dm) = (1.3, 10, 1.3) -> 20 clusters
  (reference tests/test_device_points.cpp:252-268, tests/test_host_points.cpp:437-450);
* truth files data/truth_files/*_truth.csv: blob.csv @ (1, 5, 2) reproduces the truth labels
  exactly; the data_N files (parameters not recorded in the reference) agree on the number of
  clusters and on >= 99.5% of the labels at the reference tests' parameters;
* metric known answers of tests/test_distance_metrics.cpp:8-63.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z


def matched_agreement(a, b):
    """Fraction of points whose label agrees after matching clusters by maximal overlap."""
    agree = 0
    for lab in np.unique(a):
        m = a == lab
        if lab == -1:
            agree += int((b[m] == -1).sum())
            continue
        vals, cnt = np.unique(b[m], return_counts=True)
        agree += int(cnt[vals != -1].max()) if (vals != -1).any() else 0
    return agree / len(a)


def test_known_answer_20_clusters():
    z = load("data_32768")
    r = O.run(z["coords"], z["weight"], O.Config(dc=1.3, rhoc=10.0, dm=1.3))
    assert r.stats["n_clusters"] == 20
    assert r.cluster_index.max() + 1 == 20


def test_blob_truth_exact():
    z = load("blob")
    dc, rhoc, dm = (float(v) for v in z["params"])
    r = O.run(z["coords"], z["weight"], O.Config(dc=dc, rhoc=rhoc, dm=dm))
    np.testing.assert_array_equal(O.canonicalize(r.cluster_index), O.canonicalize(z["truth_cluster_ids"]))


@pytest.mark.parametrize("name", ["data_1024", "data_2048", "data_4096", "data_8192", "data_16384",
                                  "data_32768"])
def test_truth_files_agree(name):
    z = load(name)
    dc, rhoc, dm = (float(v) for v in z["params"])
    r = O.run(z["coords"], z["weight"], O.Config(dc=dc, rhoc=rhoc, dm=dm))
    truth = z["truth_cluster_ids"]
    assert r.stats["n_clusters"] == truth.max() + 1
    assert matched_agreement(r.cluster_index, truth) >= 0.995


@pytest.mark.parametrize("name", ["sissa_1000", "toyDetector_1000", "aniso_1000"])
def test_truth_files_cluster_count(name):
    z = load(name)
    dc, rhoc, dm = (float(v) for v in z["params"])
    r = O.run(z["coords"], z["weight"], O.Config(dc=dc, rhoc=rhoc, dm=dm))
    assert r.stats["n_clusters"] == z["truth_cluster_ids"].max() + 1
    assert matched_agreement(r.cluster_index, z["truth_cluster_ids"]) >= 0.95


def test_metric_known_answers():
    a2, b2 = [1.0, 2.0], [4.0, 6.0]
    assert O.metric(a2, b2, O.Config(1, 1)) == pytest.approx(5.0)
    assert O.metric(a2, b2, O.Config(1, 1, metric="weighted_euclidean", metric_par=(1.0, 2.0))) == \
        pytest.approx(np.sqrt(41.0))
    assert O.metric([-1.0, 3.0], [0.0, 6.0], O.Config(1, 1, metric="manhattan")) == pytest.approx(4.0)
    assert O.metric([-1.0, 4.0], [0.0, 6.0], O.Config(1, 1, metric="chebyshev")) == pytest.approx(2.0)
    assert O.metric([-1.0, 4.0], [0.0, 6.0],
                    O.Config(1, 1, metric="weighted_chebyshev", metric_par=(1.0, 2.0))) == pytest.approx(4.0)


def test_kernel_values():
    cfg = O.Config(1, 1, kernel="flat", kernel_par=(0.5,))
    assert O.kernel(3.0, 1, 2, cfg) == 0.5 and O.kernel(3.0, 2, 2, cfg) == 1.0
    cfg = O.Config(1, 1, kernel="exp", kernel_par=(1.0, 2.0))
    assert O.kernel(0.5, 1, 2, cfg) == pytest.approx(2.0 * np.exp(-0.5), rel=1e-6)
    cfg = O.Config(1, 1, kernel="gaus", kernel_par=(1.0, 0.5, 3.0))
    assert O.kernel(2.0, 1, 2, cfg) == pytest.approx(3.0 * np.exp(-1.0 / 0.5), rel=1e-6)


def test_grid_shape_examples():
    # nperdim for the benchmark configs: 12 (16384 2-D), 91 (1M 2-D), 32 (4M 3-D)
    for n, nd, npd in [(16384, 2, 12), (1 << 20, 2, 91), (1 << 22, 3, 32), (100, 2, 1)]:
        c = np.zeros((nd, n), np.float32)
        c[:, -1] = 1.0
        g, off, idx = O.tiles(c, O.Config(1.0, 1.0))
        assert g["nperdim"] == npd
        assert off[-1] == n


@pytest.mark.parametrize("tiebreak", ["reference", "rho_index"])
def test_nearest_higher_stage_matches_full_run(tiebreak):
    # the stage-alone entry reproduces the full run's nearest higher (before seeds are cut
    # loose) and delta, on lattice coordinates with many exact distance ties
    rng = np.random.default_rng(3)
    c = rng.integers(0, 30, size=(2, 3000)).astype(np.float32)
    w = np.ones(3000, np.float32)
    cfg = O.Config(dc=1.5, rhoc=2.0, dm=2.5, tiebreak=tiebreak)
    ref = O.run(c, w, cfg)
    nh, delta, ties = O.nearest_higher(c, ref.rho, cfg)
    keep = ref.is_seed == 0
    np.testing.assert_array_equal(nh[keep], ref.nearest_higher[keep])
    np.testing.assert_array_equal(delta.view(np.uint32), ref.delta.view(np.uint32))
    assert ties == ref.stats["nh_distance_ties"] > 0


def test_silhouette_restatement_matches_scalar_float32():
    # the oracle's silhouette against a plain float32 evaluation of the reference's definition
    # (scores.hpp:17-99) on a small labelled set
    rng = np.random.default_rng(12)
    n = 90
    c = rng.normal(size=(2, n)).astype(np.float32)
    c[0, :40] += np.float32(4.0)
    lab = np.where(np.arange(n) < 40, 0, np.where(np.arange(n) < 75, 1, 2)).astype(np.int32)
    lab[::11] = -1
    per, mean = O.silhouette(c, lab)
    f = np.float32
    k = int(lab.max()) + 1
    members = [np.nonzero(lab == q)[0] for q in range(k)]
    scores = []
    for i in range(n):
        own = lab[i]
        if own < 0 or members[own].size < 2:
            assert np.isnan(per[i])
            continue
        a, b = f(0), f(np.finfo(np.float32).max)
        for q in range(k):
            s = f(0)
            for j in members[q]:
                if q == own and j == i:
                    continue
                d = f(0)
                for dd in range(2):
                    t = f(c[dd, i] - c[dd, j])
                    d = f(d + f(t * t))
                s = f(s + f(np.sqrt(d)))
            if q == own:
                a = f(s / f(members[q].size - 1))
            else:
                m = f(s / f(members[q].size))
                b = m if m < b else b
        sc = f(f(b - a) / (b if a < b else a))
        assert per[i].view(np.uint32) == sc.view(np.uint32), i
        scores.append(sc)
    acc = f(0)
    for sc in scores:
        acc = f(acc + sc)
    assert np.float32(mean).view(np.uint32) == f(acc / f(len(scores))).view(np.uint32)
