"""Device association map (clue_get_clusters): the CSR the reference's host fill builds
(data_structures/AssociationMap.hpp:53-74 -- keys 0..max label, point indexes ascending inside a
key, label -1 left out), computed on the GPU, and the centroids computed from it."""
import os

import numpy as np
import pytest

from parity_util import gpu_args, random_blobs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def host_csr(labels):
    k = int(labels.max()) + 1 if labels.size and labels.max() >= 0 else 0
    keep = labels >= 0
    order = np.argsort(labels[keep], kind="stable")
    points = np.nonzero(keep)[0][order].astype(np.int32)
    counts = np.bincount(labels[keep], minlength=k)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return k, offsets, points


def device_csr(ctx, labels):
    import torch
    n = labels.size
    d_lab = torch.from_numpy(labels).cuda()
    off = torch.full((n + 1,), -5, dtype=torch.int32, device="cuda")
    pts = torch.full((n,), -5, dtype=torch.int32, device="cuda")
    k, m = ctx.get_clusters(d_lab.data_ptr(), n, off.data_ptr(), pts.data_ptr())
    return k, m, off.cpu().numpy(), pts.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n,k,outlier_frac", [(1, 1, 0.0), (1000, 2, 0.0), (65537, 300, 0.2), (1 << 20, 5000, 0.1),
                                              (777, 0, 1.0)])
def test_get_clusters_random_labels(gpu_context, n, k, outlier_frac):
    rng = np.random.default_rng(n + k)
    labels = rng.integers(0, max(k, 1), n).astype(np.int32)
    labels[rng.random(n) < outlier_frac] = -1
    kk, offsets, points = host_csr(labels)
    got_k, got_m, off, pts = device_csr(gpu_context, labels)
    assert got_k == kk
    assert got_m == points.size
    np.testing.assert_array_equal(off[:kk + 1], offsets)
    assert np.all(off[kk + 1:] == points.size)
    np.testing.assert_array_equal(pts[:points.size], points)


@pytest.mark.gpu
def test_get_clusters_of_a_clustering(gpu_context):
    rng = np.random.default_rng(5)
    c, w = random_blobs(rng, 50000, 2, nblobs=12, extent=80.0)
    res = gpu_context.make_clusters_host(c, w, *gpu_args(dc=1.2, rhoc=5.0, dm=1.5))
    kk, offsets, points = host_csr(res.cluster_index)
    got_k, got_m, off, pts = device_csr(gpu_context, res.cluster_index)
    assert got_k == kk == res.info.n_clusters
    np.testing.assert_array_equal(off[:kk + 1], offsets)
    np.testing.assert_array_equal(pts[:got_m], points)


@pytest.mark.gpu
def test_get_clusters_rejects_labels_out_of_range(gpu_context):
    from cluestering_alpaka3_b200 import capi
    labels = np.array([0, 1, 7, -1, -2], np.int32)  # 7 >= n and -2 < -1
    with pytest.raises(capi.ClueError):
        device_csr(gpu_context, labels)


@pytest.mark.gpu
@pytest.mark.parametrize("name,ndim", [("data_4096", 2), ("blobs3d", 3)])
def test_silhouette_gpu_matches_oracle(gpu_context, name, ndim):
    # clue_silhouette against the oracle's restatement of the reference's scores.hpp: every
    # point's score bit for bit (cluster sums in ascending point order, separately rounded
    # FP32), points not scored NaN, and the FP32 mean in index order
    import os
    import torch
    from oracle import oracle as O
    if name == "data_4096":
        z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
        coords, weight = z["coords"], z["weight"]
        dc_, rhoc_, dm_ = (float(v) for v in z["params"])
        kw = dict(dc=dc_, rhoc=rhoc_, dm=dm_)
    else:
        rng = np.random.default_rng(151)
        coords, weight = random_blobs(rng, 3000, 3, nblobs=6, extent=30.0, sigma=0.8)
        kw = dict(dc=1.2, rhoc=3.0, dm=1.6)
    res = gpu_context.make_clusters_host(coords, weight, *gpu_args(**kw))
    labels = res.cluster_index
    assert labels.max() >= 1  # at least two clusters
    n = coords.shape[1]
    dc = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.float32)).cuda()
    dl = torch.from_numpy(labels.astype(np.int32)).cuda()
    per = torch.empty(n, dtype=torch.float32, device="cuda")
    mean = gpu_context.silhouette_device(dc.data_ptr(), dl.data_ptr(), ndim, n, per.data_ptr())
    ref_per, ref_mean = O.silhouette(coords, labels)
    got = per.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(got), np.isnan(ref_per))
    ok = ~np.isnan(ref_per)
    np.testing.assert_array_equal(got[ok].view(np.uint32), ref_per[ok].view(np.uint32))
    assert np.float32(mean).view(np.uint32) == np.float32(ref_mean).view(np.uint32)


@pytest.mark.gpu
def test_silhouette_gpu_reference_known_answer(gpu_context):
    # the reference's check on data_32768 (tests/test_device_points.cpp:252-268): 20 clusters
    # with silhouette >= 0.9
    import os
    import torch
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "data_32768.npz"))
    coords, weight = z["coords"], z["weight"]
    res = gpu_context.make_clusters_host(coords, weight, *gpu_args(dc=1.3, rhoc=10.0, dm=1.3))
    assert res.info.n_clusters == 20
    n = coords.shape[1]
    dc = torch.from_numpy(np.ascontiguousarray(coords, dtype=np.float32)).cuda()
    dl = torch.from_numpy(res.cluster_index.astype(np.int32)).cuda()
    assert gpu_context.silhouette_device(dc.data_ptr(), dl.data_ptr(), 2, n) >= 0.9


@pytest.mark.gpu
def test_cluster_centroids_gpu_bits(gpu_context):
    # Centroids on the GPU (clue_cluster_centroids) against the reference's host loop
    # (utils/detail/cluster_centroid.hpp:39-65): FP32 sums from 0 in ascending point order,
    # divided by the cluster size as a float; bit for bit.  Sizes are the clusters' point counts.
    import numpy as np
    from oracle import oracle as O
    for name, ndim in (("data_4096", 2), ("blob", 3)):
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        c, w = g["coords"], g["weight"]
        dc, rhoc, dm = (float(v) for v in g["params"])
        labels = O.run(c, w, O.Config(dc=dc, rhoc=rhoc, dm=dm)).cluster_index
        cen, sizes = gpu_context.cluster_centroids(c, labels)
        k = int(labels.max()) + 1
        assert cen.shape == (k, c.shape[0])
        for cl in range(k):
            members = np.nonzero(labels == cl)[0]
            assert sizes[cl] == members.size
            for d in range(c.shape[0]):
                s = np.cumsum(c[d, members].astype(np.float32), dtype=np.float32)[-1]  # sequential FP32
                exp = np.float32(s) / np.float32(members.size)
                assert cen[cl, d].view(np.uint32) == np.float32(exp).view(np.uint32), (name, cl, d)
    # no clustered point: zero clusters, nothing written
    cen, sizes = gpu_context.cluster_centroids(np.zeros((2, 10), np.float32), np.full(10, -1, np.int32))
    assert cen.shape == (0, 2)
