"""Device association map (clue_get_clusters): the CSR the reference's host fill builds
(data_structures/AssociationMap.hpp:53-74 -- keys 0..max label, point indexes ascending inside a
key, label -1 left out), computed on the GPU."""
import numpy as np
import pytest

from parity_util import gpu_args, random_blobs


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
