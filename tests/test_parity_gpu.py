"""GPU parity: libclue_b200 against the CPU restatement of the reference's serial path.

Flat-kernel runs are compared bit for bit on every output (rho and delta included): the
device sums in the reference's candidate order with separately rounded float ops.
Exponential / Gaussian kernels call CUDA's expf, which may differ from glibc's by an ulp,
so rho is held to 1e-5 relative of the FP64 oracle, every later stage must be exact on the
device's own densities, and every difference from the restatement's own run must trace back to
a counted near-threshold decision (parity_util.check_tolerant).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from parity_util import assert_exact, random_blobs, run_both

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-5


def _golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z["coords"], z["weight"], tuple(float(v) for v in z["params"])


@pytest.mark.parametrize("name", ["data_1024", "data_2048", "data_4096", "data_8192", "data_16384",
                                  "data_32768", "blob", "sissa_1000", "toyDetector_1000", "aniso_1000"])
def test_golden_inputs_exact(gpu_context, name):
    c, w, (dc, rhoc, dm) = _golden(name)
    ref, got = run_both(gpu_context, c, w, dc=dc, rhoc=rhoc, dm=dm)
    assert_exact(ref, got)


def test_known_answer_20_clusters(gpu_context):
    # tests/test_device_points.cpp:252-268 of the reference: data_32768 @ (1.3, 10, 1.3) -> 20
    c, w, _ = _golden("data_32768")
    ref, got = run_both(gpu_context, c, w, dc=1.3, rhoc=10.0, dm=1.3)
    assert got.info.n_clusters == 20
    assert int(got.cluster_index.max()) + 1 == 20
    assert_exact(ref, got)


def test_blobs2d_16k_config(gpu_context):
    from cluestering_alpaka3_b200 import synthetic
    wl = synthetic.blobs_2d_16k()
    ref, got = run_both(gpu_context, wl.coords, wl.weight, dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm)
    assert_exact(ref, got)
    assert got.info.n_clusters >= 15


@pytest.mark.parametrize("ndim", list(range(1, 11)))
def test_dimensions_flat(gpu_context, ndim):
    rng = np.random.default_rng(100 + ndim)
    n = 3000
    c, w = random_blobs(rng, n, ndim, nblobs=6, extent=40.0, sigma=1.0)
    dc = 1.0 + 0.35 * ndim
    ref, got = run_both(gpu_context, c, w, dc=dc, rhoc=3.0, dm=1.5 * dc)
    assert_exact(ref, got)


@pytest.mark.parametrize("metric", [("euclidean", ()), ("weighted_euclidean", (0.5, 2.0, 1.0)),
                                    ("manhattan", ()), ("chebyshev", ()),
                                    ("weighted_chebyshev", (1.5, 0.7, 1.0)),
                                    ("periodic_euclidean", (0.0, 0.0, 0.0))])
def test_metrics_flat_3d(gpu_context, metric):
    rng = np.random.default_rng(7)
    c, w = random_blobs(rng, 6000, 3, nblobs=10, extent=60.0)
    ref, got = run_both(gpu_context, c, w, dc=1.7, rhoc=4.0, dm=2.5, metric=metric)
    assert_exact(ref, got)


def _assert_tolerant(ref, got, coords, weight, kw):
    """Exponential / Gaussian kernels: the tolerance rule of parity_util.check_tolerant (rho within
    1e-5 of FP64; nearest highers, seeds and labels exact on the device's own densities; every
    difference from the restatement's own run attributed to a counted near-threshold point)."""
    from parity_util import check_tolerant, oracle_cfg
    cfg = oracle_cfg(**{k: v for k, v in kw.items() if k != "flags"})
    cfg.nthreads = os.cpu_count() or 1
    return check_tolerant(coords, weight, cfg, got, ref=ref, rtol=RTOL)


@pytest.mark.parametrize("flags", [0, 1])
@pytest.mark.parametrize("kernel", [("exp", (1.0, 1.0)), ("gaus", (0.0, 0.5, 1.0)), ("gaus", (1.0, 2.0, 1.5))])
def test_exp_gauss_kernels(gpu_context, kernel, flags):
    # flags 0: spatial summation order (default for these kernels); 1: reference order
    rng = np.random.default_rng(11)
    c, w = random_blobs(rng, 8000, 2, nblobs=12, extent=80.0, sigma=1.2)
    kw = dict(dc=2.0, rhoc=4.0, dm=3.0, kernel=kernel)
    ref, got = run_both(gpu_context, c, w, flags=flags, **kw)
    np.testing.assert_array_equal(got.delta > 0, ref.delta > 0)
    _assert_tolerant(ref, got, c, w, kw)


@pytest.mark.parametrize("ndim", [2, 3, 4])
def test_flat_spatial_order_tolerance(gpu_context, ndim):
    from cluestering_alpaka3_b200 import capi
    rng = np.random.default_rng(40 + ndim)
    c, w = random_blobs(rng, 6000, ndim, nblobs=8, extent=40.0)
    kw = dict(dc=1.5 + 0.3 * ndim, rhoc=3.0, dm=2.0 + 0.3 * ndim, kernel=("flat", (0.5,)))
    ref, got = run_both(gpu_context, c, w, flags=capi.FLAG_SPATIAL_DENSITY, **kw)
    _assert_tolerant(ref, got, c, w, kw)


def test_seed_capacity_policies(gpu_context):
    # seed_dc < dm: seeds with a nearest higher beyond seed_dc exist and can overflow the
    # reference's SeedArray (capacity = #points without nearest higher).
    rng = np.random.default_rng(5)
    c, w = random_blobs(rng, 5000, 2, nblobs=20, extent=50.0, sigma=0.8)
    for cap in (0, -1, 3):
        ref, got = run_both(gpu_context, c, w, dc=0.6, rhoc=2.0, dm=3.0, seed_dc=0.6, seed_capacity=cap)
        assert_exact(ref, got)
    ref0, _ = run_both(gpu_context, c, w, dc=0.6, rhoc=2.0, dm=3.0, seed_dc=0.6, seed_capacity=0)
    assert ref0.stats["dropped_seeds"] >= 0


def test_tiebreak_rho_index(gpu_context):
    rng = np.random.default_rng(9)
    # integer lattice coordinates: many exact distance ties
    c = rng.integers(0, 30, size=(2, 4000)).astype(np.float32)
    w = np.ones(4000, np.float32)
    for tb in ("reference", "rho_index"):
        ref, got = run_both(gpu_context, c, w, dc=1.5, rhoc=2.0, dm=2.5, tiebreak=tb)
        assert ref.stats["nh_distance_ties"] > 0
        assert_exact(ref, got)


def test_wrapped_coordinates(gpu_context):
    rng = np.random.default_rng(13)
    n = 4000
    # an angle-like periodic first coordinate with blobs straddling the wrap point
    ang = np.concatenate([rng.normal(0.0, 0.2, n // 2) % (2 * np.pi), rng.normal(3.0, 0.2, n // 2)])
    rad = rng.normal(5.0, 0.3, n)
    c = np.stack([ang, rad]).astype(np.float32)
    w = np.ones(n, np.float32)
    ref, got = run_both(gpu_context, c, w, dc=0.3, rhoc=3.0, dm=0.5, wrapped=(1, 0),
                        metric=("periodic_euclidean", (2 * np.pi, 0.0)))
    assert_exact(ref, got)


@pytest.mark.parametrize("ppbin", [1, 7, 128, 5000, 100000])
def test_points_per_tile(gpu_context, ppbin):
    rng = np.random.default_rng(17)
    c, w = random_blobs(rng, 3000, 2, nblobs=5, extent=30.0)
    ref, got = run_both(gpu_context, c, w, dc=1.0, rhoc=3.0, dm=1.5, ppbin=ppbin)
    assert_exact(ref, got)


def test_edge_single_point(gpu_context):
    c = np.array([[1.0], [2.0]], np.float32)
    w = np.array([3.0], np.float32)
    ref, got = run_both(gpu_context, c, w, dc=1.0, rhoc=1.0)
    assert_exact(ref, got)
    assert got.cluster_index[0] == 0 and got.is_seed[0] == 1


def test_edge_identical_points(gpu_context):
    c = np.full((2, 700), 4.25, np.float32)
    w = np.ones(700, np.float32)
    ref, got = run_both(gpu_context, c, w, dc=0.5, rhoc=2.0)
    assert_exact(ref, got)


def test_edge_below_threshold(gpu_context):
    rng = np.random.default_rng(3)
    c = rng.uniform(0, 1000, size=(2, 500)).astype(np.float32)
    w = np.ones(500, np.float32)
    ref, got = run_both(gpu_context, c, w, dc=0.5, rhoc=100.0)
    assert_exact(ref, got)
    assert (got.cluster_index == -1).all()


def test_deep_chains_1d(gpu_context):
    # a 1-D density ramp: nearest-higher chains span the whole set (tens of thousands deep)
    n = 40000
    x = np.sqrt(np.linspace(0.0, 1.0, n, dtype=np.float64)).astype(np.float32) * 1000.0
    c = x[None, :].copy()
    w = np.ones(n, np.float32)
    ref, got = run_both(gpu_context, c, w, dc=0.2, rhoc=1.0, dm=0.5)
    assert_exact(ref, got)


def test_negative_and_zero_weights(gpu_context):
    rng = np.random.default_rng(21)
    c, w = random_blobs(rng, 3000, 2, nblobs=4, extent=-40.0)
    w[::7] = 0.0
    w[::11] = -0.5
    ref, got = run_both(gpu_context, c, w, dc=1.2, rhoc=2.0, dm=1.8)
    assert_exact(ref, got)


def test_device_path_and_determinism(gpu_context):
    import torch
    from cluestering_alpaka3_b200 import capi
    from parity_util import gpu_args
    rng = np.random.default_rng(23)
    c, w = random_blobs(rng, 20000, 3, nblobs=10, extent=60.0)
    host = gpu_context.make_clusters_host(c, w, *gpu_args(dc=1.5, rhoc=4.0, dm=2.0))
    dc_ = torch.from_numpy(c).cuda()
    dw = torch.from_numpy(w).cuda()
    outs = {k: torch.empty(c.shape[1], dtype=dt, device="cuda") for k, dt in
            (("cluster_index", torch.int32), ("is_seed", torch.int32), ("rho", torch.float32),
             ("nearest_higher", torch.int32), ("delta", torch.float32))}
    for _ in range(2):
        info = gpu_context.make_clusters_device(dc_.data_ptr(), dw.data_ptr(), 3, c.shape[1],
                                                {k: v.data_ptr() for k, v in outs.items()},
                                                *gpu_args(dc=1.5, rhoc=4.0, dm=2.0))
        np.testing.assert_array_equal(outs["cluster_index"].cpu().numpy(), host.cluster_index)
        np.testing.assert_array_equal(outs["rho"].cpu().numpy().view(np.uint32), host.rho.view(np.uint32))
        np.testing.assert_array_equal(outs["nearest_higher"].cpu().numpy(), host.nearest_higher)
        assert info.n_clusters == host.info.n_clusters
    assert capi is not None


def test_nonfinite_rejected(gpu_context):
    from cluestering_alpaka3_b200 import capi
    from parity_util import gpu_args
    c = np.zeros((2, 100), np.float32)
    c[0, 5] = np.nan
    w = np.ones(100, np.float32)
    with pytest.raises(capi.ClueInvalidArgument):
        gpu_context.make_clusters_host(c, w, *gpu_args(dc=1.0, rhoc=1.0))
    # the context stays usable afterwards
    c[0, 5] = 0.0
    r = gpu_context.make_clusters_host(c, w, *gpu_args(dc=1.0, rhoc=1.0))
    assert r.cluster_index.shape == (100,)


@pytest.mark.parametrize("dim,where", [(2, 0), (0, 300_001), (3, 599_999)])
def test_nonfinite_rejected_large_event(gpu_context, dim, where):
    """Many CTAs reduce one event's box (four points per thread and step, then a remainder):
    a non-finite coordinate or weight anywhere is reported (dim 3: the weight)."""
    from cluestering_alpaka3_b200 import capi
    from parity_util import gpu_args
    rng = np.random.default_rng(7)
    c = rng.uniform(0.0, 100.0, (3, 600_000)).astype(np.float32)
    w = np.ones(600_000, np.float32)
    if dim == 3:
        w[where] = np.nan
    else:
        c[dim, where] = np.inf
    with pytest.raises(capi.ClueInvalidArgument):
        gpu_context.make_clusters_host(c, w, *gpu_args(dc=1.0, rhoc=1.0))


def test_blobs2d_medium_exact(gpu_context):
    from cluestering_alpaka3_b200 import synthetic
    wl = synthetic.blobs_2d_1m(n=1 << 17)
    ref, got = run_both(gpu_context, wl.coords, wl.weight, dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm)
    assert_exact(ref, got)


# ---- symmetric density sweep (Euclidean / Manhattan / Chebyshev, no wrapped coordinate) ----
@pytest.mark.parametrize("metric", [("euclidean", ()), ("manhattan", ()), ("chebyshev", ())])
@pytest.mark.parametrize("kernel", [("exp", (1.0, 1.0)), ("exp", (0.7, 2.0)), ("gaus", (0.0, 0.8, 1.0)),
                                    ("gaus", (0.5, 1.0, 1.3))])
def test_symmetric_density_metrics_kernels(gpu_context, metric, kernel):
    rng = np.random.default_rng(71)
    c, w = random_blobs(rng, 7000, 2, nblobs=10, extent=60.0, sigma=1.0)
    kw = dict(dc=1.8, rhoc=3.0, dm=2.5, kernel=kernel, metric=metric)
    ref, got = run_both(gpu_context, c, w, **kw)
    np.testing.assert_array_equal(got.delta > 0, ref.delta > 0)
    _assert_tolerant(ref, got, c, w, kw)


@pytest.mark.parametrize("ndim", [1, 3, 4])
def test_symmetric_density_dimensions(gpu_context, ndim):
    rng = np.random.default_rng(80 + ndim)
    c, w = random_blobs(rng, 8000, ndim, nblobs=8, extent=30.0, sigma=0.8)
    kw = dict(dc=1.0 + 0.2 * ndim, rhoc=3.0, dm=1.5 + 0.2 * ndim, kernel=("exp", (1.0, 1.0)))
    ref, got = run_both(gpu_context, c, w, **kw)
    _assert_tolerant(ref, got, c, w, kw)


def test_symmetric_density_negative_weights(gpu_context):
    # the mirrored terms are accumulated in fixed point scaled by the event's largest |weight|
    rng = np.random.default_rng(91)
    c, w = random_blobs(rng, 5000, 2, nblobs=6, extent=40.0)
    w = (w - 0.8).astype(np.float32)
    kw = dict(dc=1.5, rhoc=0.5, dm=2.0, kernel=("exp", (1.0, 1.0)))
    ref, got = run_both(gpu_context, c, w, **kw)
    rho64 = O.rho_f64(c, w, O.Config(dc=1.5, rhoc=0.5, dm=2.0, kernel="exp", kernel_par=(1.0, 1.0)))
    scale = np.abs(w).max() * 50
    assert np.max(np.abs(got.rho.astype(np.float64) - rho64)) <= 1e-5 * scale


def test_symmetric_density_deterministic_and_placement_free(gpu_context):
    # an event alone and the same event inside a batch (other events before it) give the same bits
    from parity_util import gpu_args
    rng = np.random.default_rng(95)
    c1, w1 = random_blobs(rng, 3000, 2, nblobs=5, extent=25.0)
    c2, w2 = random_blobs(rng, 4321, 2, nblobs=7, extent=25.0)
    p, k, m = gpu_args(dc=1.5, rhoc=3.0, dm=2.0, kernel=("exp", (1.0, 1.0)))
    alone = gpu_context.make_clusters_host(c2, w2, p, k, m)
    again = gpu_context.make_clusters_host(c2, w2, p, k, m)
    np.testing.assert_array_equal(alone.rho.view(np.uint32), again.rho.view(np.uint32))
    coords = np.ascontiguousarray(np.concatenate([c1, c2], axis=1))
    weight = np.concatenate([w1, w2])
    res, _ = gpu_context.batch_host(coords, weight, [0, c1.shape[1], coords.shape[1]], p, k, m)
    np.testing.assert_array_equal(res.rho[c1.shape[1]:].view(np.uint32), alone.rho.view(np.uint32))
    np.testing.assert_array_equal(res.cluster_index[c1.shape[1]:], alone.cluster_index)


def _nh_on_own_rho(got, c, cfg):
    """The device's nearest higher and delta against the oracle's nearest-higher stage run on
    the device's own densities (bit for bit, ties included)."""
    nh, delta, ties = O.nearest_higher(c, got.rho, cfg)
    keep = got.is_seed == 0
    np.testing.assert_array_equal(got.nearest_higher[keep], nh[keep], err_msg="nearest_higher")
    np.testing.assert_array_equal(got.delta.view(np.uint32), delta.view(np.uint32), err_msg="delta bits")
    return ties


@pytest.mark.parametrize("tiebreak", ["reference", "rho_index"])
@pytest.mark.parametrize("kernel,metric,ndim", [(("exp", (1.0, 1.0)), ("euclidean", ()), 2),
                                                (("gaus", (0.0, 0.8, 1.0)), ("euclidean", ()), 3),
                                                (("exp", (0.7, 2.0)), ("manhattan", ()), 2),
                                                (("gaus", (0.5, 1.0, 1.3)), ("chebyshev", ()), 2)])
def test_symmetric_path_nearest_higher_ties_exact(gpu_context, kernel, metric, ndim, tiebreak):
    # The symmetric density path sorts each tile's points by Morton code, not by index, and
    # ranks equal distances by (search-box position of the tile, original index).  Integer
    # lattice coordinates give many exact distance ties; weights from a few values give equal
    # densities.
    from parity_util import oracle_cfg, gpu_args
    rng = np.random.default_rng(120 + ndim)
    n = 6000
    c = rng.integers(0, 25 if ndim == 2 else 12, size=(ndim, n)).astype(np.float32)
    w = rng.choice(np.array([0.5, 1.0, 1.5], np.float32), size=n)
    kw = dict(dc=1.5, rhoc=2.0, dm=2.5, kernel=kernel, metric=metric, tiebreak=tiebreak)
    got = gpu_context.make_clusters_host(c, w, *gpu_args(**kw))
    ties = _nh_on_own_rho(got, c, oracle_cfg(**kw))
    assert ties > 0


def test_symmetric_path_nearest_higher_batched_exact(gpu_context):
    # the same check per event inside one batched call (events of uneven size)
    from parity_util import oracle_cfg, gpu_args
    rng = np.random.default_rng(133)
    sizes = [1, 40, 700, 3000, 129, 2500]
    cs = [rng.integers(0, 20, size=(2, s)).astype(np.float32) for s in sizes]
    ws = [rng.choice(np.array([0.5, 1.0, 1.5], np.float32), size=s) for s in sizes]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    kw = dict(dc=1.5, rhoc=2.0, dm=2.5, kernel=("exp", (1.0, 1.0)))
    res, _ = gpu_context.batch_host(np.ascontiguousarray(np.concatenate(cs, axis=1)), np.concatenate(ws),
                                    off, *gpu_args(**kw))
    cfg = oracle_cfg(**kw)
    for e, c in enumerate(cs):
        a, b = off[e], off[e + 1]
        nh, delta, _ = O.nearest_higher(c, res.rho[a:b], cfg)
        keep = res.is_seed[a:b] == 0
        got_nh = res.nearest_higher[a:b]  # batch-wide indices
        np.testing.assert_array_equal(np.where(got_nh >= 0, got_nh - a, -1)[keep], nh[keep], err_msg=f"event {e}")
        np.testing.assert_array_equal(res.delta[a:b].view(np.uint32), delta.view(np.uint32), err_msg=f"event {e}")


@pytest.mark.parametrize("n_pad", [100_000, 200_000])
def test_symmetric_event_bits_independent_of_batch_size(gpu_context, n_pad):
    # An event gives the same bits alone and inside batches with ~100k tiles (one composite
    # (tile, Morton) sort) and ~200k tiles (tile sort plus Morton sort): both sort paths order the
    # records by (tile, the same Morton bits, index).  Single-point events pad the tile count.
    from parity_util import gpu_args
    rng = np.random.default_rng(140)
    c, w = random_blobs(rng, 3000, 2, nblobs=5, extent=25.0)
    p, k, m = gpu_args(dc=1.5, rhoc=3.0, dm=2.0, kernel=("exp", (1.0, 1.0)))
    alone = gpu_context.make_clusters_host(c, w, p, k, m)
    pad = rng.uniform(0, 25, size=(2, n_pad)).astype(np.float32)
    coords = np.ascontiguousarray(np.concatenate([pad, c], axis=1))
    weight = np.concatenate([np.ones(n_pad, np.float32), w])
    off = np.concatenate([np.arange(n_pad + 1), [n_pad + c.shape[1]]]).astype(np.int32)
    res, _ = gpu_context.batch_host(coords, weight, off, p, k, m)
    assert res.info.n_tiles > (1 << 16)
    for name in ("rho", "delta", "cluster_index", "is_seed"):
        np.testing.assert_array_equal(getattr(res, name)[n_pad:].view(np.uint32), getattr(alone, name).view(np.uint32),
                                      err_msg=name)
    nh = res.nearest_higher[n_pad:]
    np.testing.assert_array_equal(np.where(nh >= 0, nh - n_pad, -1), alone.nearest_higher)


# ---- labels by follower CSR + breadth-first walk (clue_tuning.labels_bfs) -----------------------
@pytest.mark.parametrize("case", ["blobs", "deep_chains", "seed_capacity"])
def test_labels_bfs_equal_pointer_jumping(case):
    # The breadth-first form (the reference's follower association map and a walk from the seeds,
    # level by level) gives the same labels as pointer jumping: bit for bit against the oracle,
    # also past the enqueued levels (a 1-D ramp whose chains are tens of thousands deep) and with
    # seeds dropped by the reference's seed-list capacity.
    from cluestering_alpaka3_b200 import capi
    from parity_util import gpu_args, oracle_cfg
    rng = np.random.default_rng(300)
    if case == "blobs":
        c, w = random_blobs(rng, 20000, 2, nblobs=12, extent=60.0)
        kw = dict(dc=1.2, rhoc=4.0, dm=1.8)
    elif case == "deep_chains":
        n = 30000
        c = (np.sqrt(np.linspace(0.0, 1.0, n)) * 800.0).astype(np.float32)[None, :].copy()
        w = np.ones(n, np.float32)
        kw = dict(dc=0.2, rhoc=1.0, dm=0.5)
    else:
        c, w = random_blobs(rng, 5000, 2, nblobs=20, extent=50.0, sigma=0.8)
        kw = dict(dc=0.6, rhoc=2.0, dm=3.0, seed_dc=0.6, seed_capacity=0)
    ctx = capi.Context(0)
    try:
        ctx.set_tuning(labels_bfs=1)
        got = ctx.make_clusters_host(c, w, *gpu_args(**kw))
    finally:
        ctx.close()
    ref = O.run(c, w, oracle_cfg(**kw))
    assert_exact(ref, got)
