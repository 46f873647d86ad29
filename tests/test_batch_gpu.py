"""Batched events: one pass over many events equals clustering every event alone.

Each event is checked against the CPU oracle run on that event alone (bit for bit for the
flat kernel; by the tolerance rule of parity_util.check_tolerant for the exponential kernel), and the CUDA-graph replay of the
batched pipeline is checked against the direct call.
"""
import numpy as np
import pytest

from oracle import oracle as O
from parity_util import gpu_args

pytestmark = pytest.mark.gpu


def make_events(seed, n_events, ndim=2, lo=100, hi=4000):
    from cluestering_alpaka3_b200 import synthetic
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.round(rng.lognormal(np.log(800), 1.0, size=n_events)), lo, hi).astype(int)
    evs = []
    for s in sizes:
        if ndim == 2:
            evs.append(synthetic.calo_event(rng, int(s)))
        else:
            evs.append(synthetic.blobs_4d_event(rng, int(s)) if ndim == 4 else
                       (rng.normal(0, 3, size=(ndim, int(s))).astype(np.float32),
                        rng.uniform(0.5, 1.5, int(s)).astype(np.float32)))
    off = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in evs])]).astype(np.int32)
    coords = np.ascontiguousarray(np.concatenate([e[0] for e in evs], axis=1))
    weight = np.concatenate([e[1] for e in evs])
    return evs, off, coords, weight


@pytest.mark.parametrize("ndim,kernel,params", [
    (2, ("flat", (0.5,)), dict(dc=2.0, rhoc=4.0, dm=3.0)),
    (4, ("flat", (0.5,)), dict(dc=2.5, rhoc=6.0, dm=2.5)),
    (3, ("flat", (0.5,)), dict(dc=1.5, rhoc=2.0, dm=2.0, seed_dc=1.0)),
])
def test_batch_equals_events_alone_exact(gpu_context, ndim, kernel, params):
    evs, off, coords, weight = make_events(31 + ndim, 40, ndim=ndim)
    p, k, m = gpu_args(kernel=kernel, **params)
    res, ncl = gpu_context.batch_host(coords, weight, off, p, k, m)
    tot = 0
    for e, (c, w) in enumerate(evs):
        a, b = off[e], off[e + 1]
        ref = O.run(c, w, O.Config(dc=params["dc"], rhoc=params["rhoc"], dm=params["dm"],
                                   seed_dc=params.get("seed_dc"), kernel=kernel[0], kernel_par=kernel[1]))
        np.testing.assert_array_equal(res.cluster_index[a:b], ref.cluster_index, err_msg=f"event {e}")
        np.testing.assert_array_equal(res.is_seed[a:b], ref.is_seed)
        np.testing.assert_array_equal(res.rho[a:b].view(np.uint32), ref.rho.view(np.uint32))
        nh = res.nearest_higher[a:b]
        np.testing.assert_array_equal(np.where(nh >= 0, nh - a, -1), ref.nearest_higher)
        assert ncl[e] == ref.stats["n_clusters"]
        tot += ref.stats["n_clusters"]
    assert res.info.n_clusters == tot


def test_batch_exponential_kernel_tolerance(gpu_context):
    import os
    from parity_util import check_tolerant
    evs, off, coords, weight = make_events(7, 30)
    kw = dict(dc=2.0, rhoc=4.0, dm=3.0, kernel=("exp", (1.0, 1.0)))
    res, ncl = gpu_context.batch_host(coords, weight, off, *gpu_args(**kw))
    cfg = O.Config(dc=2.0, rhoc=4.0, dm=3.0, kernel="exp", kernel_par=(1.0, 1.0), nthreads=os.cpu_count() or 1)
    rep = check_tolerant(coords, weight, cfg, res, offsets=off, tag="30 events")
    assert rep["events"] == 30


def test_single_event_batch_equals_plain(gpu_context):
    from cluestering_alpaka3_b200 import synthetic
    wl = synthetic.blobs_2d_16k(n=10000)
    p, k, m = gpu_args(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm)
    plain = gpu_context.make_clusters_host(wl.coords, wl.weight, p, k, m)
    res, ncl = gpu_context.batch_host(wl.coords, wl.weight, [0, wl.coords.shape[1]], p, k, m)
    np.testing.assert_array_equal(res.cluster_index, plain.cluster_index)
    np.testing.assert_array_equal(res.rho.view(np.uint32), plain.rho.view(np.uint32))
    assert ncl[0] == plain.info.n_clusters


def test_graph_replay_matches_direct(gpu_context):
    import torch
    evs, off, coords, weight = make_events(99, 64)
    n = coords.shape[1]
    p, k, m = gpu_args(dc=2.0, rhoc=4.0, dm=3.0)
    direct, ncl = gpu_context.batch_host(coords, weight, off, p, k, m)
    dc_ = torch.from_numpy(coords).cuda()
    dw = torch.from_numpy(weight).cuda()
    outs = {k_: torch.full((n,), -9, dtype=torch.int32, device="cuda") for k_ in ("cluster_index", "is_seed")}
    ncl_d = torch.zeros(len(off) - 1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    g = gpu_context.capture_batch(dc_.data_ptr(), dw.data_ptr(), 2, off, {k_: v.data_ptr() for k_, v in outs.items()},
                                  p, k, m, ncl_ptr=ncl_d.data_ptr(), stream=stream.cuda_stream)
    for _ in range(3):
        outs["cluster_index"].fill_(-9)
        torch.cuda.synchronize()
        g.launch(stream.cuda_stream)
        stream.synchronize()
        np.testing.assert_array_equal(outs["cluster_index"].cpu().numpy(), direct.cluster_index)
        np.testing.assert_array_equal(outs["is_seed"].cpu().numpy(), direct.is_seed)
        np.testing.assert_array_equal(ncl_d.cpu().numpy(), ncl)
    g.close()


def test_events_loop_matches_batch(gpu_context):
    import torch
    evs, off, coords, weight = make_events(5, 48)
    n = coords.shape[1]
    p, k, m = gpu_args(dc=2.0, rhoc=4.0, dm=3.0, kernel=("exp", (1.0, 1.0)))
    direct, ncl = gpu_context.batch_host(coords, weight, off, p, k, m)
    dc_ = torch.from_numpy(coords).cuda()
    dw = torch.from_numpy(weight).cuda()
    outs = {"cluster_index": torch.full((n,), -9, dtype=torch.int32, device="cuda"),
            "rho": torch.zeros(n, dtype=torch.float32, device="cuda")}
    ms = gpu_context.events_loop(dc_.data_ptr(), dw.data_ptr(), 2, off, {k_: v.data_ptr() for k_, v in outs.items()},
                                 p, k, m, event_times=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(outs["cluster_index"].cpu().numpy(), direct.cluster_index)
    np.testing.assert_array_equal(outs["rho"].cpu().numpy().view(np.uint32), direct.rho.view(np.uint32))
    assert ms.shape == (len(off) - 1,) and (ms > 0).all()


@pytest.mark.parametrize("kernel,params", [
    (("exp", (1.0, 1.0)), dict(dc=2.0, rhoc=4.0, dm=3.0)),
    (("flat", (0.5,)), dict(dc=2.0, rhoc=4.0, dm=3.0, tiebreak="rho_index")),
])
def test_host_batch_overlapped_equals_device_batch(gpu_context, kernel, params):
    # A host-memory batch of 4M points or more is cut into chunks of whole events whose copies
    # overlap the pipeline; every output (nearest-higher indices shifted to the batch, per-event
    # cluster counts, run totals) equals one device-memory pass over the whole batch.
    import torch
    evs, off, coords, weight = make_events(77, 3300, lo=200, hi=20000)
    n = coords.shape[1]
    assert n >= 4_000_000
    p, k, m = gpu_args(kernel=kernel, **params)
    res, ncl = gpu_context.batch_host(coords, weight, off, p, k, m)
    dc = torch.from_numpy(coords).cuda()
    dw = torch.from_numpy(weight).cuda()
    outs = {"cluster_index": torch.empty(n, dtype=torch.int32, device="cuda"),
            "is_seed": torch.empty(n, dtype=torch.int32, device="cuda"),
            "rho": torch.empty(n, dtype=torch.float32, device="cuda"),
            "nearest_higher": torch.empty(n, dtype=torch.int32, device="cuda"),
            "delta": torch.empty(n, dtype=torch.float32, device="cuda")}
    dncl = torch.empty(len(off) - 1, dtype=torch.int32, device="cuda")
    info = gpu_context.batch_device(dc.data_ptr(), dw.data_ptr(), 2, off, {k_: v.data_ptr() for k_, v in outs.items()},
                                    p, k, m, ncl_ptr=dncl.data_ptr())
    for name, t in outs.items():
        np.testing.assert_array_equal(getattr(res, name).view(np.uint32), t.cpu().numpy().view(np.uint32),
                                      err_msg=name)
    np.testing.assert_array_equal(ncl, dncl.cpu().numpy())
    assert res.info.n_seeds == info.n_seeds
    assert res.info.n_clusters == info.n_clusters
    assert res.info.dropped_seeds == info.dropped_seeds
    assert res.info.n_tiles == info.n_tiles
    assert res.info.seed_capacity_used == info.seed_capacity_used
    # and a second call on the same context gives the same result
    res2, ncl2 = gpu_context.batch_host(coords, weight, off, p, k, m)
    np.testing.assert_array_equal(res2.cluster_index, res.cluster_index)
    np.testing.assert_array_equal(res2.nearest_higher, res.nearest_higher)


def test_autotune_batch_cache_and_equivalence(tmp_path):
    # The autotuner times the runtime choices on a device batch, keeps the fastest and caches it
    # per (ndim, size bucket, event-count bucket, kernel, metric, flags); every choice gives the
    # same outputs (the nearest-higher split and the copy overlap exactly, the density form
    # within the 1e-5 tolerance).
    import torch
    from cluestering_alpaka3_b200 import capi
    evs, off, coords, weight = make_events(55, 300)
    p, k, m = gpu_args(kernel=("exp", (1.0, 1.0)), dc=2.0, rhoc=4.0, dm=3.0)
    dc, dw = torch.from_numpy(coords).cuda(), torch.from_numpy(weight).cuda()
    cache = tmp_path / "clue_tune.txt"
    tuned = capi.Context(0)
    chosen = tuned.autotune_batch(dc.data_ptr(), dw.data_ptr(), 2, off, p, k, m, cache_path=str(cache))
    assert chosen["symmetric_density"] in (0, 1) and chosen["nh_split_lanes"] in (0, 4, 8, 16)
    assert tuned.tuning() == chosen
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and "ndim=2" in lines[0] and "nh_split_lanes=" in lines[0]
    other = capi.Context(0)
    assert other.autotune_batch(dc.data_ptr(), dw.data_ptr(), 2, off, p, k, m, cache_path=str(cache)) == chosen
    assert cache.read_text().splitlines() == lines  # read from the cache, nothing timed or added

    base = capi.Context(0)
    ref, ref_ncl = base.batch_host(coords, weight, off, p, k, m)
    for split in (0, 4, 16):
        base.set_tuning(nh_split_lanes=split)
        got, ncl = base.batch_host(coords, weight, off, p, k, m)
        for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):
            np.testing.assert_array_equal(getattr(got, name).view(np.uint32), getattr(ref, name).view(np.uint32),
                                          err_msg=f"split {split}: {name}")
        np.testing.assert_array_equal(ncl, ref_ncl)
    base.set_tuning(nh_split_lanes=8, density_gate=1)  # the vote-gated pair steps skip only zero terms
    gated, _ = base.batch_host(coords, weight, off, p, k, m)
    for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):
        np.testing.assert_array_equal(getattr(gated, name).view(np.uint32), getattr(ref, name).view(np.uint32),
                                      err_msg=f"gated: {name}")
    import os
    from parity_util import check_tolerant
    cfg = O.Config(dc=2.0, rhoc=4.0, dm=3.0, kernel="exp", kernel_par=(1.0, 1.0), nthreads=os.cpu_count() or 1)
    for gate in (0, 1):  # 2^x on the FMA pipe: the tolerance rule
        base.set_tuning(density_gate=gate, density_exp2=1)
        poly, _ = base.batch_host(coords, weight, off, p, k, m)
        check_tolerant(coords, weight, cfg, poly, offsets=off, tag=f"exp2 on the FMA pipe, gate {gate}")
    base.set_tuning(nh_split_lanes=8, symmetric_density=0, density_gate=0, density_exp2=0)
    one_sided, _ = base.batch_host(coords, weight, off, p, k, m)
    np.testing.assert_allclose(one_sided.rho, ref.rho, rtol=2e-5)
    with pytest.raises(capi.ClueError):
        base.set_tuning(nh_split_lanes=17)
    with pytest.raises(capi.ClueError):
        base.set_tuning(symmetric_density=2)
    with pytest.raises(capi.ClueError):
        base.set_tuning(density_exp2=3)
    base.reset_tuning()
    assert base.tuning() == {"symmetric_density": 1, "nh_split_lanes": 8, "overlap_chunk_points": 2200000,
                             "density_gate": 0, "density_exp2": 0, "labels_bfs": 0, "reserved": 0}
    for c in (tuned, other, base):
        c.close()


@pytest.mark.parametrize("host", [False, True])
def test_batch_nonfinite_rejected(gpu_context, host):
    # A non-finite coordinate inside an event's span and a non-finite weight at the batch's
    # last point are reported, by the device-memory batch and by the overlapped host batch
    # (4M points or more, in chunks); the context stays usable afterwards.
    import torch
    from cluestering_alpaka3_b200 import capi
    evs, off, coords, weight = make_events(91, 3300 if host else 400, lo=200, hi=20000 if host else 4000)
    n = coords.shape[1]
    assert not host or n >= 4_000_000  # the overlapped path
    p, k, m = gpu_args(kernel=("flat", (0.5,)), dc=2.0, rhoc=4.0, dm=3.0)
    e = len(off) // 2
    for bad in ("coord", "weight"):
        c, w = coords.copy(), weight.copy()
        if bad == "coord":
            c[1, (off[e] + off[e + 1]) // 2] = np.nan
        else:
            w[n - 1] = np.inf
        with pytest.raises(capi.ClueInvalidArgument):
            if host:
                gpu_context.batch_host(c, w, off, p, k, m)
            else:
                dc_, dw_ = torch.from_numpy(c).cuda(), torch.from_numpy(w).cuda()
                lab = torch.empty(n, dtype=torch.int32, device="cuda")
                gpu_context.batch_device(dc_.data_ptr(), dw_.data_ptr(), 2, off, {"cluster_index": lab.data_ptr()},
                                         p, k, m)
    res, _ = gpu_context.batch_host(coords[:, :off[3]].copy(), weight[:off[3]].copy(), off[:4], p, k, m)
    assert res.cluster_index.shape == (int(off[3]),)
