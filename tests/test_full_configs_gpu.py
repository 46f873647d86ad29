"""Parity at the benchmark configurations' full sizes, against the restatement of the
reference's serial path.

- blobs2d_1m: 1,048,576 2-D points, FlatKernel(0.5): every output bit-exact.
- blobs3d_4m: 4,194,304 3-D points, GaussianKernel(0, 0.5, 1): the tolerance rule of
  parity_util.check_tolerant.
- calo4096: the 4096-event batch that bench.py times (13.3M points, same generator and seed),
  through the captured CUDA graph that bench.py replays, every event against the restatement
  run on that event alone: the tolerance rule, with the device's near-threshold counts checked
  against the same tests on its outputs.
The restatement runs on all host cores (OpenMP over points, or over events for the batch).
"""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from oracle import oracle as O
from parity_util import assert_exact, check_tolerant, gpu_args, run_both

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def test_blobs2d_1m_full_exact(gpu_context):
    from cluestering_alpaka3_b200 import synthetic
    wl = synthetic.blobs_2d_1m()
    cfg = O.Config(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm, nthreads=THREADS)
    ref = O.run(wl.coords, wl.weight, cfg)
    got = gpu_context.make_clusters_host(wl.coords, wl.weight, *gpu_args(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm))
    assert_exact(ref, got)
    print(f"blobs2d_1m: {got.info.n_clusters} clusters, bit-exact")


def test_blobs3d_4m_full_tolerance(gpu_context):
    from cluestering_alpaka3_b200 import synthetic
    wl = synthetic.blobs_3d_4m()
    kw = dict(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm, kernel=wl.kernel)
    got = gpu_context.make_clusters_host(wl.coords, wl.weight, *gpu_args(**kw))
    counts = gpu_context.near_counts()
    cfg = O.Config(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm, kernel=wl.kernel[0], kernel_par=wl.kernel[1], nthreads=THREADS)
    ref = O.run(wl.coords, wl.weight, cfg)
    rep = check_tolerant(wl.coords, wl.weight, cfg, got, ref=ref, near_counts=counts, tag="blobs3d_4m")
    print("device near-threshold counts", counts)
    assert rep["max_rel_rho_vs_f64"] <= 1e-5


def test_calo4096_graph_full_tolerance(gpu_context):
    import torch
    from cluestering_alpaka3_b200 import capi, synthetic
    evs, p = synthetic.calo_events(4096, seed=4000)
    off = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in evs])]).astype(np.int32)
    coords = np.ascontiguousarray(np.concatenate([e[0] for e in evs], axis=1))
    weight = np.ascontiguousarray(np.concatenate([e[1] for e in evs]))
    n = coords.shape[1]
    params, kernel, metric = gpu_args(dc=p["dc"], rhoc=p["rhoc"], dm=p["dm"], kernel=p["kernel"])
    dc_ = torch.from_numpy(coords).cuda()
    dw = torch.from_numpy(weight).cuda()
    outs = {k: torch.full((n,), -7, dtype=dt, device="cuda") for k, dt in
            (("cluster_index", torch.int32), ("is_seed", torch.int32), ("rho", torch.float32),
             ("nearest_higher", torch.int32), ("delta", torch.float32))}
    ncl = torch.zeros(len(evs), dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    graph = gpu_context.capture_batch(dc_.data_ptr(), dw.data_ptr(), 2, off, {k: v.data_ptr() for k, v in outs.items()},
                                      params, kernel, metric, ncl_ptr=ncl.data_ptr(), stream=sp)
    try:
        graph.launch(sp)
        graph.launch(sp)  # a second replay over the same buffers gives the same result
        stream.synchronize()
        counts = gpu_context.near_counts(sp)
        got = SimpleNamespace(**{k: v.cpu().numpy() for k, v in outs.items()})
    finally:
        graph.close()
    cfg = O.Config(dc=p["dc"], rhoc=p["rhoc"], dm=p["dm"], kernel=p["kernel"][0], kernel_par=p["kernel"][1],
                   nthreads=THREADS)
    ref = O.run_events(coords, weight, off, cfg)
    rep = check_tolerant(coords, weight, cfg, got, offsets=off, ref=ref, near_counts=counts, tag="calo4096")
    print("device near-threshold counts", counts)
    # clusters per event, as the graph reported them, against the seed lists of the device forest
    ev_ncl = ncl.cpu().numpy()
    for e in range(0, len(evs), 97):
        a, b = off[e], off[e + 1]
        assert ev_ncl[e] == int(got.cluster_index[a:b].max(initial=-1)) + 1
    assert rep["events"] == 4096


def test_calo_near_tie_count_covers_decision_differences(gpu_context):
    # CLUE_FLAG_NEAR_TIES: the device counts the points whose nearest-higher choice compares
    # densities within the tolerance; every nearest-higher difference from the restatement is
    # such a point, so the count bounds the differences
    from cluestering_alpaka3_b200 import capi, synthetic
    evs, p = synthetic.calo_events(256, seed=4100)
    off = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in evs])]).astype(np.int32)
    coords = np.ascontiguousarray(np.concatenate([e[0] for e in evs], axis=1))
    weight = np.ascontiguousarray(np.concatenate([e[1] for e in evs]))
    kw = dict(dc=p["dc"], rhoc=p["rhoc"], dm=p["dm"], kernel=p["kernel"])
    plain, _ = gpu_context.batch_host(coords, weight, off, *gpu_args(**kw))
    flagged, _ = gpu_context.batch_host(coords, weight, off, *gpu_args(flags=capi.FLAG_NEAR_TIES, **kw))
    counts = gpu_context.near_counts()
    for name in ("cluster_index", "is_seed", "rho", "nearest_higher", "delta"):  # the count changes nothing
        np.testing.assert_array_equal(getattr(flagged, name).view(np.uint32), getattr(plain, name).view(np.uint32))
    assert counts["nh_near_ties"] >= 0
    cfg = O.Config(dc=p["dc"], rhoc=p["rhoc"], dm=p["dm"], kernel=p["kernel"][0], kernel_par=p["kernel"][1],
                   nthreads=THREADS)
    ref = O.run_events(coords, weight, off, cfg)
    nh_diff = int(((plain.nearest_higher != ref.nearest_higher) & (plain.is_seed == ref.is_seed)).sum())
    print("near-tie points", counts["nh_near_ties"], "nearest-higher differences", nh_diff)
    assert nh_diff <= counts["nh_near_ties"]
