"""Serving: the continuous-batching request loop (clue_server_*).  Results in a mix of
concurrent requests must equal each event clustered alone (flat kernel: bit for bit), admission
respects the device budget and the per-event limit, and the load replay reports latencies."""
import numpy as np
import pytest

from parity_util import gpu_args


def params_4d():
    from cluestering_alpaka3_b200 import capi
    return capi.Params(dc=2.5, rhoc=6.0, dm=2.5), capi.FlatKernel(0.5)


# ---- host-only: validation before anything touches a GPU ------------------------------------
@pytest.mark.parametrize("field,value", [("ndim", 0), ("ndim", 11), ("n_slots", 0), ("n_slots", 17),
                                         ("max_batch_events", 0), ("max_event_points", 0), ("max_pending", 0),
                                         ("device_budget_bytes", 0)])
def test_server_config_validation(field, value):
    from cluestering_alpaka3_b200 import capi
    cfg = capi.ServerConfig(ndim=4)
    setattr(cfg, field, value)
    with pytest.raises(capi.ClueInvalidArgument):
        capi.Server(cfg, *params_4d())


def test_server_budget_too_small():
    from cluestering_alpaka3_b200 import capi
    cfg = capi.ServerConfig(ndim=4, n_slots=2, max_event_points=200000, device_budget_bytes=64 << 20)
    with pytest.raises(capi.ClueError) as e:
        capi.Server(cfg, *params_4d())
    assert e.value.status == capi.ERR_CAPACITY


def test_server_bad_params():
    from cluestering_alpaka3_b200 import capi
    with pytest.raises(capi.ClueInvalidArgument):
        capi.Server(capi.ServerConfig(ndim=2), capi.Params(dc=-1.0, rhoc=1.0), capi.FlatKernel(0.5))


# ---- GPU ------------------------------------------------------------------------------------
def alone(ctx, coords, weight):
    p, k, m = gpu_args(dc=2.5, rhoc=6.0, dm=2.5)
    return ctx.make_clusters_host(coords, weight, p, k, m)


def assert_same(res, ref, what):
    np.testing.assert_array_equal(res["cluster_index"], ref.cluster_index, err_msg=what)
    np.testing.assert_array_equal(res["is_seed"], ref.is_seed, err_msg=what)
    np.testing.assert_array_equal(res["nearest_higher"], ref.nearest_higher, err_msg=what)
    np.testing.assert_array_equal(res["rho"].view(np.uint32), ref.rho.view(np.uint32), err_msg=what)
    np.testing.assert_array_equal(res["delta"].view(np.uint32), ref.delta.view(np.uint32), err_msg=what)


@pytest.mark.gpu
def test_server_mix_equals_alone(gpu_context):
    from cluestering_alpaka3_b200 import capi, synthetic
    coords, weight, off, _ = synthetic.serving_events(160, seed=77, hi=30000)
    srv = capi.Server(capi.ServerConfig(ndim=4, n_slots=3, max_batch_events=64, max_event_points=30000,
                                        device_budget_bytes=2 << 30), *params_4d())
    try:
        tickets = [srv.submit(coords[:, off[e]:off[e + 1]], weight[off[e]:off[e + 1]]) for e in range(len(off) - 1)]
        results = [srv.wait(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    assert st["completed"] == len(tickets) and st["failed"] == 0
    assert st["batches"] < len(tickets), st       # events shared batches
    assert st["max_batch_seen"] > 1
    for e, r in enumerate(results):
        a, b = off[e], off[e + 1]
        ref = alone(gpu_context, np.ascontiguousarray(coords[:, a:b]), weight[a:b])
        assert_same({k: getattr(r, k) for k in ("cluster_index", "is_seed", "nearest_higher", "rho", "delta")},
                    ref, f"event {e}")
        assert r.info["n_clusters"] == ref.info.n_clusters
        assert r.info["done_s"] >= r.info["start_s"] >= r.info["submit_s"]


@pytest.mark.gpu
def test_server_replay_poisson(gpu_context):
    from cluestering_alpaka3_b200 import capi, synthetic
    coords, weight, off, _ = synthetic.serving_events(300, seed=78, hi=50000)
    arrivals = synthetic.poisson_arrivals(3000.0, len(off) - 1, seed=1)
    srv = capi.Server(capi.ServerConfig(ndim=4, n_slots=2, max_batch_events=256, max_event_points=50000,
                                        device_budget_bytes=2 << 30), *params_4d())
    try:
        res, lat, rej = srv.replay(coords, weight, off, arrivals)
        st = srv.stats()
    finally:
        srv.close()
    assert rej == 0 and np.all(lat > 0), (rej, lat.min())
    assert st["completed"] == len(off) - 1
    for e in range(0, len(off) - 1, 7):
        a, b = off[e], off[e + 1]
        ref = alone(gpu_context, np.ascontiguousarray(coords[:, a:b]), weight[a:b])
        assert_same({k: v[a:b] for k, v in res.items()}, ref, f"event {e}")  # nearest_higher is event-local


@pytest.mark.gpu
def test_server_refusals(gpu_context):
    from cluestering_alpaka3_b200 import capi, synthetic
    coords, weight, off, _ = synthetic.serving_events(3, seed=79, lo=3000, hi=3000)
    srv = capi.Server(capi.ServerConfig(ndim=4, n_slots=1, max_batch_events=4, max_event_points=2000,
                                        device_budget_bytes=1 << 30), *params_4d())
    try:
        with pytest.raises(capi.ClueError) as e:
            srv.submit(coords[:, :3000], weight[:3000])      # larger than max_event_points
        assert e.value.status == capi.ERR_CAPACITY
        bad = np.array(coords[:, :100])
        bad[1, 7] = np.inf
        with pytest.raises(capi.ClueError) as e:
            srv.submit(bad, weight[:100])
        assert e.value.status == capi.ERR_NONFINITE
        t = srv.submit(coords[:, :1500], weight[:1500])
        r = srv.wait(t)
        ref = alone(gpu_context, np.ascontiguousarray(coords[:, :1500]), weight[:1500])
        np.testing.assert_array_equal(r.cluster_index, ref.cluster_index)
        assert srv.stats()["rejected"] == 1
        # pooled replay without outputs (several requests of one event)
        ids = np.array([0, 1, 0, 2, 1, 0], np.int32)
        small_off = np.array([0, 500, 1200, 2000], np.int32)
        _, lat, rej = srv.replay(coords[:, :2000], weight[:2000], small_off, np.linspace(0, 0.01, 6), event_ids=ids,
                                 outputs=False)
        assert rej == 0 and np.all(lat > 0)
    finally:
        srv.close()
