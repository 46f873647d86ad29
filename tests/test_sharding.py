"""Event sharding host logic: balanced, deterministic partitions and a world_size-2 gloo run in
which each rank clusters its own events (the oracle stands in for the per-rank GPU call) and
rank 0 gathers every event exactly once, equal to a single-process run."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cluestering_alpaka3_b200.sharding import gather_event_results, partition_events


def test_partition_balanced_and_complete():
    rng = np.random.default_rng(0)
    sizes = np.clip(np.round(rng.lognormal(np.log(2000), 1.0, 4096)), 100, 60000).astype(np.int64)
    for world in (1, 2, 3, 8):
        parts = partition_events(sizes, world)
        allids = np.sort(np.concatenate(parts))
        np.testing.assert_array_equal(allids, np.arange(sizes.size))
        loads = np.array([sizes[p].sum() for p in parts])
        assert loads.max() - loads.min() <= sizes.max()
        assert all(np.all(np.diff(p) > 0) for p in parts)
        again = partition_events(sizes, world)
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))
    with pytest.raises(ValueError):
        partition_events(sizes, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from oracle import oracle as O
    from parity_util import random_blobs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(9)
        events = [random_blobs(rng, int(n), 2, nblobs=3, extent=30.0) for n in rng.integers(200, 1500, 12)]
        sizes = [e[0].shape[1] for e in events]
        mine = partition_events(sizes, world)[rank]
        local = {int(e): O.run(*events[e], O.Config(dc=1.0, rhoc=3.0)).cluster_index for e in mine}
        merged = gather_event_results(local, world, rank)
        if rank == 0:
            q.put({k: v.tolist() for k, v in merged.items()})
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_gather_every_event_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from oracle import oracle as O
    from parity_util import random_blobs
    rng = np.random.default_rng(9)
    events = [random_blobs(rng, int(n), 2, nblobs=3, extent=30.0) for n in rng.integers(200, 1500, 12)]
    assert sorted(got) == list(range(len(events)))
    for e, (c, w) in enumerate(events):
        np.testing.assert_array_equal(np.array(got[e]), O.run(c, w, O.Config(dc=1.0, rhoc=3.0)).cluster_index)
