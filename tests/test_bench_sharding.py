"""bench.py's multi-GPU path on CPU: under torchrun every rank takes its share of the job's
events (bench.rank_share over bench.make_workload), clusters them, and rank 0 gathers the
per-event cluster counts and prints the checksum of block 0's events.  Here two gloo ranks run
that path with the restatement standing in for each rank's GPU, on a shortened workload (64
events per rank instead of 4096), and the checksum must equal the single-rank run's."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

EVENTS = 64


def _per_event_clusters(wl):
    from oracle import oracle as O
    kname, kpar = wl.kernel
    cfg = O.Config(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm, kernel=kname, kernel_par=kpar, nthreads=2)
    res = O.run_events(wl.coords, wl.weight, wl.offsets, cfg)
    return {int(i): int(c) for i, c in zip(wl.ids, res.stats["ev_n_clusters"])}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    import bench
    from cluestering_alpaka3_b200.sharding import gather_event_results
    bench.EVENTS_PER_GPU = EVENTS
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        wl_all = bench.make_workload("calo4096", world)
        mine = bench.rank_share(wl_all, world, rank)
        merged = gather_event_results(_per_event_clusters(mine), world, rank)
        if rank == 0:
            q.put({"checksum": bench.events_checksum(merged), "events": sorted(merged),
                   "config": bench.workload_config(wl_all, world), "points": int(mine.coords.shape[1]),
                   "total_points": int(wl_all.coords.shape[1])})
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_events_and_match_one_rank():
    import bench
    bench.EVENTS_PER_GPU = EVENTS
    try:
        one = bench.make_workload("calo4096", 1)
        single = bench.events_checksum(_per_event_clusters(one))
    finally:
        bench.EVENTS_PER_GPU = 4096
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got["events"] == list(range(2 * EVENTS))  # every event of both blocks, once
    assert got["checksum"] == single  # block 0 clusters the same on one rank and on two
    assert got["config"]["parallelism"] == "events sharded over 2 ranks"
    assert got["config"]["n_events"] == 2 * EVENTS
    assert 0 < got["points"] < got["total_points"]
