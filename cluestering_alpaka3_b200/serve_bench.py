"""Serving sweep: a Poisson stream of 4-D events through the continuous-batching server.

    python -m cluestering_alpaka3_b200.serve_bench --rates 1000,2000,5000,10000,20000,50000 --seconds 10

For every offered load (events/s) the native replay thread submits events at Poisson arrival
times drawn from a pool of pre-generated events (sizes lognormal, median 2000, sigma 1,
clipped to [100, 200000]; 5-50 blobs of sigma 1 in [0,100]^4 plus 10% noise; dc=2.5, rhoc=6,
dm=2.5, FlatKernel(0.5)).  Latency is completion minus scheduled arrival.  One JSON line per
rate: p50/p99/mean latency, achieved events/s and points/s, batches, refusals.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def make_pool(n_pool: int, seed: int = 5000):
    from . import synthetic
    return synthetic.serving_events(n_pool, seed=seed)


def run_rate(srv, coords, weight, off, rate: float, seconds: float, seed: int) -> dict:
    from . import synthetic
    n = max(1, int(round(rate * seconds)))
    rng = np.random.default_rng(seed)
    ids = rng.integers(0, len(off) - 1, size=n).astype(np.int32)
    arrivals = synthetic.poisson_arrivals(rate, n, seed=seed + 1)
    before = srv.stats()
    t0 = time.perf_counter()
    _, lat, rej = srv.replay(coords, weight, off, arrivals, event_ids=ids, outputs=False)
    wall = time.perf_counter() - t0
    after = srv.stats()
    ok = lat >= 0
    sizes = (off[ids + 1] - off[ids]).astype(np.int64)
    span = float(np.max(arrivals[ok] + lat[ok])) if ok.any() else wall
    batches = after["batches"] - before["batches"]
    return {
        "offered_events_per_s": rate,
        "events": int(n),
        "refused": int(rej),
        "p50_ms": float(np.percentile(lat[ok], 50) * 1e3) if ok.any() else None,
        "p99_ms": float(np.percentile(lat[ok], 99) * 1e3) if ok.any() else None,
        "mean_ms": float(lat[ok].mean() * 1e3) if ok.any() else None,
        "achieved_events_per_s": float(ok.sum() / span),
        "points_per_s": float(sizes[ok].sum() / span),
        "mean_event_points": float(sizes.mean()),
        "batches": int(batches),
        "events_per_batch": float(ok.sum() / max(batches, 1)),
        "max_in_flight": int(after["max_in_flight"]),
        "wall_s": wall,
    }


def make_server(ndim: int = 4, slots: int = 3, budget_gb: float = 6.0, max_batch_events: int = 2048):
    from . import capi
    cfg = capi.ServerConfig(ndim=ndim, n_slots=slots, max_batch_events=max_batch_events, max_event_points=200000,
                            max_pending=1 << 20, device_budget_bytes=int(budget_gb * (1 << 30)))
    return capi.Server(cfg, capi.Params(dc=2.5, rhoc=6.0, dm=2.5), capi.FlatKernel(0.5))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000,50000")
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--pool", type=int, default=2048)
    ap.add_argument("--slots", type=int, default=3)
    ap.add_argument("--budget-gb", type=float, default=6.0)
    ap.add_argument("--max-batch-events", type=int, default=2048)
    args = ap.parse_args()
    coords, weight, off, _ = make_pool(args.pool)
    srv = make_server(slots=args.slots, budget_gb=args.budget_gb, max_batch_events=args.max_batch_events)
    try:
        st = srv.stats()
        run_rate(srv, coords, weight, off, 2000.0, 0.5, seed=99)  # warm-up
        for i, r in enumerate(float(x) for x in args.rates.split(",")):
            rec = run_rate(srv, coords, weight, off, r, args.seconds, seed=1000 + i)
            rec.update(slots=args.slots, slot_points=st["slot_points"], slot_events=st["slot_events"],
                       device_bytes=st["device_bytes"], pool_events=len(off) - 1)
            print(json.dumps(rec), flush=True)
    finally:
        srv.close()


if __name__ == "__main__":
    main()
