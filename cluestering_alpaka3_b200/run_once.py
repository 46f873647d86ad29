"""Run the clustering pipeline a few times on a synthetic workload (for profilers).

    python -m cluestering_alpaka3_b200.run_once --workload calo4096 --passes 2 [--events 1024]

Each pass enqueues the whole pipeline once (batched entry point; one event for the plain
workloads) on one stream and waits for it; the wall time of each pass is printed.  Useful as
the target command of `ncu` launch lists and kernel captures.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def build(name: str, events: int = 4096):
    from . import synthetic
    if name == "calo4096":
        evs, p = synthetic.calo_events(4096)
        evs = evs[:events]
        off = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in evs])]).astype(np.int32)
        coords = np.ascontiguousarray(np.concatenate([e[0] for e in evs], axis=1))
        weight = np.ascontiguousarray(np.concatenate([e[1] for e in evs]))
        return coords, weight, off, p["dc"], p["rhoc"], p["dm"], p["kernel"]
    wl = synthetic.CONFIGS[name]()
    n = wl.coords.shape[1]
    return wl.coords, wl.weight, np.array([0, n], np.int32), wl.dc, wl.rhoc, wl.dm, wl.kernel


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="calo4096",
                    choices=["calo4096", "blobs2d_16k", "blobs2d_1m", "blobs3d_4m"])
    ap.add_argument("--passes", type=int, default=2)
    ap.add_argument("--events", type=int, default=4096,
                    help="calo4096: cluster only the first EVENTS events (small cases for profilers)")
    ap.add_argument("--stages", action="store_true",
                    help="time the four stages with CUDA events and print their medians")
    args = ap.parse_args()

    import torch

    from . import capi
    coords, weight, off, dc, rhoc, dm, (kname, kpar) = build(args.workload, args.events)
    ndim, n = coords.shape
    kernel = {"flat": capi.FlatKernel, "exp": capi.ExponentialKernel, "gaus": capi.GaussianKernel}[kname](*kpar)
    params = capi.Params(dc=dc, rhoc=rhoc, dm=dm)
    ctx = capi.Context(0)
    dcoords = torch.from_numpy(coords).cuda()
    dweight = torch.from_numpy(weight).cuda()
    outs = {k: torch.empty(n, dtype=dt, device="cuda") for k, dt in
            (("cluster_index", torch.int32), ("is_seed", torch.int32), ("rho", torch.float32),
             ("nearest_higher", torch.int32), ("delta", torch.float32))}
    optr = {k: v.data_ptr() for k, v in outs.items()}
    stream = torch.cuda.Stream()
    if args.stages:
        ctx.set_timing(True)
    stage_ms = []
    for p in range(args.passes):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.batch_device(dcoords.data_ptr(), dweight.data_ptr(), ndim, off, optr, params, kernel, capi.Metric(),
                         stream=stream.cuda_stream, blocking=False)
        stream.synchronize()
        print(f"pass {p}: {1e3 * (time.perf_counter() - t0):.3f} ms wall, {n} points, "
              f"{len(off) - 1} events", flush=True)
        if args.stages:
            stage_ms.append(ctx.stage_times())
    if args.stages and stage_ms:
        med = np.median(np.array(stage_ms), axis=0)
        print("stage ms (median): tiles %.3f density %.3f nearest_higher %.3f seeds_labels %.3f total %.3f"
              % (med[0], med[1], med[2], med[3], med.sum()), flush=True)
    info = ctx.read_info(stream.cuda_stream)
    print(f"clusters {info.n_clusters}, seeds {info.n_seeds}")
    ctx.close()


if __name__ == "__main__":
    main()
