#!/usr/bin/env python
"""Benchmark of the CLUE make_clusters path on B200 (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

A step is one replay of the CUDA graph of the whole batched pipeline (bounding boxes, tile
sort, local density, nearest higher, seeds, labels, output scatter) over this rank's events,
already resident in HBM (`value`: device time from CUDA events on the launching stream, L2
flushed between steps by writing a 256 MiB buffer).  `e2e` repeats the step through the C ABI
(clue_batch_make_clusters) with pinned host buffers: the host->device copy of coordinates and
weights, the pipeline, and the device->host copy of the labels and seed flags (what the
reference's make_clusters hands back to the caller), all inside the timed region.

Under torchrun the workload is 4096 calorimeter events per rank (block b of 4096 events is
generated with seed 4000 + b, so block 0 is the single-GPU workload); the events of all blocks
are partitioned over the ranks by size (sharding.partition_events), every rank clusters its
share with no collective on the data path ("scaling": "weak"), the step time is the max over
ranks, and rank 0 gathers the per-event cluster counts (sharding.gather_event_results) and
prints a checksum of block 0's events, comparable between runs on any number of GPUs.

--impl reference times the CPU restatement of the reference's serial path (oracle/, the
reference itself cannot be built: its alpaka3 dependency is fetched over the network) on a
bounded sample of the same workload, with all host cores, on rank 0 only.  It emits the same
`config` object as the GPU arm.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "points/sec batched vs plain launch on 1 B200; p50/p99 event latency"
EVENTS_PER_GPU = 4096
CPU_SAMPLE_STRIDE = 8      # cpu baseline / reference arm: every 8th event of block 0 (512 events)
SERIAL_SAMPLE_STRIDE = 64  # serial restatement: every 64th event of block 0 (64 events)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Events:
    """A batched workload: events concatenated into one SoA buffer with offsets.  `ids` are the
    events' numbers in the whole job (block b holds ids [4096 b, 4096 (b + 1)))."""

    def __init__(self, name, events, dc, rhoc, dm, kernel, ids=None):
        self.name = name
        self.events = events
        self.ids = np.arange(len(events)) if ids is None else np.asarray(ids)
        self.offsets = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in events])]).astype(np.int32)
        self.coords = np.ascontiguousarray(np.concatenate([e[0] for e in events], axis=1))
        self.weight = np.ascontiguousarray(np.concatenate([e[1] for e in events]))
        self.dc, self.rhoc, self.dm, self.kernel = dc, rhoc, dm, kernel

    def subset(self, ids):
        ids = np.asarray(ids)
        return Events(self.name, [self.events[i] for i in ids], self.dc, self.rhoc, self.dm, self.kernel,
                      self.ids[ids])


def make_workload(name: str, world: int):
    """The whole job's workload (every rank builds the same one)."""
    from cluestering_alpaka3_b200 import synthetic
    if name == "calo4096":
        evs, p = [], None
        for b in range(world):
            blk, p = synthetic.calo_events(EVENTS_PER_GPU, seed=4000 + b)
            evs.extend(blk)
        return Events("calo4096", evs, p["dc"], p["rhoc"], p["dm"], p["kernel"])
    if name == "blobs2d_1m":
        return synthetic.blobs_2d_1m()
    if name == "blobs2d_16k":
        return synthetic.blobs_2d_16k()
    if name == "blobs3d_4m":
        return synthetic.blobs_3d_4m()
    raise SystemExit(f"unknown workload {name}")


def rank_share(wl, world: int, rank: int):
    """This rank's part: its events of a batched workload (partitioned by size), or a replica
    of a single-event workload."""
    if not isinstance(wl, Events) or world == 1:
        return wl
    from cluestering_alpaka3_b200.sharding import partition_events
    sizes = np.diff(wl.offsets)
    return wl.subset(partition_events(sizes, world)[rank])


def workload_config(wl, world: int) -> dict:
    """The `config` object of both arms: the workload and how it is run, nothing measured."""
    ndim, n = wl.coords.shape
    kname, kpar = wl.kernel
    cfg = {"workload": wl.name, "n_points": int(n), "ndim": int(ndim), "dc": wl.dc, "rhoc": wl.rhoc, "dm": wl.dm,
           "kernel": [kname, list(kpar)], "metric": "euclidean", "points_per_tile": 128,
           "l2": "flushed between steps (256 MiB write)"}
    if isinstance(wl, Events):
        cfg.update({"n_events": len(wl.events), "events_per_gpu": EVENTS_PER_GPU,
                    "event_sizes": "lognormal(median 2000, sigma 1) clipped to [100, 60000]",
                    "seeds": f"4000 + block, {world} block(s) of {EVENTS_PER_GPU} events",
                    "parallelism": "single" if world == 1 else f"events sharded over {world} ranks",
                    "step": "one CUDA-graph replay of the batched pipeline over the rank's events"})
    else:
        cfg.update({"n_events": 1, "parallelism": "single" if world == 1 else f"{world} replicas",
                    "step": "one CUDA-graph replay of the pipeline over the whole input"})
    return cfg


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for k, nm in enumerate(names):
                    if r[4 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- CPU restatement (baseline / reference arm) ---------------------------------------------

def cpu_sample(wl, stride: int):
    """A bounded sample of the workload: every `stride`-th event of block 0 (batched workloads;
    sizes follow the same distribution), or the whole input (single-event workloads)."""
    if not isinstance(wl, Events):
        return wl
    ids = np.nonzero((wl.ids < EVENTS_PER_GPU) & (wl.ids % stride == 0))[0]
    return wl.subset(ids)


def run_cpu(sample, mode: str, threads: int):
    """One pass of the restatement over the sample; returns (seconds, points).  mode "events":
    events in parallel, one per thread, each clustered serially; "points": events one after the
    other, OpenMP over the points of each (the reference's OpenMP backend runs one make_clusters
    call that way); "serial": one thread."""
    from oracle import oracle as O
    kname, kpar = sample.kernel
    nt = 1 if mode == "serial" else threads
    cfg = O.Config(dc=sample.dc, rhoc=sample.rhoc, dm=sample.dm, kernel=kname, kernel_par=kpar, nthreads=nt)
    c, w = sample.coords, sample.weight
    off = sample.offsets if isinstance(sample, Events) else np.array([0, c.shape[1]], np.int32)
    t0 = time.perf_counter()
    if mode == "points":
        for e in range(len(off) - 1):
            O.run(c[:, off[e]:off[e + 1]], w[off[e]:off[e + 1]], cfg)
    else:
        O.run_events(c, w, off, cfg)
    return time.perf_counter() - t0, int(off[-1])


def sample_text(sample, stride: int) -> str:
    if isinstance(sample, Events):
        return (f"every {stride}th of the first {EVENTS_PER_GPU} {sample.name} events "
                f"({len(sample.events)} events, {int(sample.offsets[-1])} points), each clustered alone")
    return f"the whole {sample.name} input ({sample.coords.shape[1]} points)"


def cpu_modes(sample) -> tuple:
    return ("events", "points") if isinstance(sample, Events) and len(sample.events) > 1 else ("points",)


def reference_arm(args, rank: int, world: int):
    """The reference's path restated in C, timed on the host cores of rank 0 (other ranks exit)."""
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    wl = make_workload(args.workload, world)
    sample = cpu_sample(wl, CPU_SAMPLE_STRIDE)
    cores = os.cpu_count() or 1
    # warm-up: each parallel form once, then the faster one
    tried = {m: run_cpu(sample, m, cores)[0] for m in cpu_modes(sample)}
    mode = min(tried, key=tried.get)
    for _ in range(max(0, args.warmup - len(tried))):
        run_cpu(sample, mode, cores)
    times, pts = [], 0
    for _ in range(args.steps):
        dt, pts = run_cpu(sample, mode, cores)
        times.append(dt)
    tot = sum(times)
    v = pts * len(times) / tot
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(wl, world),
            "cpu_baseline": {"value": v, "unit": "points/s", "cores": cores, "kind": "port",
                             "sample": sample_text(sample, CPU_SAMPLE_STRIDE) + f" per step; {mode}-parallel "
                                       f"(faster in warm-up: {', '.join(f'{m} {1e3 * t:.0f} ms' for m, t in tried.items())})",
                             "build": "gcc -O2 -march=native -ffp-contract=off -fopenmp"},
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(wl, cores: int) -> dict:
    """The restatement on this host's cores beside the GPU numbers: both parallel forms on the
    bounded sample (value = the faster) and the serial restatement on a smaller one."""
    sample = cpu_sample(wl, CPU_SAMPLE_STRIDE)
    forms = {}
    for m in cpu_modes(sample):
        dt, pts = run_cpu(sample, m, cores)
        forms[m] = pts / dt
    best = max(forms, key=forms.get)
    out = {"value": forms[best], "unit": "points/s", "cores": cores, "kind": "port",
           "sample": sample_text(sample, CPU_SAMPLE_STRIDE) + f"; {best}-parallel",
           "forms_points_per_s": forms, "build": "gcc -O2 -march=native -ffp-contract=off -fopenmp"}
    if isinstance(wl, Events):
        ssample = cpu_sample(wl, SERIAL_SAMPLE_STRIDE)
        dt, pts = run_cpu(ssample, "serial", 1)
        out["serial"] = {"value": pts / dt, "unit": "points/s", "cores": 1,
                         "sample": sample_text(ssample, SERIAL_SAMPLE_STRIDE)}
    return out


# ---- GPU arm ----------------------------------------------------------------------------------

class DeviceRun:
    """One workload resident on this rank's GPU: inputs, outputs, and the captured graph of the
    batched pipeline (a single-event workload is a batch of one event, the plain path)."""

    def __init__(self, capi, torch, ctx, wl, stream, dev):
        self.wl = wl
        self.ctx, self.stream, self.sp = ctx, stream, stream.cuda_stream
        self.ndim, self.n = wl.coords.shape
        self.offsets = wl.offsets if isinstance(wl, Events) else np.array([0, self.n], np.int32)
        self.E = len(self.offsets) - 1
        kname, kpar = wl.kernel
        self.kernel = {"flat": capi.FlatKernel, "exp": capi.ExponentialKernel, "gaus": capi.GaussianKernel}[kname](*kpar)
        self.params = capi.Params(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm)
        self.metric = capi.Metric()
        self.dcoords = torch.from_numpy(wl.coords).to(dev)
        self.dweight = torch.from_numpy(wl.weight).to(dev)
        # the outputs the reference's make_clusters leaves in PointsDevice (labels, seed flags,
        # densities, nearest highers; the reference stores no delta)
        self.outs = {k: torch.empty(self.n, dtype=dt, device=dev) for k, dt in
                     (("cluster_index", torch.int32), ("is_seed", torch.int32), ("rho", torch.float32),
                      ("nearest_higher", torch.int32))}
        self.optr = {k: v.data_ptr() for k, v in self.outs.items()}
        self.ncl = torch.zeros(self.E, dtype=torch.int32, device=dev)
        self.graph = ctx.capture_batch(self.dcoords.data_ptr(), self.dweight.data_ptr(), self.ndim, self.offsets,
                                       self.optr, self.params, self.kernel, self.metric,
                                       ncl_ptr=self.ncl.data_ptr(), stream=self.sp)

    def direct(self, params=None):
        """The same pipeline enqueued directly (not from the graph)."""
        self.ctx.batch_device(self.dcoords.data_ptr(), self.dweight.data_ptr(), self.ndim, self.offsets, self.optr,
                              params or self.params, self.kernel, self.metric, ncl_ptr=self.ncl.data_ptr(),
                              stream=self.sp, blocking=False)

    def close(self):
        self.graph.close()


def time_replays(torch, run: DeviceRun, flush, steps: int, warmup: int):
    """Per-step device ms of `steps` graph replays (after `warmup`), L2 flushed before each."""
    for _ in range(warmup):
        run.graph.launch(run.sp)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for k in range(steps):
        with torch.cuda.stream(run.stream):
            flush.zero_()
            starts[k].record(run.stream)
        run.graph.launch(run.sp)
        with torch.cuda.stream(run.stream):
            ends[k].record(run.stream)
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in zip(starts, ends)]


def stage_times(torch, run: DeviceRun, flush, reps: int = 3) -> np.ndarray:
    """Mean per-stage device ms (tiles, density, nearest higher, seeds + labels) of direct runs."""
    run.ctx.set_timing(True)
    acc = np.zeros(4)
    for _ in range(reps):
        with torch.cuda.stream(run.stream):
            flush.zero_()
        run.direct()
        acc += np.array(run.ctx.stage_times())
    run.ctx.set_timing(False)
    return acc / reps


def near_counts(run: DeviceRun, capi) -> dict:
    """Near-threshold counts of one direct run with the near-tie count enabled (outside timing)."""
    import dataclasses
    run.direct(dataclasses.replace(run.params, flags=capi.FLAG_NEAR_TIES))
    c = run.ctx.near_counts(run.sp)
    c["tolerance"] = capi.NEAR_TOL
    return c


def e2e_host(torch, run: DeviceRun, steps: int) -> tuple:
    """Wall ms per step of the batch through the C ABI from pinned host memory (inputs copied
    in, labels and seed flags copied back), and the bytes copied each way per step."""
    wl, n, E = run.wl, run.n, run.E
    hc = torch.from_numpy(wl.coords).pin_memory().numpy()
    hw = torch.from_numpy(wl.weight).pin_memory().numpy()
    hout = {k: torch.empty(n, dtype=torch.int32).pin_memory().numpy() for k in ("cluster_index", "is_seed")}
    hncl = torch.empty(E, dtype=torch.int32).pin_memory().numpy()
    for _ in range(2):
        run.ctx.batch_host(hc, hw, run.offsets, run.params, run.kernel, run.metric, stream=run.sp, out=hout, ncl=hncl)
    ms = []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run.ctx.batch_host(hc, hw, run.offsets, run.params, run.kernel, run.metric, stream=run.sp, out=hout, ncl=hncl)
        ms.append(1e3 * (time.perf_counter() - t0))
    h2d = int(n * (run.ndim + 1) * 4 + 276 * E + 8)  # coordinates, weights, event table (276 B per event)
    d2h = int(n * 2 * 4 + 4 * E)                     # labels, seed flags, clusters per event
    return ms, h2d, d2h


def plain_block(capi, torch, local: int, dev, flush, peak: float, steps: int, warmup: int) -> dict:
    """The plain single-event path on the two large single-instance configurations: 1M 2-D points
    with the flat kernel and 4M 3-D points with the Gaussian kernel, one graph replay per step."""
    from cluestering_alpaka3_b200 import bytes_model
    out = {}
    ctx = capi.Context(local)
    stream = torch.cuda.Stream(device=local)
    try:
        for name in ("blobs2d_1m", "blobs3d_4m"):
            wl = make_workload(name, 1)
            run = DeviceRun(capi, torch, ctx, wl, stream, dev)
            try:
                ms = time_replays(torch, run, flush, steps, warmup)
                st = stage_times(torch, run, flush)
                e2e_ms, h2d, d2h = e2e_host(torch, run, max(3, steps // 4))
                nc = near_counts(run, capi)
                ncl = int(run.ncl.sum().item())
            finally:
                run.close()
            B = bytes_model.algorithmic_bytes(wl.coords, wl.dc, wl.dm)
            t = float(np.mean(ms))
            n = wl.coords.shape[1]
            out[name] = {
                "n_points": n, "ndim": wl.coords.shape[0], "kernel": [wl.kernel[0], list(wl.kernel[1])],
                "dc": wl.dc, "rhoc": wl.rhoc, "dm": wl.dm, "n_clusters": ncl,
                "device_ms": t, "points_per_s": n / (t / 1e3),
                "e2e": {"points_per_s": n / (float(np.mean(e2e_ms)) / 1e3), "h2d_bytes": h2d, "d2h_bytes": d2h},
                "stage_ms": dict(zip(("tiles", "density", "nearest_higher", "seeds_labels"), map(float, st))),
                "b_alg": B["total"], "b_alg_term1": B["term1"],
                "pipeline_hbm_frac": B["total"] / (t / 1e3) / 1e9 / peak,
                "density_hbm_frac": B["density_kernel"] / (st[1] / 1e3) / 1e9 / peak,
                "nearest_higher_hbm_frac": B["nearest_higher_kernel"] / (st[2] / 1e3) / 1e9 / peak,
                "near_threshold": nc}
    finally:
        ctx.close()
    return out


def serving_block():
    from cluestering_alpaka3_b200 import serve_bench
    pc, pw, po, _ = serve_bench.make_pool(512)
    srv = serve_bench.make_server(slots=3, budget_gb=6.0)
    try:
        serve_bench.run_rate(srv, pc, pw, po, 2000.0, 0.3, seed=99)  # warm-up
        rates = [serve_bench.run_rate(srv, pc, pw, po, r, 2.0, seed=1000 + i)
                 for i, r in enumerate((5000.0, 20000.0, 50000.0))]
    finally:
        srv.close()
    return {"workload": "Poisson stream of 4-D events (lognormal sizes, median 2000, clipped [100, 200000]), "
                        "dc=2.5 rhoc=6 dm=2.5 FlatKernel(0.5), 3 slots, 6 GiB device budget",
            "rates": [{k: r[k] for k in ("offered_events_per_s", "p50_ms", "p99_ms", "points_per_s",
                                         "achieved_events_per_s", "events_per_batch", "refused")} for r in rates]}


def events_checksum(per_event: dict) -> dict:
    """Checksum of the per-event cluster counts of block 0 (event ids below EVENTS_PER_GPU)."""
    ids = sorted(e for e in per_event if e < EVENTS_PER_GPU)
    arr = np.array([per_event[e] for e in ids], np.int32)
    return {"events": len(ids), "clusters": int(arr.sum()),
            "sha1_16": hashlib.sha1(np.ascontiguousarray(arr).tobytes()).hexdigest()[:16]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="calo4096", choices=["calo4096", "blobs2d_16k", "blobs2d_1m", "blobs3d_4m"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from cluestering_alpaka3_b200 import bytes_model, capi
    from cluestering_alpaka3_b200.sharding import gather_event_results

    wl_all = make_workload(args.workload, world)
    wl = rank_share(wl_all, world, rank)
    batched = isinstance(wl, Events)
    dev = f"cuda:{local}"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ctx = capi.Context(local)
    stream = torch.cuda.Stream(device=local)
    run = DeviceRun(capi, torch, ctx, wl, stream, dev)
    n, E = run.n, run.E

    # ---- timed device-resident steps: one graph replay each ---------------------------------
    for _ in range(args.warmup):
        run.graph.launch(run.sp)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    clocks = Clocks(local)
    ms = time_replays(torch, run, flush, args.steps, 0)
    clk = clocks.stop()
    total_ms = float(sum(ms))
    job_points = int(wl_all.coords.shape[1]) if batched else world * n
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    value = job_points * args.steps / (total_ms / 1e3)
    ev_ncl = run.ncl.cpu().numpy()

    # launches per replay = the launches the capture enqueued (one direct run counts them)
    run.direct()
    torch.cuda.synchronize()
    launches = (ctx.kernel_launches - launches0) * args.steps
    stage_avg = stage_times(torch, run, flush)
    near = near_counts(run, capi)

    # ---- per-event results gathered on rank 0 (comparable at every N) ------------------------
    local_res = {int(i): int(c) for i, c in zip(wl.ids, ev_ncl)} if batched else {0: int(ev_ncl.sum())}
    merged = gather_event_results(local_res, world, rank) if batched else local_res
    checksum = events_checksum(merged) if (batched and rank == 0) else None

    # ---- the plain per-event launch loop on the same events ---------------------------------
    plain_loop = None
    if batched:
        torch.cuda.synchronize()
        for _ in range(2):
            ev_ms = ctx.events_loop(run.dcoords.data_ptr(), run.dweight.data_ptr(), run.ndim, run.offsets, run.optr,
                                    run.params, run.kernel, run.metric, stream=run.sp, event_times=True)
        loop_ms = float(ev_ms.sum())
        plain_loop = {"points_per_s": n / (loop_ms / 1e3), "ms_per_pass": loop_ms,
                      "event_latency_ms": {"p50": float(np.percentile(ev_ms, 50)),
                                           "p99": float(np.percentile(ev_ms, 99))}}

    # ---- end to end through the C ABI with pinned host buffers -------------------------------
    e2e_ms, h2d, d2h = e2e_host(torch, run, args.steps)
    e2e_total = float(sum(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    run.close()

    # ---- roofline of the dominant kernel (the longer of the two sweeps) -----------------------
    peak, peak_kind = load_peaks()
    B = bytes_model.algorithmic_bytes(wl.coords, wl.dc, wl.dm, run.offsets)
    nh_dominant = float(stage_avg[2]) > float(stage_avg[1])
    dom_ms = float(stage_avg[2] if nh_dominant else stage_avg[1])
    dom_bytes = B["nearest_higher_kernel" if nh_dominant else "density_kernel"]
    if nh_dominant:
        dom_kernel = "k_nearest_higher"
    else:
        dom_kernel = "k_density" if wl.kernel[0] == "flat" else "k_density_sym"
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic, issue = None, None
    tfile = os.path.join(ROOT, "profiles", f"traffic_{wl.name}.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f)
        traffic = tj.get("nearest_higher_bytes_per_launch" if nh_dominant else "density_bytes_per_launch")
        if "density_issue_active" in tj:
            issue = {"bound": "issue", "kernel": dom_kernel,
                     "issue_active_frac": tj.get("nearest_higher_issue_active") if nh_dominant
                     else tj["density_issue_active"],
                     "density_issue_active_frac": tj["density_issue_active"],
                     "density_xu_pipe_frac": tj.get("density_xu_pipe"),
                     "nearest_higher_issue_active_frac": tj.get("nearest_higher_issue_active"),
                     "source": tj.get("source")}

    solo = rank == 0 and world == 1
    cpu = cpu_baseline(wl, os.cpu_count() or 1) if solo and not args.no_cpu_baseline else None
    plain = plain_block(capi, torch, local, dev, flush, peak, args.steps, max(3, args.warmup)) \
        if solo and batched and not args.no_plain else None
    serving = serving_block() if solo and not args.no_serving else None

    if rank == 0:
        step_ms = total_ms / args.steps
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(wl_all, world),
            "e2e": {"value": job_points * args.steps / (e2e_total / 1e3), "unit": "points/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": dom_kernel,
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes": dom_bytes,
                         "launch_ms": dom_ms,
                         "density_frac": B["density_kernel"] / (float(stage_avg[1]) / 1e3) / 1e9 / peak,
                         "nearest_higher_frac": B["nearest_higher_kernel"] / (float(stage_avg[2]) / 1e3) / 1e9 / peak},
            "secondary_bound": issue,
            "stage_ms": dict(zip(("tiles", "density", "nearest_higher", "seeds_labels"), map(float, stage_avg))),
            "b_alg_total": B["total"], "pipeline_hbm_frac": B["total"] / (step_ms / 1e3) / 1e9 / peak,
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
            "n_clusters": int(sum(merged.values())) if (batched and rank == 0) else int(ev_ncl.sum()),
            "near_threshold": near,
        }
        if batched:
            line["batched"] = {"n_events_rank0": E, "points_per_s_per_gpu": value / world,
                               "plain_loop": plain_loop, "batched_vs_plain": (value / world) / plain_loop["points_per_s"],
                               "batch_latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
                               "events_checksum": checksum}
        line["plain"] = plain
        line["serving"] = serving
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
