#!/usr/bin/env python
"""Benchmark of the CLUE make_clusters path on B200 (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

A step is one pass of the five CLUE stages over one synthetic workload already resident in
HBM (`value`, device time from CUDA events on the launching stream, L2 flushed between steps
by writing a 256 MiB buffer).  `e2e` repeats the step through the C ABI with pinned host
buffers: host->device copy of coordinates and weights, the stages, and device->host copy of
the labels, seed flags, densities, nearest highers and deltas, all inside the timed region.
Under torchrun every rank clusters its own replica of the workload (seeded by rank, no
collective on the data path, scaling "weak"); the step time is the max over ranks.

--impl reference times the CPU restatement of the reference's serial path (OpenMP over points,
all host cores) on the same workload, on rank 0 only.
"""
from __future__ import annotations

import argparse
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


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Events:
    """A batched workload: events concatenated into one SoA buffer with offsets."""

    def __init__(self, name, events, dc, rhoc, dm, kernel):
        self.name = name
        self.events = events
        self.offsets = np.concatenate([[0], np.cumsum([e[0].shape[1] for e in events])]).astype(np.int32)
        self.coords = np.ascontiguousarray(np.concatenate([e[0] for e in events], axis=1))
        self.weight = np.ascontiguousarray(np.concatenate([e[1] for e in events]))
        self.dc, self.rhoc, self.dm, self.kernel = dc, rhoc, dm, kernel


def make_workload(name: str, rank: int):
    from cluestering_alpaka3_b200 import synthetic
    if name == "calo4096":
        evs, p = synthetic.calo_events(4096, seed=4000 + rank)
        return Events("calo4096", evs, p["dc"], p["rhoc"], p["dm"], p["kernel"])
    if name == "blobs2d_1m":
        return synthetic.blobs_2d_1m(seed=2000 + rank)
    if name == "blobs2d_16k":
        return synthetic.blobs_2d_16k(seed=1000 + rank)
    if name == "blobs3d_4m":
        return synthetic.blobs_3d_4m(seed=3000 + rank)
    raise SystemExit(f"unknown workload {name}")


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


CPU_SAMPLE_EVENTS = 512


def cpu_baseline_run(wl, nthreads: int):
    """The CPU restatement on the workload (batched workloads: its first CPU_SAMPLE_EVENTS
    events, each clustered alone).  Returns (seconds, points, last result)."""
    from oracle import oracle as O
    kname, kpar = wl.kernel
    cfg = O.Config(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm, kernel=kname, kernel_par=kpar, nthreads=nthreads)
    if isinstance(wl, Events):
        pts, r = 0, None
        t0 = time.perf_counter()
        for c, w in wl.events[:CPU_SAMPLE_EVENTS]:
            r = O.run(c, w, cfg)
            pts += c.shape[1]
        return time.perf_counter() - t0, pts, r
    t0 = time.perf_counter()
    r = O.run(wl.coords, wl.weight, cfg)
    return time.perf_counter() - t0, wl.coords.shape[1], r


def sample_text(wl) -> str:
    if isinstance(wl, Events):
        n = int(wl.offsets[min(CPU_SAMPLE_EVENTS, len(wl.events))])
        return f"first {CPU_SAMPLE_EVENTS} of {len(wl.events)} {wl.name} events ({n} points), each clustered alone"
    return f"full {wl.name} workload ({wl.coords.shape[1]} points)"


def reference_arm(args, rank: int):
    """The reference's path restated in C (the reference itself cannot be built: its alpaka3
    dependency is fetched over the network), timed on the host cores."""
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    wl = make_workload(args.workload, 0)
    n = wl.coords.shape[1]
    cores = os.cpu_count() or 1
    cpu_baseline_run(wl, cores)
    times, pts = [], 0
    for _ in range(args.steps):
        dt, pts, _ = cpu_baseline_run(wl, cores)
        times.append(dt)
    tot = sum(times)
    v = pts * len(times) / tot
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": wl.name, "n_points": n, "ndim": wl.coords.shape[0], "dc": wl.dc,
                       "rhoc": wl.rhoc, "dm": wl.dm, "kernel": list(wl.kernel)},
            "cpu_baseline": {"value": v, "unit": "points/s", "cores": cores, "kind": "port",
                             "sample": sample_text(wl) + " per step, OpenMP over points"},
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="calo4096",
                    choices=["calo4096", "blobs2d_16k", "blobs2d_1m", "blobs3d_4m"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    from cluestering_alpaka3_b200 import bytes_model, capi

    wl = make_workload(args.workload, rank)
    batched = isinstance(wl, Events)
    ndim, n = wl.coords.shape
    dev = f"cuda:{local}"
    kname, kpar = wl.kernel
    kernel = {"flat": capi.FlatKernel, "exp": capi.ExponentialKernel, "gaus": capi.GaussianKernel}[kname](*kpar)
    params = capi.Params(dc=wl.dc, rhoc=wl.rhoc, dm=wl.dm)
    metric = capi.Metric()

    ctx = capi.Context(local)
    stream = torch.cuda.Stream(device=local)
    sp = stream.cuda_stream
    dcoords = torch.from_numpy(wl.coords).to(dev)
    dweight = torch.from_numpy(wl.weight).to(dev)
    outs = {k: torch.empty(n, dtype=dt, device=dev) for k, dt in
            (("cluster_index", torch.int32), ("is_seed", torch.int32), ("rho", torch.float32),
             ("nearest_higher", torch.int32), ("delta", torch.float32))}
    optr = {k: v.data_ptr() for k, v in outs.items()}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    E = len(wl.offsets) - 1 if batched else 1
    offsets = wl.offsets if batched else np.array([0, n], np.int32)
    ncl = torch.zeros(E, dtype=torch.int32, device=dev)

    # the step: one replay of the whole pipeline captured in a CUDA graph
    graph = ctx.capture_batch(dcoords.data_ptr(), dweight.data_ptr(), ndim, offsets, optr, params, kernel, metric,
                              ncl_ptr=ncl.data_ptr(), stream=sp)

    def step():
        graph.launch(sp)

    torch.cuda.synchronize()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed device-resident steps --------------------------------------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    clocks = Clocks(local)
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            starts[k].record(stream)
        step()
        with torch.cuda.stream(stream):
            ends[k].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = [s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)]
    total_ms = float(sum(ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    value = world * n * args.steps / (total_ms / 1e3)
    n_clusters = int(ncl.sum().item())

    # launches per graph replay = the launches the capture enqueued
    ctx.batch_device(dcoords.data_ptr(), dweight.data_ptr(), ndim, offsets, optr, params, kernel, metric,
                     stream=sp, blocking=False)
    per_step_launches = ctx.kernel_launches - launches0
    launches = per_step_launches * args.steps

    # ---- per-stage device times of the same pipeline (events around stages) ------
    ctx.set_timing(True)
    stage_ms = np.zeros(4)
    for _ in range(3):
        with torch.cuda.stream(stream):
            flush.zero_()
        ctx.batch_device(dcoords.data_ptr(), dweight.data_ptr(), ndim, offsets, optr, params, kernel, metric,
                         stream=sp, blocking=False)
        stage_ms += np.array(ctx.stage_times())
    ctx.set_timing(False)
    stage_avg = stage_ms / 3

    # ---- the plain per-event launch loop on the same events -----------------------
    plain = None
    if batched:
        torch.cuda.synchronize()
        ev_ms = ctx.events_loop(dcoords.data_ptr(), dweight.data_ptr(), ndim, offsets, optr, params, kernel,
                                metric, stream=sp, event_times=True)
        ev_ms = ctx.events_loop(dcoords.data_ptr(), dweight.data_ptr(), ndim, offsets, optr, params, kernel,
                                metric, stream=sp, event_times=True)
        loop_ms = float(ev_ms.sum())
        plain = {"points_per_s": n / (loop_ms / 1e3), "ms_per_pass": loop_ms,
                 "event_latency_ms": {"p50": float(np.percentile(ev_ms, 50)),
                                      "p99": float(np.percentile(ev_ms, 99))}}

    # ---- end to end through the C ABI with pinned host buffers ----------------
    # inputs and the step's result (labels and seed flags, as the reference's make_clusters
    # returns them) live in pinned host memory; densities and nearest highers stay on the device
    hc = torch.from_numpy(wl.coords).pin_memory().numpy()
    hw = torch.from_numpy(wl.weight).pin_memory().numpy()
    hout = {k: torch.empty(n, dtype=torch.int32).pin_memory().numpy() for k in ("cluster_index", "is_seed")}
    hncl_buf = torch.empty(E, dtype=torch.int32).pin_memory().numpy()
    for _ in range(2):
        res, hncl = ctx.batch_host(hc, hw, offsets, params, kernel, metric, stream=sp, out=hout, ncl=hncl_buf)
    e2e_ms = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res, hncl = ctx.batch_host(hc, hw, offsets, params, kernel, metric, stream=sp, out=hout, ncl=hncl_buf)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_total = float(sum(e2e_ms))
    if world > 1:
        t = torch.tensor([e2e_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())

    # ---- roofline of the dominant kernel (local density) ------------------------
    peak, peak_kind = load_peaks()
    B = bytes_model.algorithmic_bytes(wl.coords, wl.dc, wl.dm, offsets)
    dens_ms = float(stage_avg[1])
    achieved = B["density_kernel"] / (dens_ms / 1e3) / 1e9
    traffic = None
    issue = None  # the sweeps' real bound: instruction issue and the MUFU (XU) pipe, from ncu
    tfile = os.path.join(ROOT, "profiles", f"traffic_{wl.name}.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f)
        traffic = tj.get("density_bytes_per_launch")
        if "density_issue_active" in tj:
            issue = {"bound": "issue", "kernel": tj.get("density_kernel"),
                     "issue_active_frac": tj["density_issue_active"], "xu_pipe_frac": tj.get("density_xu_pipe"),
                     "nearest_higher_issue_active_frac": tj.get("nearest_higher_issue_active"),
                     "source": tj.get("source")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        dt, pts, ref = cpu_baseline_run(wl, cores)
        cpu = {"value": pts / dt, "unit": "points/s", "cores": cores, "kind": "port",
               "sample": sample_text(wl) + ", OpenMP over points"}
        if not batched:
            cpu["labels_equal_to_gpu"] = bool(np.array_equal(ref.cluster_index, res.cluster_index))

    # ---- serving: Poisson stream of 4-D events through the continuous-batching server ----
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        from cluestering_alpaka3_b200 import serve_bench
        pc, pw, po, _ = serve_bench.make_pool(512)
        srv = serve_bench.make_server(slots=3, budget_gb=6.0)
        try:
            serve_bench.run_rate(srv, pc, pw, po, 2000.0, 0.3, seed=99)  # warm-up
            serving = [serve_bench.run_rate(srv, pc, pw, po, r, 2.0, seed=1000 + i)
                       for i, r in enumerate((5000.0, 20000.0, 50000.0))]
        finally:
            srv.close()

    if rank == 0:
        step_ms = total_ms / args.steps
        config = {"workload": wl.name, "n_points": n, "ndim": ndim, "dc": wl.dc, "rhoc": wl.rhoc, "dm": wl.dm,
                  "kernel": [kname, list(kpar)], "metric": "euclidean", "points_per_tile": 128,
                  "l2": "flushed between steps (256 MiB write)",
                  "parallelism": "replicas" if world > 1 else "single", "n_clusters": n_clusters,
                  "step": "one CUDA-graph replay of the whole pipeline"}
        if batched:
            config.update({"n_events": E, "batched_points_per_s": value / world,
                           "plain_loop": plain, "batched_vs_plain": (value / world) / plain["points_per_s"],
                           "batched_event_latency_ms": {"p50": step_ms, "p99": step_ms}})
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "e2e": {"value": world * n * args.steps / (e2e_total / 1e3), "unit": "points/s",
                    "h2d_bytes_per_step": int(n * (ndim + 1) * 4 + 12 * E + 264 * E),
                    "d2h_bytes_per_step": int(n * 2 * 4 + 4 * E)},
            "roofline": {"bound": "hbm", "kernel": "k_density" if kname == "flat" else "k_density_sym",
                         "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes": B["density_kernel"], "launch_ms": dens_ms},
            "secondary_bound": issue,
            "stage_ms": {"tiles": stage_avg[0], "density": stage_avg[1], "nearest_higher": stage_avg[2],
                         "seeds_labels": stage_avg[3]},
            "b_alg_total": B["total"],
            "pipeline_hbm_frac": B["total"] / (step_ms / 1e3) / 1e9 / peak,
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
            "serving": None if serving is None else {
                "workload": "Poisson stream of 4-D events (lognormal sizes, median 2000, clipped [100, 200000]), "
                            "dc=2.5 rhoc=6 dm=2.5 FlatKernel(0.5), 3 slots, 6 GiB device budget",
                "rates": [{k: r[k] for k in ("offered_events_per_s", "p50_ms", "p99_ms", "points_per_s",
                                             "achieved_events_per_s", "events_per_batch", "refused")}
                          for r in serving]},
        }
        print(json.dumps(line), flush=True)
    graph.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
