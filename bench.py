#!/usr/bin/env python
"""Throughput of batched directional-subiteration thinning on one node.

Workload (per GPU): the mixed batch -- 512 2D images with sides log-uniform
64..2048 px (aspect 0.5..2) of Bezier strokes, plus 32 3D volumes with sides
log-uniform 64..192 of tubular trees -- uint8 {0,1}, seeded synthetic data.
A step is one pass of the hot path over the whole batch: batch-wide pack of
the uint8 inputs (resident in HBM) into bit-packed words, one persistent
engine launch that thins every instance to its own fixed point, batch-wide
unpack to uint8 outputs; replayed as one CUDA graph.  ``value`` is thinned
Mvoxel/s (pixels count as voxels) over all ranks.

Also reported: ``e2e`` (the same step with inputs copied from pinned host
memory and outputs copied back inside the timed region), the plain path
(one launch per pass per instance with a host readback of the change flag
after every pass) on the same batch, the roofline of the engine kernel, the
CPU baseline (the oracle's OpenMP thinning on this host's cores, on a bounded
sample) and the SM clocks sampled during the timed region.

``--impl reference`` times the reference's own thinning rules on the host
cores (oracle/_ref: the reference's rule functions run globally by an OpenMP
driver) on a bounded sample of the same workload.

Multi-GPU (torchrun): every rank thins its own batch (seed offset by rank);
no collective is on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "thinned Mvoxel/s batched vs plain, bit-exact, 1xB200; serving p99 latency"
UNIT = "Mvoxel/s"
WORKLOAD = ("mixed batch: 512 2D stroke images, sides log-uniform 64-2048 (aspect 0.5-2), "
            "+ 32 3D tree volumes, sides log-uniform 64-192; uint8 {0,1}")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="bgt", choices=["bgt", "reference"])
    p.add_argument("--seed", type=int, default=3)
    p.add_argument("--n2d", type=int, default=512, help="2D instances per GPU (smaller only for profiling)")
    p.add_argument("--n3d", type=int, default=32, help="3D instances per GPU (smaller only for profiling)")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--tune", default="cache", choices=["cache", "run", "off"],
                   help="tile configurations: cached autotuner table (tune when absent), retune, or defaults")
    p.add_argument("--e2e-chunks", type=int, default=4, help="pipeline depth of the host-to-host leg")
    p.add_argument("--e2e-buffers", type=int, default=2,
                   help="device buffer sets used in turn by consecutive host-to-host steps")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-centerline", action="store_true", help="skip the CenterlineExtraction timing block")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the single-instance legs (512^2 strokes, 4096^2 vessels, 256^3 trees)")
    p.add_argument("--serve-seconds", type=float, default=4.0, help="measured seconds of the serving run")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples every 100 ms; only the samples
    whose timestamps fall inside the timed region (mark_start .. mark_end)
    are summarised."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None
        self.t0 = self.t1 = None

    def mark_start(self):
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        self.t1 = datetime.datetime.now()

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        inside = [r for r in rows if self.t0 and self.t1 and self.t0 <= r[0] <= self.t1]
        window = "timed region"
        if not inside:  # timed region shorter than the sampling period
            inside, window = rows, "timed region and the 0.3 s before it (region shorter than one sample period)"
        sm = [r[1] for r in inside]
        smax = [r[2] for r in inside]
        reasons = {n for r in inside for n, v in zip(names, r[3]) if v.lower() == "active"}
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel: str = "engine_kernel"):
    """Per-launch DRAM bytes of `kernel` on the mixed batch from its committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_mixed_batch.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip().split()[0])
    except Exception:
        pass
    return None


def workload(seed: int, n2d: int = 512, n3d: int = 32):
    from begputhinning_b200 import synth
    imgs, vols = synth.mixed_batch(seed, n2d, n3d)
    return imgs + vols


def oracle_outputs(items):
    """The oracle's thinning of every instance (OpenMP over this host's
    cores), timed: the parity reference of the whole batch and the CPU
    baseline in one pass."""
    from oracle import pyoracle as po
    cores = host_cores()
    outs = []
    t0 = time.perf_counter()
    for it in items:
        outs.append(po.thin2d(it, cores)[0] if it.ndim == 2 else po.thin3d(it, cores)[0])
    dt = time.perf_counter() - t0
    vox = sum(it.size for it in items)
    base = {"value": vox / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"all {len(items)} instances ({vox / 1e6:.1f} Mvoxel), oracle OpenMP thinning"}
    return outs, base


def run_bgt(args, rank, world, local):
    import numpy as np
    import torch
    import torch.distributed as dist

    import begputhinning_b200 as bgt

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    items = workload(args.seed + 1000 * rank, args.n2d, args.n3d)
    from begputhinning_b200 import tune
    table = None
    if args.tune == "cache":
        table = tune.load_cache(local)
    if args.tune == "run" or (args.tune == "cache" and table is None):
        table = tune.autotune(items, device=local)["table"]
        if rank == 0:
            tune.save_cache(table, local)
    table = table or {}
    sizes = [it.size for it in items]
    units = int(sum(sizes))
    total = sum(sizes)
    offs = np.cumsum([0] + sizes)

    # inputs resident in HBM (one allocation), outputs likewise
    host_in = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    hv = host_in.numpy()
    for it, o in zip(items, offs):
        hv[o:o + it.size] = it.reshape(-1)
    host_out = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    dev_in = host_in.to(dev)
    dev_out = torch.empty_like(dev_in)

    ctx = bgt.Context(local)
    stream = torch.cuda.Stream(dev)
    ctx.set_stream(stream)
    b = bgt.Batch(ctx)
    ids = [b.add(it.shape) for it in items]
    b.finalize()
    for i, it, o in zip(ids, items, offs):
        b.set_io(i, dev_in[o:o + it.size], dev_out[o:o + it.size])
    torch.cuda.synchronize()

    def step():
        b.run(graph=True, sync=False)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()

    # bit-exactness of every instance of the timed batch against the oracle
    out_np = dev_out.cpu().numpy()
    want_all, cpu_base = oracle_outputs(items)
    checked = 0
    for k, (it, want) in enumerate(zip(items, want_all)):
        got = out_np[offs[k]:offs[k] + it.size].reshape(it.shape)
        if not np.array_equal(got, want):
            raise SystemExit(f"bench parity check failed on instance {k} shape {it.shape}: "
                             f"{int((got != want).sum())} voxels differ")
        checked += 1
    del want_all
    plans = [b.plan(i) for i in ids]

    gpu_uuid = None
    try:
        gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
        if not gpu_uuid.startswith("GPU-"):
            gpu_uuid = "GPU-" + gpu_uuid
    except Exception:
        gpu_uuid = None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_uuid)
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark_start()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark_end()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps

    # engine kernel alone: stage events recorded by the library on the same stream
    eng_ms, pack_ms, unpack_ms, res_ms, ring_ms = [], [], [], [], []
    for _ in range(max(3, args.steps // 2)):
        with torch.cuda.stream(stream):
            step()
        p, e, u = b.stage_ms()
        r, g = b.engine_ms()
        eng_ms.append(e)
        pack_ms.append(p)
        unpack_ms.append(u)
        res_ms.append(r)
        ring_ms.append(g)
    tiles, words = b.work()

    # end to end: pinned host -> device, thin, device -> pinned host
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(3, args.steps // 2)
    with torch.cuda.stream(stream):
        dev_in.copy_(host_in, non_blocking=True)
        step()
        host_out.copy_(dev_out, non_blocking=True)
        h0.record(stream)
        for _ in range(e2e_steps):
            dev_in.copy_(host_in, non_blocking=True)
            step()
            host_out.copy_(dev_out, non_blocking=True)
        h1.record(stream)
    torch.cuda.synchronize()
    e2e_serial_ms = h0.elapsed_time(h1) / e2e_steps
    if not torch.equal(host_out, dev_out.cpu()):
        raise SystemExit("e2e output mismatch")

    # end to end, pipelined: chunks copied in / thinned / copied out on three
    # streams (volumes first: their chains of passes start earliest)
    order = [k for k, it in enumerate(items) if it.ndim == 3] + [k for k, it in enumerate(items) if it.ndim == 2]
    pb = bgt.PipelinedBatch([items[k].shape for k in order], chunks=args.e2e_chunks, device=local,
                            buffers=args.e2e_buffers)
    p_in = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    p_out = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    pv = p_in.numpy()
    for k, o in zip(order, pb.offs):
        pv[o:o + items[k].size] = items[k].reshape(-1)
    for _ in range(2):
        pb.run(p_in, p_out)
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(pb.s_in)
    for _ in range(e2e_steps):
        pb.run(p_in, p_out)
    q1.record(pb.s_out)
    torch.cuda.synchronize()
    e2e_ms = q0.elapsed_time(q1) / e2e_steps
    po_np = p_out.numpy()
    hv_out = host_out.numpy()
    for k, o in zip(order, pb.offs):
        if not np.array_equal(po_np[o:o + items[k].size], hv_out[offs[k]:offs[k] + items[k].size]):
            raise SystemExit(f"pipelined e2e output differs on instance {k}")
    pb.close()

    # plain path on the same batch (one launch per pass, host readback per pass)
    plain = None
    if not args.no_plain:
        # one untimed run (first launches of the per-pass kernels), then the
        # fastest of three: the path is bound by host round trips per pass and
        # single runs on a shared host were seen up to 4x slower; the fastest
        # run is the plain path's best case, which keeps the ratio conservative
        plain_runs = []
        for k in range(4):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.run(plain=True, sync=True)
            if k > 0:
                plain_runs.append(time.perf_counter() - t0)
        plain_s = min(plain_runs)
        if not torch.equal(dev_out.cpu(), host_out):
            raise SystemExit("plain path output differs from the engine")
        plain = {"value": units / plain_s / 1e6, "unit": UNIT, "ms_per_step": plain_s * 1e3,
                 "what": "one launch per pass per instance, host readback of the change flag after each pass; "
                         "fastest of 3 runs after one untimed run"}
        # the same passes with the loop on the device: a graph with one
        # conditional WHILE node per instance (the first run builds it)
        dl_runs = []
        for k in range(4):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.run(plain=True, device_loop=True, sync=True)
            if k > 0:
                dl_runs.append(time.perf_counter() - t0)
        dl_s = min(dl_runs)
        if not torch.equal(dev_out.cpu(), host_out):
            raise SystemExit("plain path (device loop) output differs from the engine")
        plain["device_loop"] = {"value": units / dl_s / 1e6, "unit": UNIT, "ms_per_step": dl_s * 1e3,
                                "what": "the same passes, one CUDA graph with a conditional WHILE node per "
                                        "instance (no host readback); fastest of 3 replays after the run "
                                        "that builds the graph"}

    # cross-rank aggregation: max time, summed units
    t = torch.tensor([ms, e2e_ms, statistics.median(eng_ms)], device=dev, dtype=torch.float64)
    u = torch.tensor([units], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    ms_max, e2e_max, eng_max = t.tolist()
    units_all = u.item()

    if rank != 0:
        return None
    peak, peak_kind = measured_peaks()
    eng = statistics.median(eng_ms)
    res, ring = statistics.median(res_ms), statistics.median(ring_ms)
    n_res = sum(1 for r, _ in plans if r)
    # the dominant kernel: the resident kernel when it takes the batch, else the tile-ring engine
    kernel, kms = ("resident_kernel", res) if res >= ring else ("engine_kernel", ring)
    alg_bytes = words * 8.0  # one 4-byte read + one 4-byte write per packed core word per pass
    achieved = alg_bytes / (kms * 1e-3) / 1e9
    # kernels per step: batch pack, scheduler reset, resident reset, resident kernel, the
    # tile-ring seed + engine (when some instance may use them), batch unpack
    any_ring = n_res < len(items) or any(it.ndim == 3 for it in items)
    launches_per_step = 4 + (1 if n_res else 0) + (2 if any_ring else 0)
    n2 = sum(1 for it in items if it.ndim == 2)
    line = {
        "metric": METRIC,
        "value": units_all / (ms_max * 1e-3) / 1e6,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded generators of the workload shapes; no public dataset)",
        "config": {"workload": WORKLOAD, "instances_2d": n2, "instances_3d": len(items) - n2,
                   "voxels_per_gpu": units, "input_bytes_per_gpu": total,
                   "l2": "inputs larger than L2 (uint8 inputs and outputs of several hundred MB per step)",
                   "step": "batch-wide pack + persistent engine + batch-wide unpack, one CUDA graph",
                   "tile_configs": {f"{d}D class {c}": v for (d, c), v in sorted(table.items())},
                   "parallelism": f"instances per rank, {world} rank(s), no collective"},
        "e2e": {"value": units_all / (e2e_max * 1e-3) / 1e6, "unit": UNIT, "h2d_bytes_per_step": total,
                "d2h_bytes_per_step": total,
                "path": f"pinned host -> HBM copies, batch C ABI runs, HBM -> pinned host copies; "
                        f"{args.e2e_chunks} chunks pipelined on three streams, {args.e2e_buffers} device "
                        f"buffer sets used in turn by consecutive steps (PipelinedBatch)",
                "serial_value": units / (e2e_serial_ms * 1e-3) / 1e6},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": ncu_traffic(kernel), "peak_kind": peak_kind,
                     "kernel": kernel, "launch_ms": kms,
                     "algorithmic_bytes_per_launch": alg_bytes, "work_units": tiles},
        "stage_ms": {"pack": statistics.median(pack_ms), "engine": eng, "resident_kernel": res,
                     "tile_rings": ring, "unpack": statistics.median(unpack_ms)},
        "instances_resident": n_res,
        "gpu_launches": launches_per_step * args.steps,
        "parity_checked_instances": checked,
        "clocks": clk,
    }
    if plain:
        line["plain"] = plain
        line["batched_over_plain"] = line["value"] / plain["value"]
    b.close()
    ctx.close()
    if world == 1:
        line["cpu_baseline"] = cpu_base
        if not args.no_serve:
            from begputhinning_b200.serve import run_workload
            s = run_workload(duration_s=args.serve_seconds, device=local)
            line["serving"] = {
                "workload": "Poisson arrivals: 16 streams x 30 fps of 1024x1024 frames (70% of requests) + "
                            "tree volumes with sides U[128,320] (30%); 64 GB HBM budget",
                "frame_p50_ms": s["frames"]["p50_ms"], "frame_p99_ms": s["frames"]["p99_ms"],
                "volume_p50_ms": s["volumes"]["p50_ms"], "volume_p99_ms": s["volumes"]["p99_ms"],
                "frames_completed": s["frames"]["completed"], "volumes_completed": s["volumes"]["completed"],
                "frame_mvoxel_per_s": s["frames"]["mvoxel_per_s"],
                "volume_mvoxel_per_s": s["volumes"]["mvoxel_per_s"],
                "offered_requests_per_s": s["offered_rate_per_s"], "measured_seconds": s["duration_s"],
                "latency": "submission to output in pinned host memory",
                "admission": "by bytes against one resident arena of the budget (staging + batch pool per launch)",
            }
            # the same frame streams with a growing share of volume requests
            sweep = []
            for vshare in (0.5, 0.7):
                v = run_workload(duration_s=args.serve_seconds / 2, device=local, frame_share=1.0 - vshare)
                sweep.append({"volume_share": vshare, "frame_p50_ms": v["frames"]["p50_ms"],
                              "frame_p99_ms": v["frames"]["p99_ms"], "volume_p50_ms": v["volumes"]["p50_ms"],
                              "volume_p99_ms": v["volumes"]["p99_ms"],
                              "frames_completed": v["frames"]["completed"],
                              "volumes_completed": v["volumes"]["completed"],
                              "offered_requests_per_s": v["offered_rate_per_s"]})
            line["serving"]["volume_share_sweep"] = [
                {"volume_share": 0.3, "frame_p50_ms": s["frames"]["p50_ms"], "frame_p99_ms": s["frames"]["p99_ms"],
                 "volume_p50_ms": s["volumes"]["p50_ms"], "volume_p99_ms": s["volumes"]["p99_ms"],
                 "frames_completed": s["frames"]["completed"], "volumes_completed": s["volumes"]["completed"],
                 "offered_requests_per_s": s["offered_rate_per_s"]}] + sweep
        if not args.no_centerline:
            line["centerline"] = centerline_block()
        if not args.no_configs:
            line["configs"] = config_legs(local, peak, peak_kind)
    return line


def config_legs(local: int, peak: float, peak_kind: str, reps: int = 10) -> dict:
    """The single-instance workloads at their named sizes: 512x512 Bezier
    strokes, 4096x4096 vessel trees with salt and holes, 256^3 tubular trees
    with ellipsoids.  Per workload, thinning and segment extraction are
    timed separately: thinning device-resident (pack + engine + unpack of a
    one-instance batch, CUDA events on its stream, graph replay) and end to
    end through the host API (Thinning2D/Thinning3D: host buffers, copies
    included); segments by the device ExtractSegmentsV on the thinned image.
    Beside them the reference's own CPU code on the same input: its rule
    functions run globally with OpenMP on every host core (oracle/_ref), and
    its single-threaded ExtractSegmentsV; outputs are compared."""
    import numpy as np
    import torch

    import begputhinning_b200 as bgt
    from begputhinning_b200 import synth
    from oracle import pyoracle as po
    cores = host_cores()
    cases = [("strokes_512x512", synth.frame512(0)),
             ("vessels_4096x4096", synth.vessels4096(1)),
             ("trees_256x256x256", synth.trees256(2))]
    dev = torch.device("cuda", local)
    ctx = bgt.Context(local)
    stream = torch.cuda.Stream(dev)
    ctx.set_stream(stream)
    out = {}
    for name, data in cases:
        e = {"shape": list(data.shape), "voxels": int(data.size), "foreground": float((data != 0).mean())}
        d_in = torch.from_numpy(data).to(dev)
        d_out = torch.empty_like(d_in)
        b = bgt.Batch(ctx)
        i = b.add(data.shape)
        b.finalize()
        b.set_io(i, d_in, d_out)
        resident, bands = b.plan(i)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for _ in range(3):
                b.run(graph=True, sync=False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(reps):
                b.run(graph=True, sync=False)
            e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        pk, en, un = b.stage_ms()
        rk, rg = b.engine_ms()
        _, words = b.work()
        st = b.stats(i)
        thinned = d_out.cpu().numpy()
        kms = rk if rk >= rg else rg
        achieved = words * 8.0 / (kms * 1e-3) / 1e9
        e["thinning"] = {
            "ms": ms, "mvoxel_per_s": data.size / ms / 1e3, "stage_ms": {"pack": pk, "engine": en, "unpack": un},
            "engine_kernels_ms": {"resident_kernel": rk, "tile_rings": rg}, "iterations": st["passes"],
            "resident": resident, "bands": bands,
            "roofline": {"bound": "hbm", "kernel": "resident_kernel" if rk >= rg else "engine_kernel",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": words * 8.0}}
        b.close()
        thin_api = bgt.Thinning2D if data.ndim == 2 else bgt.Thinning3D
        thin_api(data, ctx)
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            api_out = thin_api(data, ctx)
            ts.append((time.perf_counter() - t0) * 1e3)
        e2e = statistics.median(ts)
        e["thinning"]["e2e"] = {"ms": e2e, "mvoxel_per_s": data.size / e2e / 1e3,
                                "path": "Thinning2D/Thinning3D C ABI: host buffer in, host buffer out"}
        segs = bgt.ExtractSegmentsV(d_out, ctx)
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            segs = bgt.ExtractSegmentsV(d_out, ctx)
            ts.append((time.perf_counter() - t0) * 1e3)
        e["segments"] = {"ms": statistics.median(ts), "segments": int(segs.nseg),
                         "path": "device ExtractSegmentsV on the thinned image in device memory, "
                                 "segment arrays copied to the host"}
        which = "2d" if data.ndim == 2 else "3d"
        if po.have_ref(which):
            t0 = time.perf_counter()
            ref_thin = po.ref_thin2d(data) if data.ndim == 2 else po.ref_thin3d(data)
            ref_ms = (time.perf_counter() - t0) * 1e3
            t0 = time.perf_counter()
            ref_segs = po.ref_segments2d(ref_thin) if data.ndim == 2 else po.ref_segments3d(ref_thin)
            seg_ms = (time.perf_counter() - t0) * 1e3
            e["reference_cpu"] = {
                "thinning_ms": ref_ms, "thinning_mvoxel_per_s": data.size / ref_ms / 1e3, "thinning_cores": cores,
                "segments_ms": seg_ms, "segments_threads": 1,
                "kind": "reference (its rule functions with a global synchronous OpenMP driver; its ExtractSegmentsV)"}
            e["identical_to_reference"] = {
                "thinning": bool(np.array_equal(thinned, ref_thin) and np.array_equal(api_out, ref_thin)),
                "segments": segs.as_lists() == ref_segs.as_lists()}
            e["speedup_vs_reference_cpu"] = {"thinning_e2e": ref_ms / e2e, "segments": seg_ms / e["segments"]["ms"]}
        if name.startswith("vessels"):
            e["reference_gpu"] = ("not run: the reference's Thinning2D divides by zero on the host for widths "
                                  "2049-4096 (2D/LibThinning2D.cu:66)")
        out[name] = e
    ctx.close()
    return out


def centerline_block(calls: int = 10) -> dict:
    """The reference-facing CenterlineExtraction call (host buffers in and
    out: H2D, thinning, device segments, device pruning/smoothing/CSR, D2H)
    on the 512x512 stroke frame and the 256^3 tree volume, timed per call
    beside the reference's own CPU CenterlineExtraction (its .cpp code and
    rules, oracle/_ref) on the same inputs; the outputs are compared."""
    import numpy as np
    from begputhinning_b200 import CenterlineExtraction, synth
    from begputhinning_b200.api import dtype_code
    from oracle import pyoracle as po
    ml, sp = 10, 3
    out = {"max_segment_length": ml, "smoothing_span": sp}
    for name, data in (("frame_512x512", synth.frame512(0)), ("volume_256x256x256", synth.trees256(2))):
        res = CenterlineExtraction(data, ml, sp)  # warm-up (allocations, tuning of the single-instance batch)
        ts = []
        for _ in range(calls):
            t0 = time.perf_counter()
            res = CenterlineExtraction(data, ml, sp)
            ts.append((time.perf_counter() - t0) * 1e3)
        ms = statistics.median(ts)
        entry = {"ms_per_call": ms, "mvoxel_per_s": data.size / ms / 1e3, "segments": int(len(res[-1]) - 1)}
        if po.have_ref("2d" if data.ndim == 2 else "3d"):
            t0 = time.perf_counter()
            ref = (po.ref_centerline2d if data.ndim == 2 else po.ref_centerline3d)(data, dtype_code(data.dtype), ml, sp)
            rms = (time.perf_counter() - t0) * 1e3
            same = np.array_equal(res[-1], ref.idx) and all(
                np.array_equal(a.view(np.uint32), b.view(np.uint32))
                for a, b in zip(res[:-1], [ref.x, ref.y] + ([ref.z] if data.ndim == 3 else [])))
            entry.update({"reference_cpu_ms_per_call": rms, "identical_to_reference": bool(same),
                          "speedup_vs_reference_cpu": rms / ms})
        out[name] = entry
    return out


def run_reference(args, rank, world):
    """The reference's own thinning rules on the host cores (oracle/_ref)."""
    import numpy as np

    from oracle import pyoracle as po
    if rank != 0:
        return None
    items = workload(args.seed, args.n2d, args.n3d)
    have_ref = po.have_ref("2d") and po.have_ref("3d")
    kind = "reference" if have_ref else "port"
    # a bounded sample: a fixed subset of the batch sized so that every step
    # takes a few seconds (probe the speed on the first instances)
    order = list(range(len(items)))
    rng = np.random.default_rng(0)
    rng.shuffle(order)

    def thin(it):
        if have_ref:
            return po.ref_thin2d(it) if it.ndim == 2 else po.ref_thin3d(it)
        return po.thin2d(it)[0] if it.ndim == 2 else po.thin3d(it)[0]

    t0 = time.perf_counter()
    sample = []
    for k in order:
        thin(items[k])
        sample.append(k)
        if time.perf_counter() - t0 > 1.5:
            break
    budget = max(0.2, 120.0 / max(1, args.steps + args.warmup))  # seconds per step
    rate = sum(items[k].size for k in sample) / (time.perf_counter() - t0)
    target = rate * budget
    sample, vox = [], 0
    for k in order:
        if vox >= target and sample:
            break
        sample.append(k)
        vox += items[k].size
    for _ in range(args.warmup):
        for k in sample[:1]:
            thin(items[k])
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for k in sample:
            thin(items[k])
        times.append(time.perf_counter() - t0)
    mean = statistics.mean(times)
    value = vox / mean / 1e6
    cores = host_cores()
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generators of the workload shapes)",
        "config": {"workload": WORKLOAD, "sample_instances": len(sample), "sample_voxels": vox},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{len(sample)} of {len(items)} instances ({vox / 1e6:.1f} Mvoxel) per step; "
                                   + ("the reference's rule functions, global synchronous OpenMP driver"
                                      if have_ref else "the oracle's OpenMP port")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    try:
        line = run_bgt(args, rank, world, local)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
