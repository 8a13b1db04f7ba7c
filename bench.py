"""Benchmark: the acoustic hall, 256³ nodes, 5000 steps per run (FP32 fields, FP64 audits).

One bench step is one full run of the workload: `timesteps` calls of `Hall::step`, each with
its fused FP64 invariant and on-device audit, over the 256³ grid (16.8 M nodes; 268 MB of f32
state, larger than the 126 MB L2, so no flush is needed between steps).

  value  node-updates/s with the state resident in HBM, timed with CUDA events on the stream
         the kernels run on, max over ranks. FP32 chosen form.
  e2e    the same through the C ABI with host buffers: release from pinned host memory (H2D),
         the run, the pressure field and the ledger back to the host (D2H), every step.
  plain_f64  the bit-exact f64 form on the same workload, for the FP32/f64 ratio.
  roofline   the hall kernel's algorithmic bytes (32 B per FP32 node-update: p, vx, vy, vz read
             and written once) per launch over its average launch time, against the measured
             HBM copy bandwidth.
  cpu_baseline  the reference's CPU path for this workload (the oracle's restatement of
             `Simulation::advance` over `Hall::step` and its ledger), on a bounded sample.

`--impl reference` times that CPU path alone, on all usable host cores (one independent hall per
thread, the reference's `Ensemble` pattern), and prints its own line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s (acoustic hall 256^3, FP32 fields + FP64 audit)"
UNIT = "Gcell-updates/s"
BYTES_F32 = 32  # per node-update: p, vx, vy, vz, read and written once
BYTES_F64 = 64
# DRAM traffic per launch, dram__bytes_read.sum + dram__bytes_write.sum, as one ncu capture of the
# kernel measured it (ncu cannot run inside the timed process; the capture's command is the bench's
# own, on one GPU). The hall kernel at 256³: 270.4 MB read + 219.5 MB written.
HALL_F32_TRAFFIC = 489971968
# The Yee kernel, per cell: 463.1 MB read + 385.7 MB written at 256³ cells. A launch at another
# size moves about that many bytes per cell (it reads and writes each cell's six values once; the
# wall column and row are a smaller share of a larger cavity).
YEE_F32_TRAFFIC_PER_CELL = (463146240 + 385735424) / 256 ** 3
# The ensemble brick kernel over the 512-block heat ensemble, per cell: 1.004 GB read + 772.1 MB
# written for 187,991,031 cells.
ENS_F32_TRAFFIC_PER_CELL = (1004143360 + 772071936) / 187991031


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.samples = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def summary(self):
        if not getattr(self, "samples", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for s in self.samples for q in range(4) if s[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def hall_workload(n, timesteps):
    from pantometry_b200 import workloads as W

    return W.acoustic_hall(n, steps=timesteps)


def run_ours(args):
    import numpy as np
    import torch

    from pantometry_b200 import workloads as W

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    cfg = hall_workload(args.n, args.timesteps)
    nodes = args.n ** 3
    T = args.timesteps
    stream = torch.cuda.Stream(device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed_runs(precision, k, w):
        """Each bench step is the whole workload: the hall released from the noise (outside the
        timed region, on the handle's stream), then `T` audited steps with the source from its
        first sample, timed with CUDA events around the steps alone."""
        hall = W.build_hall(cfg, precision=precision, device=local)
        hall.set_stream(stream.cuda_stream)
        hall.set_tolerance(1e-6 if precision == "f32" else 1e-9)
        if precision == "f32":
            tiles.append(hall.autotune(trial_steps=16))  # the tile shape, timed on this grid
        for _ in range(w):
            hall.release(cfg["pressure"])
            v = hall.step(cfg["dt"], T)
            assert v is None, v
        barrier()
        ms = 0.0
        with Clocks(local) as clk:
            for _ in range(k):
                hall.release(cfg["pressure"])
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                v = hall.step(cfg["dt"], T)
                end.record(stream)
                assert v is None, v
                end.synchronize()
                ms += start.elapsed_time(end)
        barrier()
        return hall, max_over_ranks(ms), clk

    # FP32 chosen form (the headline) and the plain f64 form, device-resident; each handle ends
    # holding one whole run of the workload
    tiles = []
    h32, ms32, clk = timed_runs("f32", args.steps, args.warmup)
    led32 = h32.ledger()
    p32 = h32.fields()["p"]
    del h32
    plain_steps = max(1, args.steps // 2)
    h64, ms64, _ = timed_runs("f64", plain_steps, max(1, args.warmup // 2))
    led64 = h64.ledger()
    p64 = h64.fields()["p"]
    del h64
    # the FP32 run against the f64 run, both one whole run of the workload from the release
    field_err = float(np.abs(p32 - p64).max())
    ledger_err = abs(led32["total"] - led64["total"]) / max(abs(led64["total"]), led64["scale"])

    # e2e through the C ABI with host buffers
    pinned = torch.empty(nodes, dtype=torch.float64, pin_memory=True).numpy()
    pinned[:] = cfg["pressure"]
    out = torch.empty(nodes, dtype=torch.float64, pin_memory=True).numpy()
    hall = W.build_hall(cfg, precision="f32", device=local)
    hall.set_stream(stream.cuda_stream)
    hall.set_tolerance(1e-6)
    for _ in range(args.warmup):
        hall.release(pinned)
        hall.step(cfg["dt"], T)
    barrier()
    t0 = time.perf_counter()
    s0 = torch.cuda.Event(enable_timing=True)
    e0 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        hall.release(pinned)
        v = hall.step(cfg["dt"], T)
        assert v is None, v
        hall.ledger()
        hall.download_pressure(out)
    e0.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    e2e_ms = max_over_ranks(max(s0.elapsed_time(e0), wall_ms))
    del hall

    peak, peak_kind = peaks()
    per_launch_ms = ms32 / (args.steps * T)
    achieved = BYTES_F32 * nodes / (per_launch_ms * 1e-3) / 1e9
    value = world * nodes * T * args.steps / (ms32 * 1e-3) / 1e9
    plain = world * nodes * T * plain_steps / (ms64 * 1e-3) / 1e9
    per_launch64 = ms64 / (plain_steps * T)
    line = {
        "metric": METRIC.replace("256^3", f"{args.n}^3"),
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms32 / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 fields, f64 audit",
        "data": "synthetic (seeded Rng::for_index noise + Ricker source)",
        "config": {"workload": f"acoustic_hall {args.n}^3 nodes, {T} timesteps per step, CFL 0.5, "
                               "rigid walls, FP64 audit every timestep; each step released from the noise "
                               "(outside the timed region) so the Ricker source runs from its first sample",
                   "nodes": nodes, "timesteps_per_step": T, "parallelism": f"replicas x{world}",
                   "l2": "state 268 MB > 126 MB L2, no flush"},
        "e2e": {"value": round(world * nodes * T * args.steps / (e2e_ms * 1e-3) / 1e9, 3), "unit": UNIT,
                "h2d_bytes_per_step": nodes * 8, "d2h_bytes_per_step": nodes * 8 + 8 * 16},
        "gpu_launches": args.steps * T,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": HALL_F32_TRAFFIC,
                     "kernel": f"hall_tma_step (FP32, TMA-staged, {tiles[0][0]} planes x {tiles[0][1]} stages, autotuned)",
                     "bytes_per_launch": BYTES_F32 * nodes,
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "plain_f64": {"value": round(plain, 3), "unit": UNIT, "ms_per_step": round(ms64 / plain_steps, 3),
                      "roofline_frac": round(BYTES_F64 * nodes / (per_launch64 * 1e-3) / 1e9 / peak, 4),
                      "fp32_over_f64": round(value / plain, 3)},
        "error_vs_f64": {"max_abs_pressure_pa": field_err, "ledger_rel": ledger_err, "after_timesteps": T},
        "clocks": clk.summary(),
    }
    if not args.no_side_records:
        line["cavity"] = cavity_record(local, stream, peak)
        line["ensemble"] = ensemble_record(local, stream, peak)
        line["heat_block"] = heat_block_record(local, stream, peak)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.n, sample_steps=args.cpu_sample_steps, threads=1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(n, sample_steps=2, threads=1):
    """The reference's CPU path, restated (the oracle): `Simulation::advance` with one `Hall`:
    ledger before, `attribute`'s own ledger, `Hall::step`, ledger after, audit — one thread per
    hall, `threads` independent halls at once (the `Ensemble` pattern)."""
    import oracle
    from pantometry_b200 import workloads as W

    cfg = W.acoustic_hall(n, steps=sample_steps + 1)
    w, h, d = cfg["size"]
    halls = []
    for _ in range(threads):
        o = oracle.Hall(w, h, d, cfg["across"], cfg["speed"], cfg["density"])
        o.release(cfg["pressure"])
        o.set_source(cfg["source_node"], cfg["wave"])
        assert o.advance(cfg["dt"], 1) is None  # warm-up, and the leapfrog's opening half step
        halls.append(o)
    times = [0.0] * threads

    def work(q):
        t0 = time.perf_counter()
        assert halls[q].advance(cfg["dt"], sample_steps) is None
        times[q] = time.perf_counter() - t0

    ths = [threading.Thread(target=work, args=(q,)) for q in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    secs = max(times)
    value = threads * n ** 3 * sample_steps / secs / 1e9
    return {"value": round(value, 6), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{threads} x {sample_steps} audited Simulation::advance steps of the {n}^3 hall "
                      f"(after 1 warm-up step), {secs:.2f} s"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    try:
        import psutil

        avail = psutil.virtual_memory().available
    except Exception:  # noqa: BLE001
        avail = 64 << 30
    per_hall = 6 * (args.n ** 3) * 8
    threads = max(1, min(ncpu, int(avail * 0.6 // per_hall)))
    samples = []
    for _ in range(args.steps):
        samples.append(cpu_baseline(args.n, sample_steps=args.cpu_sample_steps, threads=threads))
    value = statistics.median(s["value"] for s in samples)
    line = {
        "metric": METRIC.replace("256^3", f"{args.n}^3"), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Rng::for_index noise + Ricker source)",
        "impl": "reference",
        "config": {"workload": f"acoustic_hall {args.n}^3 nodes, audited Simulation::advance steps", "nodes": args.n ** 3},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": samples[0]["sample"] + "; the Rust reference cannot be built here (no cargo), "
                                   "so this is the oracle's C++ restatement of its loops"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


ENS_METRIC = "Gcell-updates/s (heat ensemble, 512 uneven grids of 16..128 cells per axis, FP32 fields + FP64 audit)"


def init_dist(local):
    import datetime

    import torch
    import torch.distributed as dist

    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return dist


def run_ensemble(args):
    """Config 4: every grid its own `Solid3D` with Dirichlet 300 K films and dt at 0.9 of its own
    limit; one bench step = `timesteps` steps of every grid (one persistent brick-list kernel
    launch per timestep, graphs of 64), FP64 ledger and audit per grid every timestep."""
    import numpy as np
    import torch

    from pantometry_b200 import sharding
    from pantometry_b200 import workloads as W
    from pantometry_b200.domains import Ensemble

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = init_dist(local) if world > 1 else None
    cfg = W.heat_ensemble(count=args.grids, steps=args.timesteps)
    all_grids = W.ensemble_grids(cfg)
    sizes = [int(np.prod(g["counts"])) for g in all_grids]
    share = sharding.partition(sizes, world)[rank]
    grids = [all_grids[g] for g in share]
    cells = np.concatenate([W.ensemble_cells(cfg["grids"][g]) for g in share])
    total_cells = sum(sizes)
    T = args.timesteps
    stream = torch.cuda.Stream(device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def build(precision):
        e = Ensemble(grids, precision=precision, device=local)
        e.set_stream(stream.cuda_stream)
        e.upload(cells)
        return e

    def timed(e, k, w, tol):
        e.set_tolerance(tol)
        for _ in range(w):
            v = e.step(T)
            assert v is None, v
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            start.record(stream)
            for _ in range(k):
                v = e.step(T)
                assert v is None, v
            end.record(stream)
            torch.cuda.synchronize()
        ms = start.elapsed_time(end)
        barrier()
        return max_over_ranks(ms), clk

    e32 = build("f32")
    shape32 = e32.autotune(trial_steps=10)
    ms32, clk = timed(e32, args.steps, args.warmup, 1e-6)
    plain_steps = max(1, args.steps // 2)
    e64 = build("f64")
    shape64 = e64.autotune(trial_steps=5)
    ms64, _ = timed(e64, plain_steps, max(1, args.warmup // 2), 1e-9)
    # error of FP32 against the f64 form after one bench step from the same start
    e32.upload(cells)
    e64.upload(cells)
    assert e32.step(T) is None and e64.step(T) is None
    field_err = float(np.abs(e32.download() - e64.download()).max())
    led32, led64 = e32.ledgers(), e64.ledgers()
    ledger_err = max(abs(a["total"] - b["total"]) / max(abs(b["total"]), b["scale"], 1e-300) for a, b in zip(led32, led64))
    del e64

    # e2e through the C ABI with host buffers: upload from pinned memory, run, ledgers back
    pinned = torch.empty(cells.size, dtype=torch.float64, pin_memory=True).numpy()
    pinned[:] = cells
    for _ in range(args.warmup):
        e32.upload(pinned)
        e32.step(T)
    barrier()
    t0 = time.perf_counter()
    s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        e32.upload(pinned)
        v = e32.step(T)
        assert v is None, v
        ledgers = sharding.gather_ledgers(e32.ledgers(), share, len(all_grids), dist)
    e0.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    e2e_ms = max_over_ranks(max(s0.elapsed_time(e0), wall_ms))
    del e32
    assert len(ledgers) == len(all_grids)

    peak, peak_kind = peaks()
    local_cells = int(cells.size)
    per_launch_ms = ms32 / (args.steps * T)
    achieved = 8 * local_cells / (per_launch_ms * 1e-3) / 1e9
    value = total_cells * T * args.steps / (ms32 * 1e-3) / 1e9
    plain = total_cells * T * plain_steps / (ms64 * 1e-3) / 1e9
    tma = tuple(shape32[:2]) == (32, 8)  # the 32 × 8 bricks run the TMA-staged kernel
    line = {
        "metric": ENS_METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms32 / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak" if world == 1 else "strong",
        "vs_baseline": None,
        "dtype": "f32 fields, f64 audit",
        "data": "synthetic (seeded Rng::for_index sizes, diffusivities and hot spots)",
        "config": {"workload": f"heat ensemble: {len(all_grids)} grids, 16..128 cells per axis, {total_cells} cells, "
                               f"{T} timesteps per step, Dirichlet 300 K faces, dt 0.9 x each grid's limit, "
                               "FP64 audit per grid every timestep",
                   "grids": len(all_grids), "cells": total_cells, "timesteps_per_step": T,
                   "parallelism": f"grids sharded over {world} rank(s)", "brick_f32": list(shape32),
                   "brick_f64": list(shape64), "l2": f"state {8 * total_cells / 1e9:.2f} GB > 126 MB L2, no flush",
                   "grids_per_s": round(len(all_grids) * args.steps / (ms32 * 1e-3), 3)},
        "e2e": {"value": round(total_cells * T * args.steps / (e2e_ms * 1e-3) / 1e9, 3), "unit": UNIT,
                "h2d_bytes_per_step": local_cells * 8, "d2h_bytes_per_step": len(grids) * 56},
        "gpu_launches": args.steps * T * (2 if tma else 1),  # the TMA step and its books kernel
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": round(ENS_F32_TRAFFIC_PER_CELL * local_cells) if tma else None,
                     "traffic_source": "ncu capture of the 512-grid ensemble, per cell",
                     "kernel": "ens_tma_step (FP32, TMA-staged)" if tma else
                               "ens_step<float> (four cells per thread)" if shape32[0] * shape32[1] == 1024 else "ens_step<float>",
                     "bytes_per_launch": 8 * local_cells, "peak_source": f"{peak_kind} hbm_gbs"},
        "plain_f64": {"value": round(plain, 3), "unit": UNIT, "ms_per_step": round(ms64 / plain_steps, 3),
                      "roofline_frac": round(16 * local_cells / (ms64 / (plain_steps * T) * 1e-3) / 1e9 / peak, 4),
                      "fp32_over_f64": round(value / plain, 3)},
        "error_vs_f64": {"max_abs_kelvin": field_err, "ledger_rel_max_over_grids": ledger_err, "after_timesteps": T},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_ensemble(cfg, all_grids, sample_steps=args.cpu_sample_steps, threads=1,
                                                     sample_grids=48)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


HEAT_METRIC = "Gcell-updates/s (heat block 64^3, plain f64, energy audit every step)"


def run_heat(args):
    """Config 1: a 64³ block (or `--n`) of the heat substance with Dirichlet 300 K films on every
    face and a 50 K Gaussian hot spot at a seed-jittered point, dt at 0.9 of the limit; one bench
    step = `timesteps` audited steps. `value` is the plain f64 form the config names; the FP32
    form (four cells per thread where the rows allow) is reported beside it. The 64³ state fits
    in L2, so L2 is flushed before every bench step, outside the events that time it."""
    import numpy as np
    import torch

    from pantometry_b200 import workloads as W

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = init_dist(local) if world > 1 else None
    n, T = args.n, args.timesteps
    cfg = W.heat_block(n, steps=T)
    cells = n ** 3
    stream = torch.cuda.Stream(device=local)
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device=local)  # 256 MB, twice the L2

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(precision, k, w, tol):
        b = W.build_heat(cfg, precision=precision, device=local)
        b.set_stream(stream.cuda_stream)
        b.set_tolerance(tol)
        dt = cfg["dt_fraction"] * b.max_stable_dt()
        for _ in range(w):
            v = b.step(dt, T)
            assert v is None, v
        barrier()
        ms = 0.0
        with Clocks(local) as clk:
            for _ in range(k):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                v = b.step(dt, T)
                assert v is None, v
                end.record(stream)
                torch.cuda.synchronize()
                ms += start.elapsed_time(end)
        barrier()
        return b, dt, max_over_ranks(ms), clk

    b64, dt, ms64, clk = timed("f64", args.steps, args.warmup, 1e-9)
    field64, led64 = b64.cells, b64.ledger()
    kernel64, launches64 = b64.step_kernel(T)  # what each bench step ran, as the library reports it
    del b64
    b32, _, ms32, _ = timed("f32", args.steps, args.warmup, 1e-6)
    kernel32, launches32 = b32.step_kernel(T)
    del b32
    # FP32 against f64 after the same steps from the same start
    a32, _, _, _ = timed("f32", 0, args.warmup + args.steps, 1e-6)
    field_err = float(np.abs(a32.cells - field64).max())
    l32 = a32.ledger()
    ledger_err = abs(l32["total"] - led64["total"]) / max(abs(led64["total"]), led64["scale"], 1e-300)
    del a32

    # e2e through the C ABI with host buffers: the block's kelvin from pinned memory, the run, the
    # ledger back, every bench step
    b = W.build_heat(cfg, precision="f64", device=local)
    b.set_stream(stream.cuda_stream)
    b.set_tolerance(1e-9)
    pinned = torch.empty(cells, dtype=torch.float64, pin_memory=True).numpy()
    pinned[:] = cfg["cells"]
    for _ in range(args.warmup):
        b.cells = pinned
        b.step(dt, T)
    barrier()
    t0 = time.perf_counter()
    s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        b.cells = pinned
        v = b.step(dt, T)
        assert v is None, v
        b.ledger()
    e0.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    e2e_ms = max_over_ranks(max(s0.elapsed_time(e0), wall_ms))
    del b

    peak, peak_kind = peaks()
    value = world * cells * T * args.steps / (ms64 * 1e-3) / 1e9
    fp32 = world * cells * T * args.steps / (ms32 * 1e-3) / 1e9
    line = {
        "metric": HEAT_METRIC.replace("64^3", f"{n}^3"), "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms64 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (300 K block, 50 K Gaussian hot spot, sigma 8 cells, seed-jittered centre)",
        "config": {"workload": f"heat_block {n}^3 cells, diffusivity 1e-4 m^2/s, dx 1 mm, dt 0.9 x the limit, "
                               f"Dirichlet 300 K faces, {T} timesteps per step, energy audit every timestep",
                   "cells": cells, "timesteps_per_step": T, "parallelism": f"replicas x{world}",
                   "l2": f"state {16 * cells / 1e6:.1f} MB (f64, both parities); L2 flushed before every bench step, "
                         "outside the timed events"},
        "e2e": {"value": round(world * cells * T * args.steps / (e2e_ms * 1e-3) / 1e9, 3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * cells, "d2h_bytes_per_step": 64},
        "gpu_launches": args.steps * launches64,
        "roofline": {"bound": "hbm", "achieved": round(16 * cells * T * args.steps / (ms64 * 1e-3) / 1e9, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(16 * cells * T * args.steps / (ms64 * 1e-3) / 1e9 / peak, 4), "traffic": None,
                     "kernel": f"{kernel64} (f64)", "bytes_per_step": 16 * cells,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "note": "L2-resident within a bench step at 64^3" if 16 * cells < 126e6 else "state larger than L2"},
        "fp32": {"value": round(fp32, 3), "unit": UNIT, "ms_per_step": round(ms32 / args.steps, 3),
                 "kernel": kernel32, "gpu_launches": args.steps * launches32,
                 "roofline_frac": round(8 * cells * T * args.steps / (ms32 * 1e-3) / 1e9 / peak, 4),
                 "fp32_over_f64": round(fp32 / value, 3)},
        "error_vs_f64": {"max_abs_kelvin": field_err, "ledger_rel": ledger_err,
                         "after_timesteps": T * (args.warmup + args.steps)},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_heat(cfg, T if n <= 64 else args.cpu_sample_steps)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline_heat(cfg, sample_steps):
    """`Simulation::advance` over the block's `Solid3D::step` and its ledger, restated (the
    oracle), one core."""
    import oracle

    nx, ny, nz = cfg["counts"]
    s = cfg["substance"]
    o = oracle.Heat(cfg["counts"], cfg["dx"], s["density"], s["conductivity"], s["specific_heat"], cfg["initial"],
                    emissivity=s["emissivity"])
    for f, amb, h, area in cfg["films"]:
        o.losing_from(f, amb, h, area)
    o.cells = cfg["cells"]
    dt = cfg["dt_fraction"] * o.max_stable_dt()
    assert o.advance(dt, 1, tol=1e-9) is None  # warm-up
    t0 = time.perf_counter()
    assert o.advance(dt, sample_steps, tol=1e-9) is None
    secs = time.perf_counter() - t0
    cells = nx * ny * nz
    return {"value": round(cells * sample_steps / secs / 1e9, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"the {nx}x{ny}x{nz} block, {sample_steps} audited Simulation::advance steps "
                      f"(after 1 warm-up step), 1 thread, {secs:.2f} s"}


CAV_METRIC = "Gcell-updates/s (Yee cavity 384^3, FP32 fields + FP64 audit)"


def heat_block_record(local, stream, peak, n=64, timesteps=1000, steps=5, warmup=3):
    """The heat block of config 1 (n³ cells, Dirichlet 300 K faces, a 50 K Gaussian hot spot at a
    seed-jittered point, dt at 0.9 of the limit) as an object of the default line: the plain f64 form
    the configuration names and the FP32 form, each `steps` calls of `timesteps` audited timesteps
    after `warmup` calls, L2 flushed before each call outside the events (the 64³ state fits in L2);
    the FP32 field and books against the f64 run's after the same calls from the same start."""
    import numpy as np
    import torch

    from pantometry_b200 import workloads as W

    cfg = W.heat_block(n, steps=timesteps)
    cells = n ** 3
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device=local)  # 256 MB, twice the L2

    def run(precision, tol):
        b = W.build_heat(cfg, precision=precision, device=local)
        b.set_stream(stream.cuda_stream)
        b.set_tolerance(tol)
        dt = cfg["dt_fraction"] * b.max_stable_dt()
        for _ in range(warmup):
            assert b.step(dt, timesteps) is None
        ms = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            v = b.step(dt, timesteps)
            assert v is None, v
            end.record(stream)
            torch.cuda.synchronize()
            ms += start.elapsed_time(end)
        return b, ms

    b64, ms64 = run("f64", 1e-9)
    b32, ms32 = run("f32", 1e-6)
    kernel64, launches64 = b64.step_kernel(timesteps)
    kernel32, _ = b32.step_kernel(timesteps)
    l64, l32 = b64.ledger(), b32.ledger()
    field_err = float(np.abs(b32.cells - b64.cells).max())
    ledger_err = abs(l32["total"] - l64["total"]) / max(abs(l64["total"]), l64["scale"], 1e-300)
    del b64, b32, flush
    us64, us32 = ms64 * 1e3 / (steps * timesteps), ms32 * 1e3 / (steps * timesteps)
    return {
        "workload": f"heat_block {n}^3 cells, diffusivity 1e-4 m^2/s, dx 1 mm, dt 0.9 x the limit, Dirichlet 300 K "
                    f"faces, {timesteps} audited timesteps per call, L2 flushed before each call",
        "value": round(cells * timesteps * steps / (ms64 * 1e-3) / 1e9, 3), "unit": UNIT, "dtype": "f64",
        "us_per_timestep": round(us64, 3), "grids_per_s": round(1e6 / us64, 1), "timed_calls": steps,
        "kernel": kernel64, "gpu_launches": steps * launches64,
        "fp32": {"value": round(cells * timesteps * steps / (ms32 * 1e-3) / 1e9, 3), "us_per_timestep": round(us32, 3),
                 "kernel": kernel32},
        "error_vs_f64": {"max_abs_kelvin": field_err, "ledger_rel": ledger_err,
                         "after_timesteps": timesteps * (warmup + steps)},
        "note": "state 4.2 MB (f64, both parities): L2-resident within a call, bound by the per-step grid wait",
    }


def ensemble_record(local, stream, peak, timesteps=2000, steps=2):
    """The heat ensemble (512 uneven blocks of 16..128 cells per axis, Dirichlet 300 K films, dt at
    0.9 of each block's own limit, FP64 books and audit per block every timestep) as an object of the
    default line: the FP32 form (brick shape autotuned) over `steps` runs of `timesteps` timesteps and
    the plain f64 form over one, device-resident, CUDA events on the ensemble's stream; the FP32
    fields and books against the f64 run's after one run from the same start."""
    import numpy as np
    import torch

    from pantometry_b200 import workloads as W
    from pantometry_b200.domains import Ensemble

    cfg = W.heat_ensemble(count=512, steps=timesteps)
    grids = W.ensemble_grids(cfg)
    cells = np.concatenate([W.ensemble_cells(g) for g in cfg["grids"]])
    total = int(cells.size)

    def run(precision, k, tol, tune):
        e = Ensemble(grids, precision=precision, device=local)
        e.set_stream(stream.cuda_stream)
        e.upload(cells)
        shape = e.autotune(trial_steps=tune)
        e.upload(cells)
        e.set_tolerance(tol)
        assert e.step(64) is None  # warm-up: graphs captured
        e.upload(cells)
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for q in range(k):
            v = e.step(timesteps)
            assert v is None, v
        end.record(stream)
        torch.cuda.synchronize()
        return e, start.elapsed_time(end), shape

    e32, ms32, shape32 = run("f32", steps, 1e-6, 10)
    e64, ms64, shape64 = run("f64", 1, 1e-9, 5)
    # both hold one run from the same start after their first timed run; the FP32 one has run more
    e32.upload(cells)
    assert e32.step(timesteps) is None
    d32, d64 = e32.download(), e64.download()
    l32, l64 = e32.ledgers(), e64.ledgers()
    ledger_err = max(abs(a["total"] - b["total"]) / max(abs(b["total"]), b["scale"], 1e-300) for a, b in zip(l32, l64))
    field_err = float(np.abs(d32 - d64).max())
    del e32, e64
    value = total * timesteps * steps / (ms32 * 1e-3) / 1e9
    plain = total * timesteps / (ms64 * 1e-3) / 1e9
    achieved = 8 * total / (ms32 / (steps * timesteps) * 1e-3) / 1e9
    tma = tuple(shape32[:2]) == (32, 8)
    return {
        "workload": f"heat ensemble: 512 grids, 16..128 cells per axis, {total} cells, {timesteps} timesteps per run, "
                    "Dirichlet 300 K faces, dt 0.9 x each grid's limit, FP64 audit per grid every timestep",
        "value": round(value, 3), "unit": UNIT, "timed_runs": steps, "ms_per_run": round(ms32 / steps, 3),
        "brick_f32": list(shape32), "brick_f64": list(shape64),
        "plain_f64": {"value": round(plain, 3), "ms_per_run": round(ms64, 3),
                      "roofline_frac": round(16 * total / (ms64 / timesteps * 1e-3) / 1e9 / peak, 4)},
        "fp32_over_f64": round(value / plain, 3),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "kernel": "ens_tma_step (FP32, TMA-staged)" if tma else "ens_step<float>",
                     "bytes_per_timestep": 8 * total,
                     "traffic": round(ENS_F32_TRAFFIC_PER_CELL * total) if tma else None,
                     "traffic_source": "ncu capture of the 512-grid ensemble, per cell"},
        "error_vs_f64": {"max_abs_kelvin": field_err, "ledger_rel_max_over_grids": ledger_err, "after_timesteps": timesteps},
    }


def cavity_record(local, stream, peak, n=384, timed_steps=2000, compare_steps=10000, every=10):
    """The Yee cavity (n³ cells, vacuum, conducting walls, Courant 0.99/√3, the soft dipole current)
    as an object of the default line. Throughput: `timed_steps` audited timesteps of the FP32 and
    of the plain f64 form, device-resident, after 128 warm-up steps (CUDA events on the handle's
    stream). Error: an FP32 and an f64 cavity stepped side by side `every` steps at a time for
    `compare_steps` steps, the FP32 ledger against the f64 one at each comparison, relative to the
    f64 ledger's scale then (its largest entry, the audit's own scale)."""
    import torch

    from pantometry_b200 import workloads as W

    cfg = W.yee_cavity(n, steps=compare_steps + 128 + timed_steps)
    cells = n ** 3
    dt = cfg["dt"]

    tiles = {}

    def timed(precision, tol):
        c = W.build_cavity(cfg, precision=precision, device=local)
        c.set_stream(stream.cuda_stream)
        if precision == "f32":  # the TMA kernel's tile shape, timed on this grid
            tiles[precision] = list(c.autotune(trial_steps=8))
        c.set_tolerance(tol)
        assert c.step(dt, 128) is None
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        v = c.step(dt, timed_steps)
        end.record(stream)
        torch.cuda.synchronize()
        assert v is None, v
        del c
        return start.elapsed_time(end)

    ms32 = timed("f32", 1e-6)
    ms64 = timed("f64", 1e-9)
    runs = {}
    for p, tol in (("f32", 1e-6), ("f64", 1e-9)):
        runs[p] = W.build_cavity(cfg, precision=p, device=local)
        runs[p].set_stream(stream.cuda_stream)
        runs[p].set_tolerance(tol)
    worst, at = 0.0, 0
    for q in range(compare_steps // every):
        for c in runs.values():
            v = c.step(dt, every)
            assert v is None, v
        a, b = runs["f32"].ledger(), runs["f64"].ledger()
        gap = abs(a["total"] - b["total"]) / max(b["scale"], 1e-300)
        if gap > worst:
            worst, at = gap, (q + 1) * every
    final = abs(a["total"] - b["total"]) / max(b["scale"], 1e-300)
    del runs
    value = cells * timed_steps / (ms32 * 1e-3) / 1e9
    plain = cells * timed_steps / (ms64 * 1e-3) / 1e9
    achieved = 48 * cells / (ms32 / timed_steps * 1e-3) / 1e9
    return {
        "workload": f"yee_cavity {n}^3 cells, vacuum, conducting walls, Courant 0.99/sqrt(3), soft z-current at the "
                    f"centre Ez edge (its 5^3 near field in f64), FP64 audit every timestep",
        "value": round(value, 3), "unit": UNIT, "timed_timesteps": timed_steps,
        "ms_per_timestep": round(ms32 / timed_steps, 4), "tile_planes_stages": tiles.get("f32"),
        "plain_f64": {"value": round(plain, 3), "ms_per_timestep": round(ms64 / timed_steps, 4),
                      "roofline_frac": round(96 * cells / (ms64 / timed_steps * 1e-3) / 1e9 / peak, 4)},
        "fp32_over_f64": round(value / plain, 3),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "kernel": "yee_tma_step + yee_near_step (FP32)",
                     "bytes_per_timestep": 48 * cells,
                     "traffic": round(YEE_F32_TRAFFIC_PER_CELL * cells), "traffic_source": "ncu capture at 256^3, scaled by cells"},
        "error_vs_f64": {"ledger_rel": worst, "at_timestep": at, "final_ledger_rel": final,
                         "compared_every": every, "over_timesteps": compare_steps},
    }


def run_cavity(args):
    """Config 3: a vacuum cavity of n³ cells with conducting walls, Courant 0.99/√3, and the soft
    z-current on the centre Ez edge; one bench step = `timesteps` steps, each with the fused FP64
    invariant and the audit (tolerance 1e-5, FP32)."""
    import numpy as np
    import torch

    from pantometry_b200 import workloads as W

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = init_dist(local) if world > 1 else None
    n, T = args.n, args.timesteps
    cfg = W.yee_cavity(n, steps=T * (args.steps + args.warmup + 1))
    cells = n ** 3
    stream = torch.cuda.Stream(device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(precision, k, w, tol):
        c = W.build_cavity(cfg, precision=precision, device=local)
        c.set_stream(stream.cuda_stream)
        c.set_tolerance(tol)
        for _ in range(w):
            v = c.step(cfg["dt"], T)
            assert v is None, v
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            start.record(stream)
            for _ in range(k):
                v = c.step(cfg["dt"], T)
                assert v is None, v
            end.record(stream)
            torch.cuda.synchronize()
        ms = start.elapsed_time(end)
        barrier()
        return c, max_over_ranks(ms), clk

    c32, ms32, clk = timed("f32", args.steps, args.warmup, 1e-5)
    del c32
    plain_steps = max(1, args.steps // 2)
    c64, ms64, _ = timed("f64", plain_steps, max(1, args.warmup // 2), 1e-9)
    del c64
    # FP32 against f64 after one bench step from the same start
    a32, _, _ = timed("f32", 0, 1, 1e-5)
    a64, _, _ = timed("f64", 0, 1, 1e-9)
    f32f, f64f = a32.fields(), a64.fields()
    # max |FP32 − f64| over E (and over H), relative to the largest |f64| value of that field
    e_scale = max(float(np.abs(f64f[q]).max()) for q in ("ex", "ey", "ez"))
    h_scale = max(float(np.abs(f64f[q]).max()) for q in ("hx", "hy", "hz"))
    field_err = max(max(float(np.abs(f32f[q] - f64f[q]).max()) for q in ("ex", "ey", "ez")) / max(e_scale, 1e-300),
                    max(float(np.abs(f32f[q] - f64f[q]).max()) for q in ("hx", "hy", "hz")) / max(h_scale, 1e-300))
    l32, l64 = a32.ledger(), a64.ledger()
    ledger_err = abs(l32["total"] - l64["total"]) / max(abs(l64["total"]), l64["scale"], 1e-300)
    del a32, a64, f32f, f64f

    # e2e through the C ABI with host buffers: the six fields from pinned memory, the run, the
    # ledger and Ez back every bench step
    c = W.build_cavity(cfg, precision="f32", device=local)
    c.set_stream(stream.cuda_stream)
    c.set_tolerance(1e-5)
    shapes = c.shapes()
    pinned = {q: torch.zeros(m, dtype=torch.float64, pin_memory=True).numpy() for q, m in shapes.items()}
    ez_out = torch.empty(shapes["ez"], dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(args.warmup):
        c.set_fields(pinned, started=False)
        c.step(cfg["dt"], T)
    barrier()
    t0 = time.perf_counter()
    s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        c.set_fields(pinned, started=False)
        v = c.step(cfg["dt"], T)
        assert v is None, v
        c.ledger()
        c.download_component("ez", ez_out)
    e0.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    e2e_ms = max_over_ranks(max(s0.elapsed_time(e0), wall_ms))
    del c

    peak, peak_kind = peaks()
    per_launch_ms = ms32 / (args.steps * T)
    achieved = 48 * cells / (per_launch_ms * 1e-3) / 1e9
    value = world * cells * T * args.steps / (ms32 * 1e-3) / 1e9
    plain = world * cells * T * plain_steps / (ms64 * 1e-3) / 1e9
    h2d = sum(m for m in shapes.values()) * 8
    line = {
        "metric": CAV_METRIC.replace("384^3", f"{n}^3"), "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms32 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 audit",
        "data": "synthetic (zero fields, Gaussian-modulated dipole current)",
        "config": {"workload": f"yee_cavity {n}^3 cells, vacuum, conducting walls, Courant 0.99/sqrt(3), "
                               f"{T} timesteps per step, soft z-current at the centre Ez edge, FP64 audit every timestep",
                   "cells": cells, "timesteps_per_step": T, "parallelism": f"replicas x{world}",
                   "l2": f"state {48 * cells / 2 / 1e9:.2f} GB > 126 MB L2, no flush"},
        "e2e": {"value": round(world * cells * T * args.steps / (e2e_ms * 1e-3) / 1e9, 3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": shapes["ez"] * 8 + 64},
        "gpu_launches": args.steps * T,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": round(YEE_F32_TRAFFIC_PER_CELL * cells),
                     "traffic_source": "ncu capture at 256^3, scaled by cells", "kernel": "yee_tma_step (FP32, TMA-staged)",
                     "bytes_per_launch": 48 * cells, "peak_source": f"{peak_kind} hbm_gbs"},
        "plain_f64": {"value": round(plain, 3), "unit": UNIT, "ms_per_step": round(ms64 / plain_steps, 3),
                      "roofline_frac": round(96 * cells / (ms64 / (plain_steps * T) * 1e-3) / 1e9 / peak, 4),
                      "fp32_over_f64": round(value / plain, 3)},
        "error_vs_f64": {"max_rel_field": field_err, "ledger_rel": ledger_err, "after_timesteps": T},
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_cavity()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def cavity_sample(n_sample, sample_steps, copies=1):
    """The reference's CPU path for the cavity (the oracle's audited `Simulation::advance` over
    `Cavity::step` with the soft z-current), `copies` independent n_sample³ cavities, one per
    thread; the oracle's cost per cell-update does not depend on the size, and a sample keeps the
    host memory bounded (about 0.4 GB per 128³ copy). Returns (Gcell-updates/s, seconds)."""
    import oracle
    from pantometry_b200 import workloads as W

    cfg = W.yee_cavity(n_sample, steps=sample_steps + 1)
    cavs = []
    for _ in range(copies):
        y = oracle.Yee(cfg["counts"], cfg["dx"])
        y.set_source(cfg["edge"], cfg["current"])
        assert y.advance(cfg["dt"], 1) is None  # warm-up
        cavs.append(y)
    refused = []

    def work(y):
        v = y.advance(cfg["dt"], sample_steps)
        if v is not None:
            refused.append(v)

    ths = [threading.Thread(target=work, args=(y,)) for y in cavs]
    t0 = time.perf_counter()
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    secs = time.perf_counter() - t0
    assert not refused, refused[0]
    return copies * n_sample ** 3 * sample_steps / secs / 1e9, secs


def cpu_baseline_cavity(n_sample=128, sample_steps=100):
    value, secs = cavity_sample(n_sample, sample_steps)
    return {"value": round(value, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"a {n_sample}^3 vacuum cavity with the same source, {sample_steps} audited Simulation::advance "
                      f"steps (after 1 warm-up step), 1 thread, {secs:.2f} s; the rate per cell-update"}


def run_reference_cavity(args):
    """The cavity's reference arm: `cavity_sample` on every usable host core (one independent
    128³ cavity per thread, at most 8 GB of host state), the median of `steps` samples."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    copies = max(1, min(ncpu, 20))
    steps = 20
    cavity_sample(128, 1, copies)  # warm-up
    runs = [cavity_sample(128, steps, copies) for _ in range(args.steps)]
    value = statistics.median(r[0] for r in runs)
    line = {
        "metric": CAV_METRIC.replace("384^3", f"{args.n}^3"), "value": round(value, 6), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (zero fields, Gaussian-modulated dipole current)", "impl": "reference",
        "config": {"workload": "yee_cavity, vacuum, conducting walls, Courant 0.99/sqrt(3), soft z-current, "
                               "audited Simulation::advance steps", "sample_cells": 128 ** 3, "copies": copies},
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": copies, "kind": "port",
                         "sample": f"{copies} independent 128^3 cavities, one per thread, {steps} audited steps each "
                                   f"per bench step (median of {args.steps}, {runs[0][1]:.2f} s for the first); the "
                                   "oracle's cost per cell-update does not depend on the size; the Rust reference "
                                   "cannot be built here (no cargo), so this is the oracle's C++ restatement of its loops"},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


MIX_METRIC = "Gcell-updates/s (1024^3 heterogeneous acoustic hall + 64 Yee 128^3 dielectric cavities, FP32 fields + FP64 audit)"


class CavityBatch:
    """The 64 cavities of the mixed workload, each its own handle, spread over `lanes` CUDA streams
    with one host thread per stream (a step call returns once its stream has finished)."""

    def __init__(self, cfg, precision, device, lanes=8):
        import torch

        from pantometry_b200 import workloads as W

        self.cfg = cfg
        self.cavs = [W.build_dielectric_cavity(cfg, g, precision=precision, device=device)
                     for g in range(len(cfg["cavities"]))]
        self.streams = [torch.cuda.Stream(device=device) for _ in range(min(lanes, len(self.cavs)))]
        for g, c in enumerate(self.cavs):
            c.set_stream(self.streams[g % len(self.streams)].cuda_stream)

    def set_tolerance(self, tol):
        for c in self.cavs:
            c.set_tolerance(tol)

    def run(self, dt, T, before=None, each=None):
        """Every cavity `T` steps; `before(g, c)` / `each(g, c)` around each cavity's run."""
        L = len(self.streams)
        errors = []

        def lane(q):
            try:
                for g in range(q, len(self.cavs), L):
                    c = self.cavs[g]
                    if before:
                        before(g, c)
                    v = c.step(dt, T)
                    assert v is None, v
                    if each:
                        each(g, c)
            except BaseException as e:  # noqa: BLE001
                errors.append(e)

        ths = [threading.Thread(target=lane, args=(q,)) for q in range(L)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        if errors:
            raise errors[0]

    def timed(self, dt, T, k, start_stream, **kw):
        """`k` runs between two events on `start_stream`; every lane waits on the start event and
        the end event waits on every lane."""
        import torch

        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(start_stream)
        for s in self.streams:
            s.wait_event(start)
        for _ in range(k):
            self.run(dt, T, **kw)
        for s in self.streams:
            e = torch.cuda.Event()
            e.record(s)
            start_stream.wait_event(e)
        end.record(start_stream)
        return start, end

    def close(self):
        for c in self.cavs:
            c.close()
        self.cavs = []


def mix_sample(hall_cells, cav_cells, n_sample=128, sample_steps=32, copies=1):
    """The reference's CPU path (the oracle) on a bounded sample of the mixed workload: `copies`
    independent pairs of an `n_sample`³ hall over the same 32³ speed blocks and an `n_sample`³
    dielectric cavity, one pair per thread, `sample_steps` audited steps of every hall and then of
    every cavity, each phase timed by the wall clock. Returns the mix's rate (its cell-updates over
    the time the measured costs per cell give for its hall and cavity cells) and those costs."""
    import oracle
    from pantometry_b200 import workloads as W

    h = W.hetero_hall(n_sample, steps=sample_steps + 1)
    c = W.dielectric_cavities(1, n_sample, steps=sample_steps + 1)
    w, ht, d = h["size"]
    halls, cavs = [], []
    for _ in range(copies):
        o = oracle.Hall(w, ht, d, h["across"], h["speed"], h["density"])
        o.release(h["pressure"])
        o.set_speed_blocks(h["block"], h["speeds"])
        o.set_source(h["source_node"], h["wave"])
        assert o.advance(h["dt"], 1) is None
        halls.append(o)
        y = oracle.Yee(c["counts"], c["dx"])
        y.set_cells(eps_r=c["cavities"][0]["eps"])
        y.set_source(c["edge"], c["current"])
        assert y.advance(c["dt"], 1) is None
        cavs.append(y)

    def phase(objs, dt):
        refused = []

        def work(o):
            v = o.advance(dt, sample_steps)
            if v is not None:
                refused.append(v)

        ths = [threading.Thread(target=work, args=(o,)) for o in objs]
        t0 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        assert not refused, refused[0]
        return (time.perf_counter() - t0) / (copies * n_sample ** 3 * sample_steps)

    t_hall = phase(halls, h["dt"])
    t_cav = phase(cavs, c["dt"])
    value = (hall_cells + cav_cells) / (t_hall * hall_cells + t_cav * cav_cells) / 1e9
    return value, t_hall, t_cav


def cpu_baseline_mix(hall_cells, cav_cells, n_sample=128, sample_steps=32):
    value, t_hall, t_cav = mix_sample(hall_cells, cav_cells, n_sample, sample_steps)
    return {"value": round(value, 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{sample_steps} audited Simulation::advance steps of a {n_sample}^3 speed-block hall "
                      f"({t_hall * 1e9:.1f} ns per node-update) and of a {n_sample}^3 dielectric cavity "
                      f"({t_cav * 1e9:.1f} ns per cell-update), weighted by the mix's cells"}


def run_reference_mix(args):
    """The mix's reference arm: `mix_sample` on every usable host core (one hall and one cavity of
    128³ per thread, at most 8 pairs), weighted by the mix's cells, the median of `steps` samples."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    copies = max(1, min(ncpu, 8))
    hall_cells, cav_cells = args.n ** 3, args.grids * args.cavity_n ** 3
    runs = [mix_sample(hall_cells, cav_cells, 128, 8, copies) for _ in range(args.steps)]
    value = statistics.median(r[0] for r in runs)
    line = {
        "metric": MIX_METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded speed blocks, inclusions and noise; Ricker and dipole sources)", "impl": "reference",
        "config": {"workload": f"{args.n}^3 speed-block hall + {args.grids} dielectric cavities of {args.cavity_n}^3, "
                               "audited Simulation::advance steps", "copies": copies},
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": copies, "kind": "port",
                         "sample": f"{copies} independent pairs of a 128^3 speed-block hall and a 128^3 dielectric "
                                   f"cavity, one pair per thread, 8 audited steps of each per bench step "
                                   f"({runs[0][1] * 1e9:.1f} and {runs[0][2] * 1e9:.1f} ns of wall clock per "
                                   "node- and cell-update), weighted by the mix's cells; the Rust reference cannot be "
                                   "built here (no cargo), so this is the oracle's C++ restatement of its loops"},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_mix(args):
    """Config 5 on one GPU: the 1024³ acoustic hall in FP32 over a medium of 32³-node blocks with c
    uniform in [300, 1500] m/s (CFL 0.5 of the fastest block, 1 Pa Ricker at the centre, ±1 mPa
    noise), then 64 Yee cavities of 128³ cells in FP32 with ε_r uniform in [1, 4] in 10% of the
    cells (Courant 0.99/√3, the dipole current at the centre edge); every timestep of both audited
    in FP64. One bench step = `timesteps` steps of the hall followed by `timesteps` steps of every
    cavity."""
    import numpy as np
    import torch

    from pantometry_b200 import workloads as W

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = init_dist(local) if world > 1 else None
    n, T, K, Wm = args.n, args.timesteps, args.steps, args.warmup
    total_steps = T * (K + Wm + 2)
    hcfg = W.hetero_hall(n, steps=total_steps)
    ccfg = W.dielectric_cavities(args.grids, args.cavity_n, steps=total_steps)
    hall_cells = n ** 3
    cav_cells = len(ccfg["cavities"]) * args.cavity_n ** 3
    stream = torch.cuda.Stream(device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def hall_run(h, k):
        for _ in range(k):
            v = h.step(hcfg["dt"], T)
            assert v is None, v

    # ---- FP32, device-resident: K bench steps after Wm warm-up steps
    hall = W.build_hetero_hall(hcfg, precision="f32", device=local)
    hall.set_stream(stream.cuda_stream)
    hall.set_tolerance(1e-5)
    cavs = CavityBatch(ccfg, "f32", local)
    cavs.set_tolerance(1e-5)
    for _ in range(Wm):
        hall_run(hall, 1)
        cavs.run(ccfg["dt"], T)
    barrier()
    with Clocks(local) as clk:
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms_hall = ms_cav = 0.0
        for _ in range(K):
            h0.record(stream)
            hall_run(hall, 1)
            h1.record(stream)
            c0, c1 = cavs.timed(ccfg["dt"], T, 1, stream)
            torch.cuda.synchronize()
            ms_hall += h0.elapsed_time(h1)
            ms_cav += c0.elapsed_time(c1)
    barrier()
    ms_hall, ms_cav = max_over_ranks(ms_hall), max_over_ranks(ms_cav)
    ms32 = max_over_ranks(ms_hall + ms_cav)

    # ---- e2e through the C ABI with host buffers: the hall's pressure and every cavity's six
    # fields from pinned memory, the runs, the hall's pressure and every ledger back, each step
    p_pin = torch.empty(hall_cells, dtype=torch.float64, pin_memory=True).numpy()
    p_pin[:] = hcfg["pressure"]
    p_out = torch.empty(hall_cells, dtype=torch.float64, pin_memory=True).numpy()
    shapes = cavs.cavs[0].shapes()
    zero = {q: torch.zeros(m, dtype=torch.float64, pin_memory=True).numpy() for q, m in shapes.items()}
    barrier()
    t0 = time.perf_counter()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(K):
        hall.release(p_pin)
        hall_run(hall, 1)
        hall.ledger()
        hall.download_pressure(p_out)
        cavs.run(ccfg["dt"], T, before=lambda g, c: c.set_fields(zero, started=False), each=lambda g, c: c.ledger())
    s1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(max(s0.elapsed_time(s1), (time.perf_counter() - t0) * 1e3))
    hall.close()
    cavs.close()
    del hall, cavs, p_pin, p_out

    # ---- drift against the f64 form (bit-exact with the oracle): one bench step of each from the
    # same start; the plain f64 rate from the same runs
    def one(precision, tol):
        h = W.build_hetero_hall(hcfg, precision=precision, device=local)
        h.set_stream(stream.cuda_stream)
        h.set_tolerance(tol)
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        hall_run(h, 1)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        out = np.empty(hall_cells, dtype=np.float64)
        h.download_pressure(out)
        led = h.ledger()
        h.close()
        return out, led, ms

    p32, l32, _ = one("f32", 1e-5)
    p64, l64, ms64_hall = one("f64", 1e-9)
    scale = float(np.abs(p64).max())
    hall_err = float(np.abs(p32 - p64).max()) / max(scale, 1e-300)
    hall_drift = abs(l32["total"] - l64["total"]) / max(abs(l64["total"]), l64["scale"], 1e-300)
    del p32, p64

    def cav_fields(precision, tol):
        b = CavityBatch(ccfg, precision, local)
        b.set_tolerance(tol)
        barrier()
        c0, c1 = b.timed(ccfg["dt"], T, 1, stream)
        torch.cuda.synchronize()
        ms = c0.elapsed_time(c1)
        got = [(c.fields(), c.ledger()) for c in b.cavs[:4]]
        b.close()
        return got, ms

    f32c, _ = cav_fields("f32", 1e-5)
    f64c, ms64_cav = cav_fields("f64", 1e-9)
    cav_err = cav_drift = 0.0
    for (fa, la), (fb, lb) in zip(f32c, f64c):
        for fam in (("ex", "ey", "ez"), ("hx", "hy", "hz")):
            sc = max(float(np.abs(fb[q]).max()) for q in fam)
            cav_err = max(cav_err, max(float(np.abs(fa[q] - fb[q]).max()) for q in fam) / max(sc, 1e-300))
        cav_drift = max(cav_drift, abs(la["total"] - lb["total"]) / max(abs(lb["total"]), lb["scale"], 1e-300))
    ms64 = max_over_ranks(ms64_hall + ms64_cav)

    peak, peak_kind = peaks()
    updates = hall_cells * T + cav_cells * T
    value = world * updates * K / (ms32 * 1e-3) / 1e9
    plain = world * updates / (ms64 * 1e-3) / 1e9
    hall_rate = hall_cells * T * K / (ms_hall * 1e-3) / 1e9
    cav_rate = cav_cells * T * K / (ms_cav * 1e-3) / 1e9
    per_launch_ms = ms_hall / (K * T)
    achieved = BYTES_F32 * hall_cells / (per_launch_ms * 1e-3) / 1e9
    # whole-step algorithmic bytes: 32 B per hall node-update; per cavity cell-update 48 B of fields
    # and 12 B of per-edge gains (f32, which also weigh the audit's electric terms)
    step_bytes = T * (BYTES_F32 * hall_cells + 60 * cav_cells)
    h2d = hall_cells * 8 + len(ccfg["cavities"]) * sum(shapes.values()) * 8
    d2h = hall_cells * 8 + 64 * (1 + len(ccfg["cavities"]))
    line = {
        "metric": MIX_METRIC.replace("1024^3", f"{n}^3").replace("64 Yee 128^3", f"{len(ccfg['cavities'])} Yee {args.cavity_n}^3"),
        "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": Wm,
        "ms_per_step": round(ms32 / K, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 fields, f64 audit",
        "data": "synthetic (seeded Rng::for_index block speeds, noise, inclusions and eps_r; Ricker and dipole sources)",
        "config": {"workload": f"hetero acoustic_hall {n}^3 nodes (c per 32^3 block in [300, 1500] m/s, CFL 0.5) "
                               f"+ {len(ccfg['cavities'])} yee_cavity {args.cavity_n}^3 cells (eps_r in [1, 4] in 10% of "
                               f"cells), {T} timesteps of each per step, FP64 audit every timestep",
                   "cells": hall_cells + cav_cells, "timesteps_per_step": T, "parallelism": f"replicas x{world}",
                   "l2": f"state {(16 * hall_cells + 24 * cav_cells) / 1e9:.1f} GB > 126 MB L2, no flush"},
        "e2e": {"value": round(world * updates * K / (e2e_ms * 1e-3) / 1e9, 3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": K * T * (1 + len(ccfg["cavities"])),
        "parts": {"hall": {"value": round(hall_rate, 3), "ms_per_step": round(ms_hall / K, 3)},
                  "cavities": {"value": round(cav_rate, 3), "ms_per_step": round(ms_cav / K, 3)}},
        "hbm_frac_whole_step": round(step_bytes / (ms32 / K * 1e-3) / 1e9 / peak, 4),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "kernel": "hall_tma_step (FP32, TMA-staged, speed blocks)",
                     "bytes_per_launch": BYTES_F32 * hall_cells, "peak_source": f"{peak_kind} hbm_gbs"},
        "plain_f64": {"value": round(plain, 3), "unit": UNIT, "fp32_over_f64": round(value / plain, 3)},
        "error_vs_f64": {"hall_max_rel_pressure": hall_err, "hall_ledger_rel": hall_drift,
                         "cavity_max_rel_field": cav_err, "cavity_ledger_rel": cav_drift, "after_timesteps": T,
                         "cavities_compared": len(f32c)},
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_mix(hall_cells, cav_cells)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline_ensemble(cfg, grids, sample_steps=2, threads=1, sample_grids=16):
    """`Ensemble::run` over `Solid3D` samples, restated (the oracle): the first `sample_grids`
    grids, each with its own audited `Simulation::advance` steps, `threads` grids at a time."""
    import queue

    import oracle
    from pantometry_b200 import workloads as W

    blocks = []
    for g in range(min(sample_grids, len(grids))):
        d = grids[g]
        nx, ny, nz = d["counts"]
        dx, s = d["dx"], d["substance"]
        o = oracle.Heat((nx, ny, nz), dx, s["density"], s["conductivity"], s["specific_heat"], d["initial"])
        areas = [(ny * dx) * (nz * dx)] * 2 + [(nx * dx) * (nz * dx)] * 2 + [(nx * dx) * (ny * dx)] * 2
        for f in range(6):
            o.losing_from(f, d["initial"], d["convection"], areas[f])
        o.cells = W.ensemble_cells(cfg["grids"][g])
        assert o.advance(d["dt"], 1) is None  # warm-up
        blocks.append((o, d["dt"], nx * ny * nz))
    work = queue.Queue()
    for b in blocks:
        work.put(b)

    def worker():
        while True:
            try:
                o, dt, _ = work.get_nowait()
            except queue.Empty:
                return
            assert o.advance(dt, sample_steps) is None

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    secs = time.perf_counter() - t0
    ncells = sum(b[2] for b in blocks)
    return {"value": round(ncells * sample_steps / secs / 1e9, 6), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(blocks)} grids ({ncells} cells) x {sample_steps} audited Simulation::advance steps "
                      f"(after 1 warm-up step), {threads} thread(s), {secs:.2f} s"}


def run_reference_heat(args):
    """The reference's CPU path for the heat block (the oracle's restatement of `Simulation::advance`
    over `Solid3D::step` and its ledger, audited at 1e-9), on every usable host core: one
    independent copy of the block per thread (the reference's `Ensemble` pattern), each bench step
    a sample of `sample_steps` audited steps of every copy."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    import oracle
    from pantometry_b200 import workloads as W

    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    n, T = args.n, args.timesteps
    cfg = W.heat_block(n, steps=T)
    cells = n ** 3
    copies = max(1, min(ncpu, int(8e9 // (16 * cells))))  # at most 8 GB of host state
    sample_steps = min(T, 100 if n <= 64 else args.cpu_sample_steps)
    s = cfg["substance"]
    blocks = []
    for _ in range(copies):
        o = oracle.Heat(cfg["counts"], cfg["dx"], s["density"], s["conductivity"], s["specific_heat"],
                        cfg["initial"], emissivity=s["emissivity"])
        for f, amb, h, area in cfg["films"]:
            o.losing_from(f, amb, h, area)
        o.cells = cfg["cells"]
        blocks.append(o)
    dt = cfg["dt_fraction"] * blocks[0].max_stable_dt()

    def sample(steps):
        refused = []

        def work(o):
            v = o.advance(dt, steps, tol=1e-9)
            if v is not None:
                refused.append(v)

        ths = [threading.Thread(target=work, args=(o,)) for o in blocks]
        t0 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        secs = time.perf_counter() - t0
        assert not refused, refused[0]
        return copies * cells * steps / secs / 1e9, secs

    sample(1)  # warm-up
    runs = [sample(sample_steps) for _ in range(args.steps)]
    value = statistics.median(r[0] for r in runs)
    line = {
        "metric": HEAT_METRIC.replace("64^3", f"{n}^3"), "value": round(value, 6), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (300 K block, 50 K Gaussian hot spot, sigma 8 cells, seed-jittered centre)",
        "impl": "reference",
        "config": {"workload": f"heat_block {n}^3 cells, Dirichlet 300 K faces, dt 0.9 x the limit, audited "
                               "Simulation::advance steps", "cells": cells, "copies": copies},
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": copies, "kind": "port",
                         "sample": f"{copies} independent copies of the {n}^3 block, one per thread, "
                                   f"{sample_steps} audited steps each per bench step (median of {args.steps}, "
                                   f"{runs[0][1]:.2f} s for the first); the Rust reference cannot be built here "
                                   "(no cargo), so this is the oracle's C++ restatement of its loops"},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_ensemble(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    from pantometry_b200 import workloads as W

    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    cfg = W.heat_ensemble(count=args.grids, steps=args.timesteps)
    grids = W.ensemble_grids(cfg)
    samples = [cpu_baseline_ensemble(cfg, grids, sample_steps=args.cpu_sample_steps, threads=ncpu,
                                     sample_grids=max(16, 2 * ncpu)) for _ in range(args.steps)]
    value = statistics.median(s["value"] for s in samples)
    line = {
        "metric": ENS_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded Rng::for_index sizes, diffusivities and hot spots)",
        "impl": "reference",
        "config": {"workload": f"heat ensemble: {len(grids)} grids, audited Simulation::advance steps per grid"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncpu, "kind": "port",
                         "sample": samples[0]["sample"] + "; the Rust reference cannot be built here (no cargo), "
                                   "so this is the oracle's C++ restatement of its loops"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hall", choices=["hall", "ensemble", "cavity", "mix", "heat"],
                    help="hall: the acoustic hall 256^3 (the headline); ensemble: 512 uneven heat grids; "
                         "cavity: the Yee cavity 384^3; mix: the 1024^3 heterogeneous hall and 64 Yee 128^3 "
                         "dielectric cavities; heat: the 64^3 heat block, plain f64 and FP32")
    ap.add_argument("--cavity-n", type=int, default=128, help="mix: cells per axis of each cavity")
    ap.add_argument("--n", type=int, default=None, help="grid size: hall 256 nodes, cavity 384, heat 64 cells per axis")
    ap.add_argument("--grids", type=int, default=None, help="ensemble: 512 heat grids; mix: 64 cavities")
    ap.add_argument("--timesteps", type=int, default=None, help="timesteps per bench step (hall 5000, ensemble 2000)")
    ap.add_argument("--cpu-sample-steps", type=int, default=None,
                    help="audited steps per CPU sample (hall 16, ensemble 8): about 10 s of one core")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-side-records", action="store_true",
                    help="hall: leave out the cavity, ensemble and heat-block objects of the default line")
    args = ap.parse_args()
    if args.n is None:
        args.n = {"cavity": 384, "mix": 1024, "heat": 64}.get(args.workload, 256)
    if args.grids is None:
        args.grids = 64 if args.workload == "mix" else 512
    if args.timesteps is None:
        args.timesteps = {"hall": 5000, "heat": 1000}.get(args.workload, 2000)
    if args.cpu_sample_steps is None:
        args.cpu_sample_steps = 16 if args.workload == "hall" else 8
    if args.workload == "mix":
        if args.impl == "reference":
            run_reference_mix(args)
        else:
            run_mix(args)
        return
    if args.workload == "heat":
        if args.impl == "reference":
            run_reference_heat(args)
        else:
            run_heat(args)
        return
    if args.workload == "cavity":
        if args.impl == "reference":
            run_reference_cavity(args)
        else:
            run_cavity(args)
        return
    if args.workload == "ensemble":
        if args.impl == "reference":
            run_reference_ensemble(args)
        else:
            run_ensemble(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
