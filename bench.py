#!/usr/bin/env python
"""Benchmark: world·cell-steps/s of the batched FP64 tissue step on B200 (one JSON line).

Workloads (``--workload``):
  grid    (default) the batched plain step: 4096 independent worlds per GPU, each a 16x16-grid
          pump-leak tissue (256 cells, 480 gap junctions, Na/K/Cl, GHK leaks, Na/K-ATPase, held
          bath), per-world parameters drawn from one seed; ARS(2,2,2) IMEX step in FP64 at
          dt = 1 ms (cells.solver.imex_ars222_face_electromigration@1);
  uneven  1024 worlds of 32-4096 cells (log-uniform), Delaunay contact graphs, NaV1.2 (m^3 h)
          and Hodgkin-Huxley K (n^4) populations on every cell, FP64, through the packed
          persistent kernel.
A bench step is one time step of every world.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed.run, one rank per GPU, each with its own 4096 worlds (weak
scaling; worlds never interact, so no collective is in the data path: NCCL carries only the
timing barrier and the max over ranks). ``--impl reference`` times the reference's CPU step (the
oracle, which reproduces it bit for bit) on the host cores instead, rank 0 only.
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

METRIC = "world·cell-steps/s"
UNIT = "world·cell-steps/s"
METHOD = "cells.solver.imex_ars222_face_electromigration@1"
METHOD_MIXED = "cells_b200.solver.imex_ars222_mixed_fp32@1"


def bytes_per_cell_step(batch):
    """Algorithmic bytes per world·cell·step: the state read and written once and the parameters
    read once per step. Per cell 2*8*(2S+4) state + 8*(4+S) parameters; per channel population
    2*8*4 state (two gate rows, transferred, dissipated) + 2*8 parameters; per junction
    2*8*(S+2) state + 8 + 8*(1+S) parameters; S = 3. The 16x16 grid (1.875 junctions per cell)
    gives 441 B."""
    s = 3
    per_cell = 2 * 8 * (2 * s + 4) + 8 * (4 + s) + batch.channel_slots * (2 * 8 * 4 + 2 * 8)
    per_edge = 2 * 8 * (s + 2) + 8 + 8 * (1 + s)
    return per_cell + per_edge * batch.edges / batch.cells


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=("grid", "uneven"), default="grid")
    ap.add_argument("--worlds", type=int, default=None,
                    help="worlds per GPU (default 4096 for grid, 1024 for uneven)")
    ap.add_argument("--side", type=int, default=16)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--fuse", type=int, default=100,
                    help="time steps per kernel launch (the largest divisor of --steps up to it)")
    ap.add_argument("--e2e-calls", type=int, default=3)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64",
                    help="mixed: the ARS(2,2,2) step with FP32 rates and FP64 accumulation")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the bind's launch configuration instead of the autotuner's")
    ap.add_argument("--no-graph", action="store_true",
                    help="issue the timed launches directly instead of replaying a CUDA graph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_cell_launch():
    """DRAM bytes per cell per launch of the step kernel (ncu, committed summary): a launch reads
    and writes its worlds' state once, whatever its step count."""
    path = os.path.join(ROOT, "profiles", "ars222_traffic.json")
    try:
        with open(path) as f:
            return float(json.load(f)["dram_bytes_per_cell_per_launch"])
    except (OSError, KeyError, ValueError):
        return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for name, flag in zip(names, r[5:9], strict=False):
                if flag.strip().lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def build_batch(args, rank):
    from cells_b200 import worlds

    if args.workload == "uneven":  # each rank its own seed
        return worlds.pack(worlds.delaunay_tissues(args.worlds, seed=2 + rank,
                                                   channels=worlds.UNEVEN_CHANNELS))
    # Each rank its own worlds: world ids rank*n .. rank*n + n - 1 of seed 1.
    ws = [worlds.grid_world(args.side, args.side, worlds.world_rng(1, rank * args.worlds + w))
          for w in range(args.worlds)]
    return worlds.pack(ws)


def sample_tasks(args, n, steps):
    """A strided sample of n of the workload's worlds, as CPU-baseline tasks."""
    from cells_b200 import worlds

    stride = max(1, args.worlds // n)
    if args.workload == "uneven":
        sizes = np.sort(worlds.uneven_sizes(args.worlds, seed=2))[::-1]
        return [("uneven", w * stride, 2, int(sizes[w * stride]), steps, args.dt)
                for w in range(n)], stride
    return [("grid", w * stride, 1, args.side, steps, args.dt) for w in range(n)], stride


def workload_name(args):
    if args.workload == "uneven":
        return (f"uneven batch: {args.worlds} worlds per GPU of 32-4096 cells (log-uniform), "
                "Delaunay contacts, NaV1.2 m^3 h + HH K n^4 populations, FP64, "
                f"dt {args.dt:g} s")
    return (f"batched plain step: {args.worlds} worlds per GPU x {args.side}x{args.side} grid "
            f"tissues, FP64, dt {args.dt:g} s")


def cpu_baseline(args, samples_per_core=2, steps=100):
    """The oracle (the reference's step restated, bit-identical) over all host cores: a strided
    sample of the workload's worlds, about 10 s of CPU work."""
    from oracle import cpu_baseline as cb

    cores = os.cpu_count() or 1
    n = cores * samples_per_core
    if args.workload == "uneven":
        steps = max(2, steps // 10)
    tasks, stride = sample_tasks(args, n, steps)
    cell_steps, wall, procs = cb.measure(tasks, cores)
    return {
        "value": cell_steps / wall,
        "unit": UNIT,
        "cores": procs,
        "kind": "port",
        "sample": (f"{n} of the {args.worlds} worlds (every {stride}th), {steps} ARS(2,2,2) "
                   f"steps each, one world per process, 1 BLAS thread, {wall:.1f} s wall"),
    }


def run_reference(args, rank):
    """The reference's CPU step (its oracle restatement) on the host cores: each bench step
    advances a strided sample of the workload's worlds (two per core) by ten time steps."""
    if rank != 0:
        return 0
    from oracle import cpu_baseline as cb

    cores = os.cpu_count() or 1
    n = cores * 2
    per_task = 10 if args.workload == "grid" else 1
    tasks, stride = sample_tasks(args, n, per_task)
    with cb.pool(cores) as pool:
        pool.map(cb.prepare, tasks, chunksize=1)
        for _ in range(max(args.warmup, 0)):
            pool.map(cb.run_world, tasks, chunksize=1)
        t0 = time.perf_counter()
        done = 0
        for _ in range(args.steps):
            res = pool.map(cb.run_world, tasks, chunksize=1)
            done += sum(r[0] for r in res)
        wall = time.perf_counter() - t0
    value = done / wall
    sample = (f"{n} of the {args.worlds} worlds (every {stride}th) advanced {per_task} "
              "ARS(2,2,2) steps per bench step, one world per process, 1 BLAS thread")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded pump-leak tissues)", "impl": "reference",
        "config": {"workload": workload_name(args) + " (sampled)", "method": METHOD,
                   "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.worlds is None:
        args.worlds = 1024 if args.workload == "uneven" else 4096
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    # The CPU baseline pool is spawned before any CUDA call.
    base = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(args)

    import torch

    from cells_b200.tissue import Tissue

    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)

    from cells_b200 import _lib as _lib_methods

    method = (_lib_methods.METHOD_ARS222_MIXED if args.precision == "mixed"
              else _lib_methods.METHOD_ARS222)
    batch = build_batch(args, rank)
    tissue = Tissue(batch, device=local_rank)
    cells = batch.cells
    fuse = max(d for d in range(1, max(1, min(args.fuse, args.steps)) + 1) if args.steps % d == 0)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    status = torch.zeros(batch.worlds, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    handle = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    tuned = None
    if not args.no_autotune:
        from cells_b200 import autotune

        best, timings = autotune.tune(tissue, state, control, args.dt,
                                      steps=min(20, fuse), repeats=2, method=method)
        tuned = {"selected": list(best),
                 "ms_per_step": {f"{k[0]}/{k[1]}/{k[2]}": round(v, 5) for k, v in timings.items()}}
    left = max(args.warmup, 1)
    while left > 0:  # warm-up steps, in launches of at most `fuse` steps
        tissue.step(state, state, control, args.dt, min(fuse, left), status, stream=handle,
                    method=method)
        left -= fuse
    torch.cuda.synchronize(dev)
    launches = args.steps // fuse
    graph = None
    if not args.no_graph:  # the timed launches as one CUDA graph
        graph = tissue.capture(state, state, control, args.dt, fuse, status, launches=launches,
                               method=method)
        stream = torch.cuda.current_stream(dev)
        handle = stream.cuda_stream
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    clocks = Clocks(local_rank)
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    if graph is not None:
        graph.replay()
    else:
        for _ in range(launches):
            tissue.step(state, state, control, args.dt, fuse, status, stream=handle,
                        method=method)
    stop.record(stream)
    torch.cuda.synchronize(dev)
    clock = clocks.stop()
    ms = start.elapsed_time(stop)
    refused = int((status != 0).sum().item())
    barrier()
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        r = torch.tensor([refused], dtype=torch.int64, device=dev)
        dist.all_reduce(r)
        refused = int(r.item())
    total_cell_steps = cells * args.steps * world_size
    value = total_cell_steps / (ms_max * 1e-3)

    # End to end through the public host entry point (cb_step_host): each call copies the packed
    # state and controls host->device from pinned memory, takes `fuse` steps, and copies the state
    # and status back.
    host_state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).pin_memory()
    host_ctl = torch.from_numpy(tissue.pack_control()).pin_memory()
    host_out = torch.empty_like(host_state).pin_memory()
    status_h = torch.zeros(batch.worlds, dtype=torch.int32).pin_memory()
    taken_h = torch.zeros(batch.worlds, dtype=torch.int32).pin_memory()
    import ctypes

    from cells_b200 import _lib

    def host_call():
        _lib.check(tissue.lib.cb_step_host(
            tissue.handle, method, ctypes.c_void_p(host_state.data_ptr()),
            ctypes.c_void_p(host_out.data_ptr()), float(args.dt),
            ctypes.c_void_p(host_ctl.data_ptr()), fuse, ctypes.c_void_p(status_h.data_ptr()),
            ctypes.c_void_p(taken_h.data_ptr())))

    e2e_value = None
    if args.e2e_calls > 0:
        host_call()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_calls):
            host_call()
        e2e_s = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_value = cells * fuse * args.e2e_calls * world_size / e2e_s
    h2d = (tissue.state_size + tissue.control_size) * 8 / fuse
    d2h = (tissue.state_size * 8 + 2 * 4 * batch.worlds) / fuse

    if rank == 0:
        peak, peak_kind = peaks()
        per_launch_s = ms * 1e-3 / launches
        algorithmic = bytes_per_cell_step(batch) * cells * fuse
        achieved = algorithmic / per_launch_s / 1e9
        traffic = traffic_per_cell_launch() if args.workload == "grid" else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 rates / f64 accumulation",
            "data": "synthetic (seeded pump-leak tissues)",
            "config": {
                "workload": workload_name(args),
                "method": METHOD if args.precision == "fp64" else METHOD_MIXED, "worlds_per_gpu": args.worlds, "steps_per_launch": fuse,
                "launch": dict(zip(("kernel", "block", "occupancy"), tissue.get_launch())),
                "autotune": tuned, "cuda_graph": graph is not None,
                "cells_per_gpu": cells, "junctions_per_gpu": batch.edges,
                "bytes_per_cell_step": bytes_per_cell_step(batch),
                "parallelism": f"independent worlds x{world_size} (no collective)",
                "l2": (f"inputs larger than L2: state {tissue.state_size * 8 / 1e6:.0f} MB + "
                       "parameters per GPU"),
            },
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": None if traffic is None else traffic * cells,
                "algorithmic_bytes_per_launch": algorithmic, "launch_ms": per_launch_s * 1e3,
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps_per_call": fuse,
                    "calls": args.e2e_calls},
            "gpu_launches": launches,
            "refused_worlds": refused,
            "clocks": clock,
        }
        if base is not None:
            line["cpu_baseline"] = base
        print(json.dumps(line), flush=True)
    del graph
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    tissue.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
