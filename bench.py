#!/usr/bin/env python
"""Benchmark: world·cell-steps/s of the batched FP64 tissue step on B200 (one JSON line).

Workloads (``--workload``):
  grid    (default) the batched plain step: 4096 independent worlds per GPU, each a 16x16-grid
          pump-leak tissue (256 cells, 480 gap junctions, Na/K/Cl, GHK leaks, Na/K-ATPase, held
          bath), per-world parameters drawn from one seed; ARS(2,2,2) IMEX step in FP64 at
          dt = 1 ms (cells.solver.imex_ars222_face_electromigration@1);
  uneven  1024 worlds of 32-4096 cells (log-uniform), Delaunay contact graphs, NaV1.2 (m^3 h)
          and Hodgkin-Huxley K (n^4) populations on every cell, FP64, through the packed
          persistent kernel;
  adjoint 512 worlds of 1024-cell Delaunay tissues with the uneven batch's laws: the gradient of
          each world's voltage-pattern loss (squared error of the final membrane voltages against
          -50 mV plus three 20 mV Gaussian bumps) after 2000 FP64 steps at dt = 1 ms (the
          ARS(2,2,2) step, or the ROS2 Rosenbrock step with --method ros2) with respect to every
          cell's P_Na, P_K, P_Cl, every junction's permeabilities and every channel population's
          permeability, checkpoints every 100 steps with recomputation.
  field   256 worlds of 1024 cells in a 128x128 extracellular grid (10 um spacing, the boundary
          ring held at the bath), 4-neighbour faces with log-normal conductivity (sigma 0.5),
          ARS(2,2,2) with implicit face electromigration at dt = 0.5 ms, the start field by the
          Newton on the floating offsets, the stage fields by sparse Cholesky, FP64.
A bench step is one time step of every world (grid, uneven, field) or one gradient of every
world's loss (adjoint: metric world-gradients/s).

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
ADJOINT_METRIC = "adjoint world-gradients/s"
ADJOINT_UNIT = "world-gradients/s"
METHOD = "cells.solver.imex_ars222_face_electromigration@1"
METHOD_MIXED = "cells_b200.solver.imex_ars222_mixed_fp32@1"
METHOD_N2 = "cells.solver.imex_ars222_implicit_conductances@1"
METHOD_N2_MIXED = "cells_b200.solver.imex_ars222_implicit_conductances_mixed@1"
METHOD_ROS2 = "cells_b200.solver.ros2_verwer@1"
METHOD_ROS2_MIXED = "cells_b200.solver.ros2_verwer_fp32_factor@1"


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
    ap.add_argument("--steps", type=int, default=None,
                    help="timed bench steps (default 1000; adjoint: 3 gradients)")
    ap.add_argument("--warmup", type=int, default=None,
                    help="untimed bench steps first (default 100; adjoint: 3 gradients)")
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=("grid", "uneven", "adjoint", "field"), default="field")
    ap.add_argument("--worlds", type=int, default=None,
                    help="worlds per GPU (default 4096 grid, 1024 uneven, 512 adjoint)")
    ap.add_argument("--cells", type=int, default=1024, help="adjoint: cells per world")
    ap.add_argument("--trajectory", type=int, default=2000, help="adjoint: steps per gradient")
    ap.add_argument("--every", type=int, default=100, help="adjoint: checkpoint interval")
    ap.add_argument("--side", type=int, default=None,
                    help="grid tissues' side (16), or the field grid's (128)")
    ap.add_argument("--field-cells", type=int, default=32, help="field: tissue side (cells)")
    ap.add_argument("--dt", type=float, default=None, help="1 ms (0.5 ms for field)")
    ap.add_argument("--fuse", type=int, default=100,
                    help="time steps per kernel launch (the largest divisor of --steps up to it)")
    ap.add_argument("--e2e-calls", type=int, default=None,
                    help="end-to-end host calls timed (default 3; adjoint: 1 gradient)")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64",
                    help="mixed: FP32 fluxes (ars222), an FP32 factor with FP64 refinement (n2), "
                         "an FP32 factor and substitutions without refinement (ros2)")
    ap.add_argument("--method", choices=("ars222", "n2", "ros2"), default="ars222",
                    help="n2: slope conductances implicit, a sparse Cholesky per world per step; "
                         "ros2: the two-stage Rosenbrock method on the same operator")
    ap.add_argument("--precision-steps", type=int, default=500,
                    help="field: steps after which the precision sub-record compares each mixed "
                         "form's state with its FP64 step's")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the bind's launch configuration instead of the autotuner's")
    ap.add_argument("--no-graph", action="store_true",
                    help="issue the timed launches directly instead of replaying a CUDA graph")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sub", action="store_true",
                    help="field: skip the grid and adjoint sub-records")
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
    """SM clocks, power and throttle reasons sampled DURING the timed region: NVML every 10 ms
    on a host thread (the device found by its UUID, so CUDA_VISIBLE_DEVICES maps right), else
    nvidia-smi every 100 ms."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.thread = None
        self.proc = None
        self.file = None
        self.halt = None
        self.nvml = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.device).uuid)
        name = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        return pynvml, pynvml.nvmlDeviceGetHandleByUUID(name)

    def start(self):
        import threading

        try:
            nvml, handle = self._nvml_handle()
            self.nvml = (nvml, handle)
            self.smax = nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM)
        except Exception:  # noqa: BLE001 - no NVML: the nvidia-smi sampler below
            self.nvml = None
        if self.nvml is not None:
            self.halt = threading.Event()

            def loop():
                nvml, handle = self.nvml
                while not self.halt.is_set():
                    try:
                        sm = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                        mask = nvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                        power = nvml.nvmlDeviceGetPowerUsage(handle) / 1e3
                        self.samples.append((sm, mask, power))
                    except Exception:  # noqa: BLE001
                        pass
                    self.halt.wait(0.01)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.halt.set()
            self.thread.join(timeout=5)
            sm = [x[0] for x in self.samples]
            reasons = set()
            for _, mask, _ in self.samples:
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        reasons.add(name)
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": self.smax, "reasons": sorted(reasons), "samples": len(sm),
                    "power_w_max": max((x[2] for x in self.samples), default=None),
                    "sampler": "nvml 10 ms"}
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
            "sampler": "nvidia-smi 100 ms",
        }


def build_batch(args, rank):
    from cells_b200 import worlds

    if args.workload == "adjoint":  # each rank its own world ids, seed 4
        return worlds.pack([worlds.uneven_world(rank * args.worlds + w, args.cells, 4,
                                                worlds.UNEVEN_CHANNELS)
                            for w in range(args.worlds)])
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
    if args.workload == "adjoint":
        kind = "adjoint_ros2" if args.method == "ros2" else "adjoint"
        return [(kind, w * stride, 4, args.cells, steps, args.dt) for w in range(n)], stride
    if args.workload == "uneven":
        sizes = np.sort(worlds.uneven_sizes(args.worlds, seed=2))[::-1]
        return [("uneven", w * stride, 2, int(sizes[w * stride]), steps, args.dt)
                for w in range(n)], stride
    return [("grid", w * stride, 1, args.side, steps, args.dt) for w in range(n)], stride


def workload_name(args):
    if args.workload == "field":
        return (f"spatial extracellular field: {args.worlds} worlds per GPU x "
                f"{args.field_cells ** 2} cells in a {args.side}x{args.side} extracellular grid "
                "(10 um, held ring), log-normal face conductivity (sigma 0.5), ARS(2,2,2) with "
                f"implicit face electromigration, FP64, dt {args.dt:g} s")
    if args.workload == "adjoint":
        return (f"adjoint sensitivities: {args.worlds} worlds per GPU x {args.cells}-cell "
                "Delaunay tissues, NaV1.2 m^3 h + HH K n^4 populations, gradient of each world's "
                "voltage-pattern loss after "
                f"{args.trajectory} FP64 {'ROS2' if args.method == 'ros2' else 'ARS(2,2,2)'} "
                f"steps (dt {args.dt:g} s) w.r.t. all membrane, junction "
                f"and channel permeabilities, checkpoints every {args.every} steps")
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
    if args.workload == "adjoint":
        tasks, stride = sample_tasks(args, n, 20)
        cell_steps, wall, procs = cb.measure(tasks, cores, fn=cb.run_adjoint_world)
        rate = cell_steps / wall
        return {
            "value": rate / (args.cells * args.trajectory), "unit": ADJOINT_UNIT,
            "cores": procs, "kind": "port",
            "adjoint_cell_steps_per_s": rate,
            "sample": (f"{n} of the {args.worlds} worlds (every {stride}th): 20 "
                       f"{'ROS2' if args.method == 'ros2' else 'ARS(2,2,2)'} steps forward "
                       "then the oracle adjoint back over them, one world per process, 1 BLAS "
                       f"thread, {wall:.1f} s wall; world-gradients/s = that rate of world-"
                       f"cell-steps / ({args.cells} cells x {args.trajectory} steps)"),
        }
    if args.workload == "field":
        tasks, stride = field_tasks(args, n, 10)
        cell_steps, wall, procs = cb.measure(tasks, cores, fn=cb.run_field_world)
        return {"value": cell_steps / wall, "unit": UNIT, "cores": procs, "kind": "port",
                "sample": field_sample(args, n, stride, 10, wall)}
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


def field_tasks(args, n, steps):
    """A strided sample of n of the field workload's own worlds (same seed, ids and shape) as
    CPU tasks."""
    stride = max(1, args.worlds // n)
    shape = (args.side, args.field_cells, 3)
    return [("field", w * stride, 7, shape, steps, args.dt) for w in range(n)], stride


def field_sample(args, n, stride, steps, wall=None):
    text = (f"{n} of the {args.worlds} field worlds (every {stride}th; {args.side}x{args.side} "
            f"grid, {args.field_cells ** 2} cells), {steps} ARS(2,2,2) steps each, one world per "
            "process, 1 BLAS thread: the field oracle's restatement of the reference's step in "
            "sparse containers (the reference's own dense offset solve would be a 15876 x 15876 "
            "LU per Newton iteration at this grid; its sparse field bind refuses the grid)")
    return text + (f", {wall:.1f} s wall" if wall is not None else "")


def run_reference(args, rank):
    """The reference's CPU step (its oracle restatement) on the host cores: each bench step
    advances a strided sample of the workload's worlds (two per core) by ten time steps."""
    if rank != 0:
        return 0
    from oracle import cpu_baseline as cb

    cores = os.cpu_count() or 1
    n = cores * 2
    adjoint = args.workload == "adjoint"
    field = args.workload == "field"
    per_task = 10 if args.workload == "grid" else 3 if adjoint else 1
    fn = cb.run_adjoint_world if adjoint else cb.run_field_world if field else cb.run_world
    if field:
        per_task = 1
        tasks, stride = field_tasks(args, n, per_task)
    else:
        tasks, stride = sample_tasks(args, n, per_task)
    with cb.pool(cores) as pool:
        pool.map(cb.prepare, tasks, chunksize=1)
        for _ in range(max(args.warmup, 0)):
            pool.map(fn, tasks, chunksize=1)
        t0 = time.perf_counter()
        done = 0
        for _ in range(args.steps):
            res = pool.map(fn, tasks, chunksize=1)
            done += sum(r[0] for r in res)
        wall = time.perf_counter() - t0
    value = done / wall
    metric, unit = METRIC, UNIT
    if adjoint:  # world-cell-steps of forward + adjoint per second -> world-gradients/s
        value = value / (args.cells * args.trajectory)
        metric, unit = ADJOINT_METRIC, ADJOINT_UNIT
        sample = (f"{n} of the {args.worlds} worlds (every {stride}th), {per_task} steps "
                  "forward then the oracle adjoint back over them per bench step, one world per "
                  "process, 1 BLAS thread (the reference has no adjoint; its gradients would "
                  "come from jax.grad, and jax is not installed)")
    elif field:
        sample = field_sample(args, n, stride, per_task) + " (per bench step)"
    else:
        sample = (f"{n} of the {args.worlds} worlds (every {stride}th) advanced {per_task} "
                  "ARS(2,2,2) steps per bench step, one world per process, 1 BLAS thread")
    line = {
        "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded pump-leak tissues)", "impl": "reference",
        "config": {"workload": workload_name(args) + " (sampled)", "method": METHOD,
                   "sample": sample},
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def vjp_bytes_per_cell_step(batch):
    """Algorithmic bytes per world-cell-step of the reverse (cb_step_vjp's reverse kernel): per
    cell the step-start dynamic state (3 amounts, 2 NCH gates) and the end amounts read, the
    parameters read (1/V, 1/C, Q0, 3 references, 3 prefactors, pump capacity and its log, area:
    12 doubles; per channel population its prefactor, abundance, law and species: 24 B), the
    controls read (2 + NCH), the dynamic cotangent read and written, the permeability gradients
    read and written (3 + NCH), and its adjacency offset; per junction its gate, 3 prefactors,
    area, threshold, minimum and control read, its endpoints and two adjacency entries, its gate
    cotangent read and written and 3 gradients read and written."""
    n = batch.channel_slots
    per_cell = 8 * ((6 + 2 * n) + 12 + (2 + n) + 2 * (3 + 2 * n) + 2 * (3 + n)) + 8 * n + 4
    per_edge = 8 * 8 + 8 + 8 + 8 * 2 + 8 * 6
    return per_cell + per_edge * batch.edges / batch.cells


def run_adjoint(args, rank, world_size, local_rank, dist, base):
    """The adjoint workload: each bench step is the gradient of every world's voltage-pattern
    loss through cells_b200.adjoint (forward in checkpointed segments, cb_step_vjp_method back),
    of the ARS(2,2,2) step or, with --method ros2, of the ROS2 step."""
    import torch

    from cells_b200 import _lib as _lib_methods
    from cells_b200 import adjoint, worlds
    from cells_b200.tissue import Tissue

    ros2 = args.method == "ros2"
    method = _lib_methods.METHOD_ROS2 if ros2 else _lib_methods.METHOD_ARS222
    fwd_name = "ros2_kernel" if ros2 else "packed_kernel"
    rev_name = "ros2_vjp_kernel" if ros2 else "vjp_kernel"

    dev = torch.device("cuda", local_rank)
    batch = build_batch(args, rank)
    tissue = Tissue(batch, device=local_rank)
    cells, w_count = batch.cells, batch.worlds
    state0 = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    target = torch.tensor(worlds.voltage_target(batch), device=dev)
    params = [t.requires_grad_() for t in adjoint.permeabilities(tissue)]
    refused = torch.zeros(w_count, dtype=torch.int32, device=dev)

    def gradient(state, perms):
        final, bits = adjoint.trajectory(tissue, state, control, args.dt, args.trajectory, *perms,
                                         every=args.every, method=method)
        loss = adjoint.voltage_loss(tissue, final, target)
        loss.sum().backward()
        return loss, bits

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        gradient(state0, params)
        for p in params:
            p.grad = None
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    clocks = Clocks(local_rank)
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        loss, bits = gradient(state0, params)
        refused |= bits
        for p in params:
            p.grad = None
    stop.record(stream)
    torch.cuda.synchronize(dev)
    clock = clocks.stop()
    ms = start.elapsed_time(stop)
    n_refused = int((refused != 0).sum().item())
    barrier()
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = w_count * world_size * args.steps / (ms_max * 1e-3)

    # Kernel durations on the same inputs (CUDA events, this stream): a fused forward segment,
    # a segment of one-step launches (the recompute), and cb_step_vjp over a segment; the
    # reverse kernel's time is the last less the recompute.
    k = min(args.every, args.trajectory)
    status = torch.zeros(w_count, dtype=torch.int32, device=dev)
    out = torch.empty_like(state0)
    ws = torch.empty(tissue.vjp_workspace_bytes(k, method), dtype=torch.uint8, device=dev)
    cot = torch.zeros_like(state0)
    o = tissue.state_offsets["amount_increment"]
    cot[o:o + 3 * cells] = 1e-3
    gm = torch.zeros(3 * cells, dtype=torch.float64, device=dev)
    gj = torch.zeros(max(3 * batch.edges, 1), dtype=torch.float64, device=dev)
    gch = torch.zeros(max(batch.channel_slots * cells, 1), dtype=torch.float64, device=dev)
    nch = batch.channel_slots

    def timed(fn, reps=3):
        fn()
        times = []
        for _ in range(reps):
            a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b_.record(stream)
            torch.cuda.synchronize(dev)
            times.append(a.elapsed_time(b_))
        return statistics.median(times)

    def one_step_segment():
        src = state0
        for _ in range(k):
            tissue.step(src, out, control, args.dt, 1, status, method=method)
            src = out

    fused_ms = timed(lambda: tissue.step(state0, out, control, args.dt, k, status,
                                         method=method))
    onestep_ms = timed(one_step_segment)
    vjp_ms = timed(lambda: tissue.step_vjp(state0, control, args.dt, k, cot, out, gm, gj,
                                           gch if nch else None, ws, status, method=method))
    reverse_ms = max(vjp_ms - onestep_ms, 1e-6)
    segments = -(-args.trajectory // args.every)
    per_gradient = {f"{fwd_name} (forward, fused)": fused_ms * segments,
                    f"{fwd_name} (recompute, one step per launch)": onestep_ms * segments,
                    f"{rev_name} (reverse)": reverse_ms * segments}
    total = sum(per_gradient.values())
    fwd_bytes = bytes_per_cell_step(batch) * cells
    rev_bytes = vjp_bytes_per_cell_step(batch) * cells
    peak, peak_kind = peaks()
    kernels = {
        fwd_name: {"ms_per_gradient": (fused_ms + onestep_ms) * segments,
                          "share": (fused_ms + onestep_ms) * segments / total,
                          "achieved_gbs_fused": fwd_bytes * k / (fused_ms * 1e-3) / 1e9,
                          "achieved_gbs_one_step": fwd_bytes * k / (onestep_ms * 1e-3) / 1e9,
                          "bytes_per_cell_step": bytes_per_cell_step(batch)},
        rev_name: {"ms_per_gradient": reverse_ms * segments,
                       "share": reverse_ms * segments / total,
                       "achieved_gbs": rev_bytes * k / (reverse_ms * 1e-3) / 1e9,
                       "bytes_per_cell_step": vjp_bytes_per_cell_step(batch)},
    }
    dominant = max(kernels, key=lambda name: kernels[name]["share"])
    if dominant == rev_name:
        launch_ms, alg = reverse_ms, rev_bytes * k
    else:
        launch_ms, alg = fused_ms, fwd_bytes * k
    achieved = alg / (launch_ms * 1e-3) / 1e9

    # End to end through the public API with host buffers: each call copies the start state and
    # the permeabilities from pinned host memory, takes the gradient, and copies the gradients
    # and the losses back.
    host_state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).pin_memory()
    host_perm = [p.detach().cpu().pin_memory() for p in params]
    host_grad = [torch.empty_like(h).pin_memory() for h in host_perm]
    host_loss = torch.empty(w_count, dtype=torch.float64).pin_memory()

    def host_call():
        st = host_state.to(dev, non_blocking=True)
        perms = [h.to(dev, non_blocking=True).requires_grad_() for h in host_perm]
        loss, _ = gradient(st, perms)
        for h, p in zip(host_grad, perms, strict=True):
            h.copy_(p.grad, non_blocking=True)
        host_loss.copy_(loss.detach(), non_blocking=True)
        torch.cuda.synchronize(dev)

    e2e_value = None
    if args.e2e_calls > 0:
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_calls):
            host_call()
        e2e_s = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_value = w_count * world_size * args.e2e_calls / e2e_s
    perm_bytes = sum(h.numel() for h in host_perm) * 8
    launches_per_gradient = 2 + segments + segments * (k + 1)
    if rank == 0:
        line = {
            "metric": ADJOINT_METRIC, "value": value, "unit": ADJOINT_UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded pump-leak tissues)",
            "config": {
                "workload": workload_name(args), "method": METHOD_ROS2 if ros2 else METHOD,
                "worlds_per_gpu": args.worlds, "cells_per_world": args.cells,
                "cells_per_gpu": cells, "junctions_per_gpu": batch.edges,
                "trajectory_steps": args.trajectory, "checkpoint_every": args.every,
                "parameters_per_gpu": perm_bytes // 8,
                "launch": dict(zip(("kernel", "block", "occupancy"), tissue.get_launch())),
                "adjoint_world_cell_steps_per_s": value * cells / w_count * args.trajectory,
                "parallelism": f"independent worlds x{world_size} (no collective)",
                "l2": (f"inputs larger than L2: state {tissue.state_size * 8 / 1e6:.0f} MB per "
                       "GPU, checkpoints and the segment workspace several GB"),
            },
            "roofline": {
                "bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": None, "algorithmic_bytes_per_launch": alg, "launch_ms": launch_ms,
            },
            "kernels": kernels,
            "e2e": {"value": e2e_value, "unit": ADJOINT_UNIT,
                    "h2d_bytes_per_step": tissue.state_size * 8 + perm_bytes,
                    "d2h_bytes_per_step": perm_bytes + w_count * 8, "calls": args.e2e_calls},
            "gpu_launches": launches_per_gradient * args.steps,
            "refused_worlds": n_refused,
            "clocks": clock,
        }
        if base is not None:
            line["cpu_baseline"] = base
    tissue.close()
    return line if rank == 0 else None


def field_bytes_per_world_step(tissue, info, factorisations=2, solve_reads=0):
    """Algorithmic bytes per world per step of the field step, by the minimal-traffic count: the
    state read and written once, the parameters read once (per cell 11 doubles, per junction 5,
    per node 6, per face 3), and each factorisation's factor written once and read once
    (factor_doubles each way). solve_reads > 0 adds that many further reads of the factor (both
    sweeps of every solve re-read it: 2 x solves), the count that charges every pass."""
    state = tissue.state_total // tissue.W
    params = 11 * tissue.N + 5 * tissue.E + 6 * tissue.O + 3 * tissue.F
    factor = info["factor_doubles"] * (2 * factorisations + solve_reads)
    return 8 * (2 * state + params + factor)


_FP64_PEAK = {}


def fp64_peak(device):
    """The device's FP64 FMA rate (FLOP/s, cb_probe_fp64: independent FMA chains on every SM,
    CUDA events), measured once per process."""
    if device not in _FP64_PEAK:
        import ctypes

        from cells_b200 import _lib

        lib = _lib.load()
        rate, ms = ctypes.c_double(), ctypes.c_double()
        _lib.check(lib.cb_probe_fp64(device, 1 << 18, ctypes.byref(rate), ctypes.byref(ms)))
        _FP64_PEAK[device] = (rate.value, ms.value)
    return _FP64_PEAK[device]


def run_field(args, rank, world_size, local_rank, dist, base):
    """The spatial-field workload: each bench step is one ARS(2,2,2) step of every world."""
    import torch

    from cells_b200 import field_worlds, worlds
    from cells_b200.field import FieldTissue

    dev = torch.device("cuda", local_rank)
    ws = [field_worlds.field_world(args.side, args.field_cells, 3,
                                   worlds.world_rng(7, rank * args.worlds + w))
          for w in range(args.worlds)]
    tissue = FieldTissue(ws, device=local_rank)
    info = tissue.info()
    cells = tissue.N * tissue.W
    state0 = tissue.pack_state(tissue.initial_state())
    state = torch.from_numpy(state0).to(dev)
    control_np = tissue.pack_control()
    control = torch.from_numpy(control_np).to(dev)
    status = torch.zeros(tissue.W, dtype=torch.int32, device=dev)
    taken = torch.zeros(tissue.W, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        tissue.step(state, state, control, args.dt, 1, status, taken,
                    stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    barrier()
    torch.cuda.synchronize(dev)
    clocks = Clocks(local_rank)
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = factorisations = solves = 0
    start.record(stream)
    for _ in range(args.steps):
        tissue.step(state, state, control, args.dt, 1, status, taken,
                    stream=stream.cuda_stream)
        c = tissue.counts()
        launches += c["launches"]
        factorisations += c["factorisations"]
        solves += c["solves"]
    stop.record(stream)
    torch.cuda.synchronize(dev)
    clock = clocks.stop()
    ms = start.elapsed_time(stop)
    n_refused = int((status != 0).sum().item())
    barrier()
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = cells * world_size * args.steps / (ms_max * 1e-3)
    launch_ms = ms / args.steps
    fact_per_step, solves_per_step = factorisations / args.steps, solves / args.steps
    alg = field_bytes_per_world_step(tissue, info, fact_per_step) * tissue.W
    alg_all = field_bytes_per_world_step(tissue, info, fact_per_step,
                                         2 * solves_per_step) * tissue.W
    achieved = alg / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    fl = tissue.flops()
    step_flops = (fact_per_step * fl["factor"] + solves_per_step * fl["solve"]) * tissue.W
    fp64_rate, fp64_ms = fp64_peak(local_rank)
    # End to end through the C ABI with host buffers (cb_field_step_host on packed, pinned host
    # buffers: the state and control copied in, one step, the state and status copied out, every
    # call).
    pinned_in = torch.from_numpy(state0).pin_memory().numpy()
    pinned_out = torch.empty(state0.size, dtype=torch.float64).pin_memory().numpy()
    pinned_ctl = torch.from_numpy(control_np).pin_memory().numpy()
    host_status = np.zeros(tissue.W, dtype=np.uint32)
    host_taken = np.zeros(tissue.W, dtype=np.int32)
    e2e_value = None
    if args.e2e_calls > 0:
        tissue.step_host_packed(pinned_in, pinned_out, pinned_ctl, args.dt, 1, host_status,
                                host_taken)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_calls):
            tissue.step_host_packed(pinned_in, pinned_out, pinned_ctl, args.dt, 1, host_status,
                                    host_taken)
        e2e_s = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_value = cells * world_size * args.e2e_calls / e2e_s
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded field worlds)",
            "config": {
                "workload": workload_name(args), "method": METHOD,
                "field_solver": "capacitive reduction, Newton on the floating offsets (chord, "
                                "face Laplacian), nested-dissection multifrontal Cholesky",
                "worlds_per_gpu": args.worlds, "cells_per_world": tissue.N,
                "outside_nodes_per_world": tissue.O, "faces_per_world": tissue.F,
                "junctions_per_world": tissue.E, "solver": info,
                "parallelism": f"independent worlds x{world_size} (no collective)",
                "l2": (f"inputs larger than L2: state {tissue.state_total * 8 / 1e6:.0f} MB, "
                       f"scratch {info['scratch_bytes'] / 1e9:.1f} GB per GPU"),
            },
            "roofline": {
                "bound": "hbm",
                "kernel": "field step (field_phase, factor_*, forward_*, backward_* launches)",
                "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": None,
                "traffic_note": ("a step is ~700 launches of 13 kernels: no one-kernel capture "
                                 "gives its DRAM bytes; the per-kernel DRAM figures are in the "
                                 "committed ncu summaries (factor_group, field_phase)"),
                "algorithmic_bytes_per_launch": alg, "launch_ms": launch_ms,
                "bytes_per_world_step": alg / tissue.W,
                "count": ("minimal traffic: state read and written once, parameters read once, "
                          "each factorisation's factor written once and read once"),
                "achieved_every_pass": alg_all / (launch_ms * 1e-3) / 1e9,
                "frac_every_pass": alg_all / (launch_ms * 1e-3) / 1e9 / peak,
                "every_pass_note": ("the same with the factor re-read by both sweeps of each "
                                    f"solve ({solves_per_step:g} solves per step)"),
            },
            "fp64": {
                "peak_tflops": fp64_rate / 1e12, "peak_kind": "measured (cb_probe_fp64)",
                "probe_ms": fp64_ms,
                "achieved_tflops": step_flops / (launch_ms * 1e-3) / 1e12,
                "frac": step_flops / (launch_ms * 1e-3) / fp64_rate,
                "flops_per_world_step": step_flops / tissue.W,
                "note": ("factorisation and substitution arithmetic of the plan only (FMA = 2), "
                         f"{fact_per_step:g} factorisations and {solves_per_step:g} solves per "
                         "step; the per-world phases' arithmetic is not counted"),
            },
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": 8 * (tissue.state_total + tissue.control_total),
                    "d2h_bytes_per_step": 8 * tissue.state_total + 8 * tissue.W,
                    "calls": args.e2e_calls},
            "gpu_launches": launches,
            "refused_worlds": n_refused,
            "clocks": clock,
        }
        if base is not None:
            line["cpu_baseline"] = base
    return line if rank == 0 else None


def load_reference_pytrees(name):
    """The reference's own padded pytrees (layout, control, the first state) from a committed
    golden fixture, as NamedTuples with the reference's field names."""
    from collections import namedtuple

    z = np.load(os.path.join(ROOT, "tests", "golden", name))
    lf = [k[len("layout_"):] for k in z.files if k.startswith("layout_")]
    cf = [k[len("control_ref_"):] for k in z.files if k.startswith("control_ref_")]
    sf = [str(f) for f in z["state_fields"]]
    p = namedtuple("ReferenceLayout", lf)(*(z["layout_" + f] for f in lf))
    control = namedtuple("ReferenceControl", cf)(*(z["control_ref_" + f] for f in cf))
    state = namedtuple("ReferenceState", sf)(*(z["refstate_" + f][0] for f in sf))
    return z, p, control, state


def run_dropin(args, rank, world_size, local_rank, dist, base):
    """The drop-in boundary timed as a caller of the reference's model protocol uses it:
    cells_b200.model.DeviceStep(p)(state, dt, control, p, active) on the reference's own padded
    @3 pytrees (one world with channel populations, from a committed fixture), one step per call
    with host pytrees in and out; its CPU baseline the oracle's step of the same world (the
    reference's step restated), one host core."""
    del base, world_size, dist
    if rank != 0:
        return None
    from cells_b200 import model
    from oracle import tissue as T

    z, p, control, state = load_reference_pytrees("pytrees_v3_channels_padded.npz")
    dt = float(z["dt"])
    step = model.DeviceStep(p, device=local_rank)
    cells = int(step.batch.cells)
    st = state
    for _ in range(5):
        st, _ = step(st, dt, control, p, p.active)
    calls = args.steps
    t0 = time.perf_counter()
    st = state
    for _ in range(calls):
        st, valid = step(st, dt, control, p, p.active)
    wall = time.perf_counter() - t0
    b = step.batch
    topo = T.topology(b)
    ost = T.initial_state(b)
    octl = T.full_control(b)
    t1 = time.perf_counter()
    n_cpu = max(1, min(calls, 50))
    for _ in range(n_cpu):
        ost, _ = T.ars222_step(ost, dt, octl, b, topo)
    cpu = (time.perf_counter() - t1) / n_cpu
    step.close()
    per_call = wall / calls
    return {
        "metric": METRIC, "value": cells / per_call, "unit": UNIT,
        "ms_per_step": 1e3 * per_call, "dtype": "f64",
        "config": {"workload": "drop-in: model.DeviceStep on the reference's own padded @3 "
                               f"pytrees ({cells} active cells, NaV1.2 + Kv1.5 populations), one "
                               "step per call, host pytrees in and out",
                   "calls": calls, "valid": bool(valid)},
        "cpu_baseline": {"value": cells / cpu, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": f"the oracle's ARS(2,2,2) step of the same world, {n_cpu} "
                                   "steps on one host core"},
        "note": ("each call maps the padded pytrees to the packed layout, copies them to the "
                 "device, steps once and copies back: call latency, not throughput; batches of "
                 "worlds go through Tissue or vector_window"),
    }


def run_precision(args, rank, world_size, local_rank, dist, base):
    """The precision forms against their FP64 steps on the 4096-world 16x16 grid batch: per pair
    (ROS2 and its FP32-factor form; N2 and its FP32 factor with FP64 refinement; ARS(2,2,2) and
    its FP32-flux form), ms per step of each (CUDA events over fused launches after warm-up), the
    mixed/plain speed ratio, and each state field's scaled difference max |mixed - plain| /
    max |plain| after a run from the same start."""
    import torch

    from cells_b200 import _lib as L
    from cells_b200.tissue import Tissue

    del base
    dev = torch.device("cuda", local_rank)
    batch = build_batch(args, rank)
    tissue = Tissue(batch, device=local_rank)
    state0 = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    status = torch.zeros(batch.worlds, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(method, steps):
        out = torch.empty_like(state0)
        tissue.step(state0, out, control, args.dt, 5, status, method=method)  # warm-up
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        tissue.step(state0, out, control, args.dt, steps, status, method=method)
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / steps

    def final(method, steps):
        out = torch.zeros_like(state0)
        tissue.step(state0, out, control, args.dt, steps, status, method=method)
        torch.cuda.synchronize(dev)
        refused = int((status != 0).sum().item())
        return tissue.unpack_state(out.cpu().numpy()), refused

    pairs = {"ros2": (L.METHOD_ROS2, L.METHOD_ROS2_MIXED, METHOD_ROS2, METHOD_ROS2_MIXED, 20),
             "n2": (L.METHOD_N2, L.METHOD_N2_MIXED, METHOD_N2, METHOD_N2_MIXED, 20),
             "ars222": (L.METHOD_ARS222, L.METHOD_ARS222_MIXED, METHOD, METHOD_MIXED, 100)}
    out = {}
    for name, (plain, mixed, plain_id, mixed_id, steps) in pairs.items():
        ms_p, ms_m = timed(plain, steps), timed(mixed, steps)
        run = args.precision_steps
        ref, refused_p = final(plain, run)
        got, refused_m = final(mixed, run)
        errors = {}
        for f, r in ref.items():
            r, g = np.asarray(r), np.asarray(got[f])
            scale = float(np.max(np.abs(r), initial=0.0))
            if scale > 0.0:
                errors[f] = float(np.max(np.abs(g - r)) / scale)
        out[name] = {
            "plain": {"method": plain_id, "ms_per_step": ms_p,
                      "value": batch.cells * world_size / (ms_p * 1e-3)},
            "mixed": {"method": mixed_id, "ms_per_step": ms_m,
                      "value": batch.cells * world_size / (ms_m * 1e-3)},
            "mixed_over_plain": ms_p / ms_m,
            "max_scaled_error": max(errors.values()),
            "scaled_error_per_field": errors,
            "error_after_steps": run,
            "refused_worlds": {"plain": refused_p, "mixed": refused_m},
        }
    tissue.close()
    if rank != 0:
        return None
    return {"metric": METRIC, "unit": UNIT, "dtype": "f64 vs mixed",
            "config": {"workload": workload_name(args), "worlds_per_gpu": args.worlds,
                       "cells_per_gpu": batch.cells},
            "pairs": out}


def run_grid(args, rank, world_size, local_rank, dist, base):
    """The held-bath workloads (grid, uneven): each bench step is one time step of every world,
    the timed launches replayed from one CUDA graph."""
    import torch

    from cells_b200.tissue import Tissue

    dev = torch.device("cuda", local_rank)
    from cells_b200 import _lib as _lib_methods

    if args.method == "ros2":
        method = (_lib_methods.METHOD_ROS2_MIXED if args.precision == "mixed"
                  else _lib_methods.METHOD_ROS2)
    elif args.method == "n2":
        method = (_lib_methods.METHOD_N2_MIXED if args.precision == "mixed"
                  else _lib_methods.METHOD_N2)
    else:
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
    if not args.no_autotune and args.method == "ars222":
        from cells_b200 import autotune

        best, timings = autotune.tune(tissue, state, control, args.dt,
                                      steps=min(20, fuse), repeats=2, method=method)
        tuned = {"selected": list(best),
                 "ms_per_step": {f"{k[0]}/{k[1]}/{k[2]}": round(v, 5) for k, v in timings.items()}}
    elif not args.no_autotune and args.method == "ros2":
        from cells_b200 import autotune

        best, timings = autotune.tune_sparse(tissue, state, control, args.dt, steps=3, repeats=2,
                                             method=method)
        tuned = {"selected": {"block": best},
                 "ms_per_step": {str(k): round(v, 5) for k, v in timings.items()}}
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
            "dtype": ("f64" if args.precision == "fp64" else
                      "f32 factor / f64 refinement" if args.method == "n2" else
                      "f32 factor and substitutions / f64 rest" if args.method == "ros2" else
                      "f32 fluxes / f64 rest"),
            "data": "synthetic (seeded pump-leak tissues)",
            "config": {
                "workload": workload_name(args),
                "method": ((METHOD_ROS2 if args.precision == "fp64" else METHOD_ROS2_MIXED)
                           if args.method == "ros2" else
                           (METHOD_N2 if args.precision == "fp64" else METHOD_N2_MIXED)
                           if args.method == "n2" else
                           METHOD if args.precision == "fp64" else METHOD_MIXED),
                "worlds_per_gpu": args.worlds, "steps_per_launch": fuse,
                "launch": ({"kernel": f"{args.method} (one world per CTA)",
                            "block": tissue.get_sparse_launch() if args.method == "ros2" else 256}
                           if args.method in ("n2", "ros2") else
                           dict(zip(("kernel", "block", "occupancy"), tissue.get_launch()))),
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
    del graph
    tissue.close()
    return line if rank == 0 else None




def main():
    args = parse()
    adjoint = args.workload == "adjoint"
    field = args.workload == "field"
    if args.worlds is None:
        args.worlds = {"uneven": 1024, "adjoint": 512, "field": 256}.get(args.workload, 4096)
    if args.side is None:
        args.side = 128 if field else 16
    if args.dt is None:
        args.dt = 5e-4 if field else 1e-3
    if args.steps is None:
        args.steps = 3 if adjoint else 10 if field else 1000
    if args.warmup is None:
        args.warmup = 3 if adjoint or field else 100
    if args.e2e_calls is None:
        args.e2e_calls = 1 if adjoint else 2 if field else 3
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
    runner = run_adjoint if adjoint else run_field if field else run_grid
    line = runner(args, rank, world_size, local_rank, dist, base)
    if field and not args.no_sub:
        # The metric's other two numbers, measured in the same run: the batched plain step on
        # 4096 16x16-grid worlds, and adjoint world-gradients/s on 512 1024-cell Delaunay worlds
        # (2000 Rosenbrock steps, the ROS2 adjoint; the ARS(2,2,2) adjoint beside it).
        subs = {}
        for name, kw in (("grid", dict(workload="grid", worlds=4096, side=16, dt=1e-3,
                                       steps=200, warmup=100, e2e_calls=1, fuse=100)),
                         ("grid_ros2", dict(workload="grid", worlds=4096, side=16, dt=1e-3,
                                            steps=20, warmup=5, e2e_calls=0, fuse=10,
                                            method="ros2")),
                         ("precision", dict(workload="grid", worlds=4096, side=16, dt=1e-3,
                                            steps=20, warmup=5, e2e_calls=0)),
                         ("drop_in", dict(workload="grid", steps=200)),
                         ("adjoint", dict(workload="adjoint", worlds=512, dt=1e-3, steps=1,
                                          warmup=1, e2e_calls=0, method="ros2")),
                         ("adjoint_ars222", dict(workload="adjoint", worlds=512, dt=1e-3,
                                                 steps=1, warmup=1, e2e_calls=0,
                                                 method="ars222"))):
            sub = argparse.Namespace(**{**vars(args), **kw})
            fn = (run_adjoint if name.startswith("adjoint") else
                  run_precision if name == "precision" else
                  run_dropin if name == "drop_in" else run_grid)
            subs[name] = fn(sub, rank, world_size, local_rank, dist, None)
        if line is not None:
            line["sub_records"] = {k: sub_record(v) for k, v in subs.items()}
    if line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def sub_record(line):
    """The keys of a workload's line that a sub-record keeps."""
    keep = ("metric", "value", "unit", "ms_per_step", "dtype", "config", "roofline", "e2e",
            "gpu_launches", "refused_worlds", "clocks", "kernels", "pairs", "cpu_baseline",
            "note")
    return {k: line[k] for k in keep if k in line}


if __name__ == "__main__":
    sys.exit(main())
