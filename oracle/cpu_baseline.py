"""Timed CPU baseline: the oracle's step, one world per task, over a process pool.

TEST/BENCH INFRASTRUCTURE ONLY (bench.py's cpu_baseline leg and its ``--impl reference`` arm).
It mirrors how the reference runs its tissue step on a CPU: the NumPy branch of
models/surface_pump.py imex_step, one world per process, BLAS pinned to one thread
(src/cells/execution/blas_threads.py:28), a pool over the host's cores. The oracle reproduces
that step bit for bit on the golden worlds (tests/test_oracle_golden.py), so its arithmetic is
the reference's; its NumPy layout differs only in packing.
"""

from __future__ import annotations

import os
import time


def _pin_blas():
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"


def run_world(task):
    """One world: (kind, world index, seed, side or size, steps, dt) -> (cell-steps, seconds)."""
    _pin_blas()
    from cells_b200 import worlds
    from oracle import tissue as T

    kind, w, seed, size, steps, dt = task
    if kind == "grid":
        world = worlds.grid_world(size, size, worlds.world_rng(seed, w))
    else:
        world = worlds.delaunay_world(size, worlds.world_rng(seed, w))
    b = worlds.pack([world])
    topo = T.topology(b)
    ctl = T.full_control(b)
    st = T.initial_state(b)
    t0 = time.perf_counter()
    for _ in range(steps):
        st, ok = T.ars222_step(st, dt, ctl, b, topo)
    elapsed = time.perf_counter() - t0
    return world.cells * steps, elapsed


def measure(tasks, processes=None):
    """Run the tasks over a spawn pool; returns (cell-steps, wall seconds, processes)."""
    import multiprocessing as mp

    _pin_blas()
    processes = processes or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes) as pool:
        pool.map(run_world, [(t[0], t[1], t[2], t[3], 1, t[5]) for t in tasks[:processes]])
        t0 = time.perf_counter()
        results = pool.map(run_world, tasks, chunksize=1)
        wall = time.perf_counter() - t0
    return sum(r[0] for r in results), wall, processes
