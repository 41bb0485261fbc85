"""Timed CPU baseline: the oracle's step, one world per task, over a process pool.

TEST/BENCH INFRASTRUCTURE ONLY (bench.py's cpu_baseline leg and its ``--impl reference`` arm).
It mirrors how the reference runs its tissue step on a CPU: the NumPy branch of
models/surface_pump.py imex_step, one world per process, BLAS pinned to one thread
(src/cells/execution/blas_threads.py:28), a pool over the host's cores. The oracle reproduces
that step bit for bit on the golden worlds (tests/test_oracle_golden.py), so its arithmetic is
the reference's; its NumPy layout differs only in packing.

Each worker process builds a world once and keeps its state, so a task times only the steps it
takes (as the reference's runner keeps a world's state between dispatches).
"""

from __future__ import annotations

import os
import time

import numpy as np

_WORLDS = {}


def _pin_blas():
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"


def _world(kind, w, seed, size):
    key = (kind, w, seed, size)
    if key not in _WORLDS:
        from cells_b200 import worlds
        from oracle import tissue as T

        if kind == "grid":
            world = worlds.grid_world(size, size, worlds.world_rng(seed, w))
        elif kind in ("uneven", "adjoint", "adjoint_ros2"):  # world w of an uneven or adjoint
            # batch (size given)
            world = worlds.uneven_world(w, size, seed, worlds.UNEVEN_CHANNELS)
        else:
            world = worlds.delaunay_world(size, worlds.world_rng(seed, w))
        b = worlds.pack([world])
        _WORLDS[key] = [b, T.topology(b), T.full_control(b), T.initial_state(b)]
    return _WORLDS[key]


def run_world(task):
    """(kind, world index, seed, side or size, steps, dt) -> (cell-steps, seconds of stepping)."""
    _pin_blas()
    from oracle import tissue as T

    kind, w, seed, size, steps, dt = task
    entry = _world(kind, w, seed, size)
    b, topo, ctl, st = entry
    t0 = time.perf_counter()
    for _ in range(steps):
        st, _ = T.ars222_step(st, dt, ctl, b, topo)
    elapsed = time.perf_counter() - t0
    entry[3] = st
    return b.cells * steps, elapsed


def run_field_world(task):
    """("field", world index, seed, (grid side, tissue side, stride), steps, dt) -> (cell-steps,
    seconds): the field oracle's ARS(2,2,2) step (the reference's face-electromigration step;
    dense node-space algebra on small grids, the same algebra in sparse containers on larger
    ones) on one field world of that shape."""
    _pin_blas()
    from cells_b200 import field_worlds, worlds
    from oracle import field as OF

    kind, w, seed, shape, steps, dt = task
    key = (kind, w, seed, tuple(shape))
    if key not in _WORLDS:
        side, cells_side, stride = shape
        world = field_worlds.field_world(side, cells_side, stride, worlds.world_rng(seed, w))
        _WORLDS[key] = [world, OF.bind(world), OF.full_control(world), OF.initial_state(world)]
    entry = _WORLDS[key]
    world, tp, ctl, st = entry
    t0 = time.perf_counter()
    for _ in range(steps):
        st, _ = OF.imex_step(st, dt, ctl, world, tp)
    elapsed = time.perf_counter() - t0
    entry[3] = st
    return world.cells * steps, elapsed


def run_adjoint_world(task):
    """(kind, world index, seed, size, steps, dt) -> (cell-steps, seconds): steps forward steps
    of the oracle, each state kept, then the oracle adjoint back over them from the cotangent of
    the voltage-pattern loss (the gradient a trajectory of that many steps takes). Kind
    "adjoint": the ARS(2,2,2) step and its adjoint; "adjoint_ros2": the ROS2 step and its."""
    _pin_blas()
    from cells_b200 import worlds
    from oracle import adjoint as A
    from oracle import ros2 as R2
    from oracle import ros2_adjoint as RA
    from oracle import tissue as T

    kind, w, seed, size, steps, dt = task
    entry = _world(kind, w, seed, size)
    b, topo, ctl, st = entry
    target = worlds.voltage_target(b)
    forward = R2.ros2_step if kind == "adjoint_ros2" else T.ars222_step
    reverse = RA.step_vjp if kind == "adjoint_ros2" else A.step_vjp
    t0 = time.perf_counter()
    states = [st]
    for _ in range(steps):
        states.append(forward(states[-1], dt, ctl, b, topo)[0])
    _, cot_n = A.voltage_loss(states[-1], b, topo, target)
    cot = (cot_n, np.zeros(b.edges), np.zeros_like(st.channel_gate))
    for t in range(steps - 1, -1, -1):
        cot, _, _, _ = reverse(states[t], dt, ctl, b, topo, *cot)
    return b.cells * steps, time.perf_counter() - t0


def prepare(task):
    """Build (and keep) a task's world in this worker without stepping it."""
    _pin_blas()
    kind, w, seed, size, _, dt = task
    if kind == "field":
        run_field_world((kind, w, seed, size, 0, dt))
    else:
        _world(kind, w, seed, size)
    return os.getpid()


def pool(processes=None):
    import multiprocessing as mp

    _pin_blas()
    ctx = mp.get_context("spawn")
    return ctx.Pool(processes or os.cpu_count() or 1)


def measure(tasks, processes=None, fn=None):
    """Run the tasks over a spawn pool; returns (cell-steps, wall seconds, processes).

    Every task's world is built in a warm-up pass (one step each) before the timed pass, so the
    wall time covers stepping and the pool's dispatch only. ``fn``: run_world (default) or
    run_adjoint_world."""
    processes = processes or os.cpu_count() or 1
    fn = fn or run_world
    with pool(processes) as p:
        p.map(fn, [t[:4] + (1, t[5]) for t in tasks], chunksize=1)
        t0 = time.perf_counter()
        results = p.map(fn, tasks, chunksize=1)
        wall = time.perf_counter() - t0
    return sum(r[0] for r in results), wall, processes
