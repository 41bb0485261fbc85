"""Launch autotuner for a bound batch: picks the kernel path and CTA shape that steps fastest.

``tune``: the explicit step's candidates, the one-world-per-CTA shared-memory kernel at 3 or 2
resident CTAs per SM (when the worlds fit it) and the packed persistent kernel with 256-, 512- and
1024-thread CTAs (when the worlds fit a work item); the fastest is left selected (cb_set_launch).
``tune_sparse``: the sparse-factor Rosenbrock kernel (ROS2, its FP32-factor form, RK4) with
128-thread CTAs at four per SM or 256-thread CTAs at two (cb_set_sparse_launch). Each candidate
advances a copy of the given state by ``steps`` steps, ``repeats`` times after one warm-up launch,
timed with CUDA events on the launching stream. Results are kept per process, keyed by the device
and the batch's shape, so a second tissue of the same shape reuses them.
"""

from __future__ import annotations

import numpy as np

from . import _lib

_CACHE = {}


def candidates(tissue):
    out = [(_lib.KERNEL_SHARED, 256, 3), (_lib.KERNEL_SHARED, 256, 2)]
    out += [(_lib.KERNEL_PACKED, b, 1) for b in (256, 512, 1024)]
    return out


def signature(tissue):
    b = tissue.batch
    sizes = np.diff(b.cell_offset)
    return (tissue.device, b.worlds, b.cells, b.edges, b.channel_slots, int(sizes.max()),
            int(sizes.min()))


def tune(tissue, state, control, dt, steps=20, repeats=2, torch=None,
         method=_lib.METHOD_ARS222):
    """Time every feasible launch configuration and select the fastest. ``state`` and ``control``
    are device tensors (packed layout); ``state`` is not modified. Returns (best, timings), the
    timings in ms per step."""
    import torch as _torch

    torch = torch or _torch
    key = signature(tissue) + (method,)
    if key in _CACHE:
        best = _CACHE[key][0]
        tissue.set_launch(*best)
        return _CACHE[key]
    dev = state.device
    work = state.clone()
    status = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    timings = {}
    for cand in candidates(tissue):
        try:
            tissue.set_launch(*cand)
        except RuntimeError:
            continue  # infeasible for these worlds
        work.copy_(state)
        try:
            tissue.step(work, work, control, dt, steps, status, stream=stream.cuda_stream,
                        method=method)
        except RuntimeError:
            continue  # this method does not run on this kernel path
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(repeats):
            tissue.step(work, work, control, dt, steps, status, stream=stream.cuda_stream,
                        method=method)
        stop.record(stream)
        torch.cuda.synchronize(dev)
        timings[cand] = start.elapsed_time(stop) / (repeats * steps)
    if not timings:
        raise RuntimeError("no launch configuration fits this batch")
    best = min(timings, key=timings.get)
    tissue.set_launch(*best)
    _CACHE[key] = (best, timings)
    return best, timings


def tune_sparse(tissue, state, control, dt, steps=5, repeats=2, torch=None,
                method=_lib.METHOD_ROS2):
    """Time the ROS2/RK4 kernel's CTA shapes (128 and 256 threads) on a copy of ``state`` and
    select the faster (cb_set_sparse_launch). Returns (best block, {block: ms per step})."""
    import torch as _torch

    torch = torch or _torch
    key = signature(tissue) + ("sparse", method)
    if key in _CACHE:
        tissue.set_sparse_launch(_CACHE[key][0])
        return _CACHE[key]
    dev = state.device
    work = state.clone()
    status = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    timings = {}
    for block in (128, 256):
        tissue.set_sparse_launch(block)
        work.copy_(state)
        tissue.step(work, work, control, dt, steps, status, stream=stream.cuda_stream,
                    method=method)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(repeats):
            tissue.step(work, work, control, dt, steps, status, stream=stream.cuda_stream,
                        method=method)
        stop.record(stream)
        torch.cuda.synchronize(dev)
        timings[block] = start.elapsed_time(stop) / (repeats * steps)
    best = min(timings, key=timings.get)
    tissue.set_sparse_launch(best)
    _CACHE[key] = (best, timings)
    return best, timings
