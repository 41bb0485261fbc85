"""Launch autotuner for a bound batch: picks the kernel path and CTA shape that steps fastest.

Candidates: the one-world-per-CTA shared-memory kernel at 3 or 2 resident CTAs per SM (when the
worlds fit it) and the packed persistent kernel with 256-, 512- and 1024-thread CTAs (when the
worlds fit a work item). Each candidate advances a copy of the given state by ``steps`` steps,
``repeats`` times after one warm-up launch, timed with CUDA events on the launching stream; the
fastest is left selected on the handle (cb_set_launch). Results are kept per process, keyed by the
device and the batch's shape, so a second tissue of the same shape reuses them.
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
