"""Windows of steps with per-row device checks over the device step (cb_step, cb_device_checks).

Restates the reference's vector window (src/cells/execution/vector_windows.py:348-410,
``_vector_window``) for a bound batch of held-bath worlds: the window's start row is checked
against itself; then, row by row, every world takes one step with the row's step size and held
control, the accepted-row checks compare the new row with the current one (first_step + row
accepted steps), and

* a world whose step is refused (bit 0, STEP_REFUSED) or whose row fails a check (bit 1 + k for
  check k, FAILURE_SHIFT = 1) records that row as its first failing row with those bits, keeps its
  current state, and takes no further rows;
* a world whose row passes advances to it, raises its diagnostic maxima (the twelve
  DEVICE_DIAGNOSTICS of cb_device_checks) and stores the row in its observation slot;
* a world stops after its own count of rows (``counts``).

Differences from the reference, by design of the C ABI: the worlds of one batch share their
accepted-step count at the window start (``first_step`` is one number; cb_device_checks takes one
step count), and a row's step size and held control are the same for every world. The state
stays on the device; the host issues two kernels per row (the step, the checks) and a few device
selects.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np

from . import tissue as _tissue

STEP_REFUSED = "step_refused"
FAILURE_SHIFT = 1  # vector_windows.FAILURE_SHIFT: bit 0 is the refused step, checks from bit 1


class Window(NamedTuple):
    state: object    # final packed state (device tensor): each world at its last accepted row
    first: object    # [W] int32: first failing row, -1 if none
    bits: object     # [W] int64: that row's failure bits (bit 0 refused step, 1 + k check k)
    maxima: object   # [W, 12]: diagnostic maxima over the accepted rows, the start row included
    rows: object     # [R, state_total]: stored observation rows (zero where never written)


def failure_names(bits):
    """The failure names of one world's bits, in order (vector_windows._unpack)."""
    names = (STEP_REFUSED, *_tissue.CHECKS)
    return tuple(n for bit, n in enumerate(names) if int(bits) & (1 << bit))


def world_of_elements(tissue):
    """[state_total] world index of every element of the packed state."""
    b = tissue.batch
    cell_world = np.repeat(np.arange(b.worlds), np.diff(b.cell_offset))
    edge_world = np.repeat(np.arange(b.worlds), np.diff(b.edge_offset))
    world = np.arange(b.worlds)
    ids = {}
    for name, value in tissue.initial_state().items():
        shape = np.shape(value)
        if name in _tissue.WORLD:
            ids[name] = np.broadcast_to(world, shape).astype(np.float64)
        elif name in _tissue.EDGE:
            ids[name] = np.broadcast_to(edge_world, shape).astype(np.float64)
        else:  # cell and channel fields end in the cell axis
            ids[name] = np.broadcast_to(cell_world, shape).astype(np.float64)
    return tissue.pack_state(ids).astype(np.int64)


def vector_window(tissue, state, dt, controls, held, *, slots=None, counts=None, first_step=0,
                  material_atol=2e-11, energy_rtol=2e-3, rows=0, method=0, world_of=None):
    """One window of every world of a bound batch (torch float64 device tensors).

    state: packed start state [state_total]; dt: [width] step sizes; controls: [n, control_total]
    the held-control table; held: [width] row -> control index; slots: [width] row -> observation
    slot (-1 or >= rows: not stored); counts: [W] rows each world takes (default: all);
    first_step: accepted steps before the window (every world's); material_atol: per species
    (fmol); energy_rtol; rows: observation slots; method: cb_step's method; world_of: the cached
    world_of_elements(tissue) as a device tensor.
    """
    import torch

    dev = state.device
    n_worlds = tissue.batch.worlds
    width = len(dt)
    held = [int(h) for h in held]
    slots = [-1] * width if slots is None else [int(s) for s in slots]
    counts_t = torch.full((n_worlds,), width, dtype=torch.int64, device=dev) if counts is None \
        else torch.as_tensor(np.asarray(counts), dtype=torch.int64, device=dev)
    if world_of is None:
        world_of = torch.from_numpy(world_of_elements(tissue)).to(dev)
    shift = torch.arange(12, dtype=torch.int64, device=dev) + FAILURE_SHIFT
    failed = torch.zeros(n_worlds, dtype=torch.int32, device=dev)
    values = torch.zeros(n_worlds * 12, dtype=torch.float64, device=dev)
    status = torch.zeros(n_worlds, dtype=torch.int32, device=dev)

    def checks(previous, row, steps):
        tissue.device_checks(previous, row, steps, material_atol, energy_rtol, failed, values)
        bits = (failed.to(torch.int64)[:, None] >> torch.arange(12, device=dev)) & 1
        return (bits << shift).sum(dim=1), values.view(n_worlds, 12).clone()

    current = state.clone()
    bits, vals = checks(current, current, first_step)
    ok = bits == 0
    first = torch.where(ok, -1, 0).to(torch.int32)
    maxima = torch.where(ok[:, None], vals, torch.zeros_like(vals))
    stored = torch.zeros((rows, current.numel()), dtype=torch.float64, device=dev)
    updated = torch.empty_like(current)
    for j in range(1, width + 1):
        tissue.step(current, updated, controls[held[j - 1]], float(dt[j - 1]), 1, status,
                    method=method)
        row_bits, vals = checks(current, updated, first_step + j)
        flags = torch.where(status == 0, row_bits, torch.ones_like(row_bits))
        live = (j <= counts_t) & ok
        failing = live & (flags != 0)
        accept = live & (flags == 0)
        first = torch.where(failing, torch.full_like(first, j), first)
        bits = torch.where(failing, flags, bits)
        current = torch.where(accept[world_of], updated, current)
        maxima = torch.where(accept[:, None], torch.maximum(maxima, vals), maxima)
        slot = slots[j - 1]
        if 0 <= slot < rows:
            stored[slot] = torch.where(accept[world_of], current, stored[slot])
        ok = ok & ~failing
    return Window(current, first, bits, maxima, stored)
