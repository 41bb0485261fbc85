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

As the reference's, each world has its own step size, held-control index and observation slot
per row (``[W, width]``; a ``[width]`` row applies to every world) and its own accepted-step count
at the window start (``first_step``: one number or ``[W]``; cb_device_checks_each). cb_step takes
one step size per launch, so a row whose worlds take different step sizes runs the step once per
distinct size and keeps each world's own result. The state stays on the device and a row is
four launches: the step; the row's checks fused with every world's bookkeeping (cb_window_row);
the copy back of the worlds that did not advance (cb_copy_worlds, after a buffer swap); and, on a
row with observation slots, the store of the advanced worlds (cb_store_worlds).
"""

from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np

from . import _lib
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


def world_of_controls(tissue):
    """[control_total] world index of every element of the packed control (padding: 0)."""
    b = tissue.batch
    cell_world = np.repeat(np.arange(b.worlds), np.diff(b.cell_offset)).astype(np.float64)
    edge_world = np.repeat(np.arange(b.worlds), np.diff(b.edge_offset)).astype(np.float64)
    return tissue.pack_control(membrane=cell_world, junction=edge_world, pump=cell_world,
                               channel=cell_world).astype(np.int64)


def _per_world(value, n_worlds, width, dtype):
    """A row table [W, width] from [width] (every world) or [W, width]."""
    a = np.asarray(value, dtype=dtype)
    if a.ndim == 1:
        a = np.broadcast_to(a[None, :], (n_worlds, a.size))
    if a.shape != (n_worlds, width):
        raise ValueError(f"expected [{width}] or [{n_worlds}, {width}], got {a.shape}")
    return np.array(a)  # a writable copy (torch refuses read-only views)


def vector_window(tissue, state, dt, controls, held, *, slots=None, counts=None, first_step=0,
                  material_atol=2e-11, energy_rtol=2e-3, rows=0, method=0, world_of=None):
    """One window of every world of a bound batch (torch float64 device tensors).

    state: packed start state [state_total]; dt: step sizes [width] or [W, width]; controls:
    [n, control_total] the held-control table (row i packs every world's control i); held: row
    -> control index, [width] or [W, width]; slots: row -> observation slot (-1 or >= rows: not
    stored), [width] or [W, width]; counts: [W] rows each world takes (default: all);
    first_step: accepted steps before the window, one number or [W]; material_atol: per species
    (fmol); energy_rtol; rows: observation slots; method: cb_step's method; world_of: the cached
    world_of_elements(tissue) as a device tensor (used where a row's worlds take several step
    sizes). The selects of the reference's window are per-world copies (cb_copy_worlds): the
    accepted worlds' new rows become current by a buffer swap, the others' states are copied
    back.
    """
    import torch

    dev = state.device
    n_worlds = tissue.batch.worlds
    width = np.asarray(dt).shape[-1]
    dt_w = _per_world(dt, n_worlds, width, np.float64)
    held_w = _per_world(held, n_worlds, width, np.int64)
    slots_w = _per_world(np.full(width, -1) if slots is None else slots, n_worlds, width,
                         np.int64)
    counts_t = torch.full((n_worlds,), width, dtype=torch.int64, device=dev) if counts is None \
        else torch.as_tensor(np.asarray(counts), dtype=torch.int64, device=dev)
    per_world_first = np.ndim(first_step) > 0
    first_t = torch.as_tensor(np.array(np.broadcast_to(np.asarray(first_step, np.int64),
                                                       (n_worlds,))),
                              dtype=torch.int64, device=dev)
    if world_of is None and np.any(dt_w != dt_w[:1]):  # only rows of several step sizes use it
        world_of = torch.from_numpy(world_of_elements(tissue)).to(dev)
    # The per-world row tables on the device once (an upload inside the loop would wait for the
    # device to drain each row).
    slots_dev = torch.as_tensor(np.ascontiguousarray(slots_w.T), device=dev)  # [width, W]
    held_dev = torch.as_tensor(held_w, device=dev)
    dt_dev = torch.as_tensor(dt_w, device=dev)
    ctl_world = None
    if np.any(held_w != held_w[:1]):
        ctl_world = torch.from_numpy(world_of_controls(tissue)).to(dev)
        ctl_index = torch.arange(controls.shape[1], device=dev)
    lib = tissue.lib
    atol = (ctypes.c_double * 3)(*np.broadcast_to(np.asarray(material_atol, float), 3))
    first_ptr = ctypes.c_void_p(first_t.data_ptr()) if per_world_first else None
    first_all = 0 if per_world_first else int(first_step)
    ok = torch.zeros(n_worlds, dtype=torch.int32, device=dev)
    first = torch.zeros(n_worlds, dtype=torch.int32, device=dev)
    bits = torch.zeros(n_worlds, dtype=torch.int64, device=dev)
    maxima = torch.zeros((n_worlds, 12), dtype=torch.float64, device=dev)
    keep = torch.ones(n_worlds, dtype=torch.int32, device=dev)
    status = torch.zeros(n_worlds, dtype=torch.int32, device=dev)

    def ptr(x):
        return ctypes.c_void_p(x.data_ptr())

    def window_row(previous, row, j):
        """cb_window_row: the row's checks and every world's bookkeeping, one launch."""
        _lib.check(lib.cb_window_row(
            tissue.handle, ptr(previous), ptr(row), j, first_ptr, first_all, atol,
            float(energy_rtol), ptr(status), ptr(counts_t), ptr(ok), ptr(first), ptr(bits),
            ptr(maxima), ptr(keep), None))  # fmt: skip

    current = state.clone()
    window_row(current, current, 0)
    stored = torch.zeros((rows, current.numel()), dtype=torch.float64, device=dev)
    updated = torch.empty_like(current)
    for j in range(1, width + 1):
        col = j - 1
        if ctl_world is None:
            control = controls[int(held_w[0, col])]
        else:
            control = controls[held_dev[:, col][ctl_world], ctl_index]
        sizes = np.unique(dt_w[:, col])
        if sizes.size == 1:
            tissue.step(current, updated, control, float(sizes[0]), 1, status, method=method)
        else:  # one launch per distinct step size, each world keeping its own
            trial = torch.empty_like(current)
            trial_status = torch.empty_like(status)
            dt_t = dt_dev[:, col]
            for size in sizes:
                tissue.step(current, trial, control, float(size), 1, trial_status,
                            method=method)
                take = dt_t == float(size)
                updated.copy_(torch.where(take[world_of], trial, updated))
                status.copy_(torch.where(take, trial_status, status))
        window_row(current, updated, j)
        # The accepted worlds advance: swap the buffers and copy the others' states back.
        tissue.copy_worlds(keep, current, updated)
        current, updated = updated, current
        if rows and np.any((slots_w[:, col] >= 0) & (slots_w[:, col] < rows)):
            _lib.check(lib.cb_store_worlds(tissue.handle, ptr(keep), ptr(slots_dev[col]),
                                           ptr(current), ptr(stored), rows, None))
    return Window(current, first, bits, maxima, stored)
