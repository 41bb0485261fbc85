"""Gradients of tissue trajectories with respect to the permeabilities, at the torch autograd
boundary: a ``torch.autograd.Function`` over cb_step (forward) and cb_step_vjp (reverse), with
checkpoints every K steps and recomputation.

    final, refused = adjoint.trajectory(tissue, state0, control, dt, n_steps,
                                        membrane, junction, channel, every=100)
    loss = adjoint.voltage_loss(tissue, final, target).sum()
    loss.backward()            # membrane.grad [3, C], junction.grad [3, E], channel.grad [NCH, C]

The forward runs the FP64 step of ``method`` (METHOD_ARS222, the reference's ARS(2,2,2), or
METHOD_ROS2, the Rosenbrock step) for n_steps steps in segments of ``every`` steps and keeps each
segment's first state (the checkpoints). The reverse walks the segments last to first:
cb_step_vjp_method recomputes a segment from its checkpoint (one step per launch, each
step-start state kept in a workspace of one segment; for ROS2 also each step's factor of its
voltage operator, which the transposed stage solves reuse) and applies the transposed step,
carrying the state's cotangent and adding the permeability gradients. Peak device memory: the
checkpoints (n_steps / every states) plus one segment of states (and, for ROS2, records).

The reference differentiates its step with JAX (``jax.jvp``/``jacfwd`` in
src/cells/analysis/stationary.py:505-514); a loss gradient there would be ``jax.grad`` of the
composed ``checked_step``. Gradients of the ledgers are not formed (they never feed back into the
dynamics); a loss that reads a ledger field gets world status CB_WORLD_LEDGER_COTANGENT in
``tissue.last_vjp_status``.
"""

from __future__ import annotations

import numpy as np


def _torch():
    import torch

    return torch


class _Trajectory:
    """Built lazily so importing this module does not import torch."""

    fn = None

    @classmethod
    def get(cls):
        if cls.fn is None:
            torch = _torch()

            class Trajectory(torch.autograd.Function):
                @staticmethod
                def forward(ctx, membrane, junction, channel, state0, tissue, control, dt,
                            n_steps, every, method):
                    nch = tissue.batch.channel_slots
                    tissue.set_permeability(membrane.contiguous(), junction.contiguous(),
                                            channel.contiguous() if nch else None)
                    dev = state0.device
                    w = tissue.batch.worlds
                    status = torch.zeros(w, dtype=torch.int32, device=dev)
                    refused = torch.zeros(w, dtype=torch.int32, device=dev)
                    checkpoints, lengths = [], []
                    state = state0.detach().clone()
                    done = 0
                    while done < n_steps:
                        k = min(every, n_steps - done)
                        checkpoints.append(state)
                        lengths.append(k)
                        nxt = torch.empty_like(state)
                        tissue.step(state, nxt, control, dt, k, status, method=method)
                        refused |= status
                        state = nxt
                        done += k
                    ctx.tissue, ctx.control, ctx.dt, ctx.method = tissue, control, dt, method
                    ctx.checkpoints, ctx.lengths = checkpoints, lengths
                    ctx.save_for_backward(membrane, junction, channel)
                    ctx.mark_non_differentiable(refused)
                    return state, refused

                @staticmethod
                def backward(ctx, grad_state, grad_status):
                    del grad_status
                    tissue = ctx.tissue
                    membrane, junction, channel = ctx.saved_tensors
                    nch = tissue.batch.channel_slots
                    b = tissue.batch
                    dev = grad_state.device
                    # The bound permeabilities may have changed since the forward.
                    tissue.set_permeability(membrane.contiguous(), junction.contiguous(),
                                            channel.contiguous() if nch else None)
                    cot = grad_state.detach().to(torch.float64).contiguous().clone()
                    gm = torch.zeros(3 * b.cells, dtype=torch.float64, device=dev)
                    gj = torch.zeros(max(3 * b.edges, 1), dtype=torch.float64, device=dev)
                    gch = torch.zeros(max(nch * b.cells, 1), dtype=torch.float64, device=dev)
                    status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
                    bits = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
                    if ctx.lengths:
                        ws = torch.empty(tissue.vjp_workspace_bytes(max(ctx.lengths), ctx.method),
                                         dtype=torch.uint8, device=dev)
                    for start, k in zip(reversed(ctx.checkpoints), reversed(ctx.lengths),
                                        strict=True):
                        tissue.step_vjp(start, ctx.control, ctx.dt, k, cot, cot, gm, gj,
                                        gch if nch else None, ws, status, method=ctx.method)
                        bits |= status
                    ctx.checkpoints = None
                    tissue.last_vjp_status = bits
                    return (gm.view(3, b.cells), gj[:3 * b.edges].view(3, b.edges),
                            gch[:nch * b.cells].view(nch, b.cells), cot,
                            None, None, None, None, None, None)

            cls.fn = Trajectory
        return cls.fn


def permeabilities(tissue, device=None):
    """The batch's permeabilities as float64 device tensors (membrane [3, C], junction [3, E],
    channel [NCH, C]), ready to take requires_grad_()."""
    torch = _torch()
    dev = torch.device("cuda", tissue.device) if device is None else device
    b = tissue.batch

    def t(a):
        return torch.tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

    return t(b.permeability), t(b.junction_permeability), t(b.channel_permeability)


def trajectory(tissue, state, control, dt, n_steps, membrane, junction, channel=None, every=100,
               method=None):
    """The state after n_steps FP64 steps of ``method`` (default METHOD_ARS222; or METHOD_ROS2)
    from ``state`` (a float64 device tensor in the state layout), differentiable with respect to
    the permeabilities (and ``state``). Returns
    (final state, refused[W]): refused holds the refusal bits met on the way (a world refused at
    a step stays where it was for that step, and its gradient is that of the map it followed)."""
    torch = _torch()
    if every < 1:
        raise ValueError("every must be at least 1")
    if channel is None:
        channel = torch.zeros((tissue.batch.channel_slots, tissue.batch.cells),
                              dtype=torch.float64, device=state.device)
    from . import _lib

    method = _lib.METHOD_ARS222 if method is None else int(method)
    if method not in (_lib.METHOD_ARS222, _lib.METHOD_ROS2):
        raise ValueError("the reverse covers METHOD_ARS222 and METHOD_ROS2")
    return _Trajectory.get().apply(membrane, junction, channel, state, tissue, control, float(dt),
                                   int(n_steps), int(every), method)


def _cell_constants(tissue, device):
    """Anchor charges, reciprocal capacitances and cell worlds on the device, kept on the
    tissue object per device."""
    cache = tissue.__dict__.setdefault("_voltage_constants", {})
    key = str(device)
    if key not in cache:
        torch = _torch()
        b = tissue.batch
        world = np.repeat(np.arange(b.worlds), np.diff(b.cell_offset))
        cache[key] = (
            torch.tensor(b.initial_charge, dtype=torch.float64, device=device),
            torch.tensor(1.0 / b.capacitance, dtype=torch.float64, device=device),
            torch.tensor(world, dtype=torch.int64, device=device),
        )
    return cache[key]


def membrane_voltage(tissue, state):
    """Membrane voltage per cell (V) of a state tensor: (Q0 + F sum_s z_s n_s) / C, the capacitor
    closure of the step, in torch ops (differentiable)."""
    from .worlds import CHARGE_PER_FMOL

    q0, icap, _ = _cell_constants(tissue, state.device)
    c = tissue.batch.cells
    o = tissue.state_offsets["amount_increment"]
    n = state[o:o + 3 * c].view(3, c)
    return (q0 + CHARGE_PER_FMOL * ((n[0] + n[1]) + (-n[2]))) * icap


def voltage_loss(tissue, state, target):
    """Per-world sum over cells of (V_m - target)^2 (V^2), [W]."""
    torch = _torch()
    _, _, world = _cell_constants(tissue, state.device)
    d = membrane_voltage(tissue, state) - target
    out = torch.zeros(tissue.batch.worlds, dtype=torch.float64, device=state.device)
    return out.index_add(0, world, d * d)
