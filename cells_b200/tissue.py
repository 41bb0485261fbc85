"""Host side of the device tissue step: bind a packed batch, pack/unpack state, step.

This mirrors the reference's model-module protocol for the resolved pump-leak tissue
(src/cells/models/surface_pump.py:124-369 and src/cells/models/surface_pump_v3.py:3989):

* ``Tissue(batch)``            ~ ``initial_values(spec)``'s layout binding (cb_bind)
* ``Tissue.initial_state()``   ~ ``initial_values(spec)``'s state (all increments zero)
* ``Tissue.step(...)``         ~ ``checked_step`` repeated ``n_steps`` times, every world at once
  on device buffers (cb_step); a refused world keeps its last accepted state, as the reference's
  ``where(valid, new, old)`` does (surface_pump.py:362).
* ``checked_step(...)``        ~ ``checked_step(state, dt, control, p, active) -> (state, valid)``
  with host arrays (cb_step_host), one step.
* ``Tissue.balances(...)``     ~ ``balances(state, p)``'s residuals (cb_balances).
* ``Tissue.device_checks(...)`` ~ @3's ``device_checks(previous, row, p, constants, steps)``
  (surface_pump_v3.py:5572-5597): the accepted-row checks, bitmask and diagnostics per world.
* ``Tissue.step_vjp(...)``     ~ ``jax.vjp`` of ``checked_step`` repeated ``n_steps`` times
  (cb_step_vjp_method: the ARS(2,2,2) step or ROS2); ``Tissue.set_permeability`` rebinds the permeabilities on the device.

State is a dict of NumPy arrays in the packed layout (``_lib.STATE_FIELDS``; cell fields [3, C]
or [C], junction fields [3, E] or [E], world fields [3, W] or [W]). Device buffers are torch
float64 CUDA tensors; torch is only the allocator and stream provider here.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

SPECIES_FIELDS = {"amount_increment", "membrane_transferred", "junction_transferred",
                  "reservoir_supplied"}
CHANNEL = ("channel_gate", "channel_transferred", "channel_dissipated")
CELL = ("amount_increment", "membrane_transferred", "membrane_dissipated", "pump_cycles",
        "pump_dissipated", "metabolic_work")
EDGE = ("junction_transferred", "junction_dissipated", "junction_gate")
WORLD = ("reservoir_supplied", "electrode_charge", "reservoir_work", "electrode_work")
# cb_device_checks' bits and diagnostics, in the reference's DEVICE_CHECKS and DEVICE_DIAGNOSTICS
# order (models/surface_pump_v3.py, device_checks).
CHECKS = ("domain", "local", "outside", "total", "charge", "electrode", "global_charge", "energy",
          "reservoir_work", "electrode_work", "metabolic_work", "dissipation")
DIAGNOSTICS = tuple("max_" + k for k in (
    "balance_error_fmol", "extracellular_balance_error_fmol", "global_balance_error_fmol",
    "capacitor_charge_error_C", "electrode_charge_error_C", "global_charge_error_C",
    "energy_balance_error_pJ", "reservoir_work_error_pJ", "electrode_work_error_pJ",
    "metabolic_work_error_pJ", "energy_balance_relative", "global_charge_bound_ratio"))


def _torch_int64():
    import torch

    return torch.int64


def _ptr(a, ctype=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Tissue:
    """A packed batch bound on one device (cb_bind)."""

    def __init__(self, batch, device=0):
        self.lib = _lib.load()
        self.batch = batch
        self.device = int(device)
        b = batch
        # Keep every host array alive for the duration of the bind call.
        self._keep = keep = {
            "cell_offset": np.ascontiguousarray(b.cell_offset, dtype=np.int64),
            "edge_offset": np.ascontiguousarray(b.edge_offset, dtype=np.int64),
            "temperature": np.ascontiguousarray(b.temperature, dtype=np.float64),
            "bath_amount": np.ascontiguousarray(b.bath_amount, dtype=np.float64),
            "bath_volume": np.ascontiguousarray(b.bath_volume, dtype=np.float64),
            "bath_potential": np.ascontiguousarray(b.bath_potential, dtype=np.float64),
            "pump": np.ascontiguousarray(b.pump, dtype=np.float64),
            "volume": np.ascontiguousarray(b.volume, dtype=np.float64),
            "area": np.ascontiguousarray(b.area, dtype=np.float64),
            "capacitance": np.ascontiguousarray(b.capacitance, dtype=np.float64),
            "permeability": np.ascontiguousarray(b.permeability, dtype=np.float64),
            "pump_capacity": np.ascontiguousarray(b.pump_capacity, dtype=np.float64),
            "amount_reference": np.ascontiguousarray(b.amount_reference, dtype=np.float64),
            "initial_charge": np.ascontiguousarray(b.initial_charge, dtype=np.float64),
            "sender": np.ascontiguousarray(b.sender, dtype=np.int32),
            "receiver": np.ascontiguousarray(b.receiver, dtype=np.int32),
            "junction_area": np.ascontiguousarray(b.junction_area, dtype=np.float64),
            "junction_permeability": np.ascontiguousarray(b.junction_permeability,
                                                          dtype=np.float64),
            "gate_threshold": np.ascontiguousarray(b.gate_threshold, dtype=np.float64),
            "gate_minimum": np.ascontiguousarray(b.gate_minimum, dtype=np.float64),
            "channel_code": np.ascontiguousarray(b.channel_code, dtype=np.int32),
            "channel_species": np.ascontiguousarray(b.channel_species, dtype=np.int32),
            "channel_permeability": np.ascontiguousarray(b.channel_permeability,
                                                         dtype=np.float64),
            "channel_abundance": np.ascontiguousarray(b.channel_abundance, dtype=np.float64),
        }
        desc = _lib.TissueDesc()
        desc.n_worlds = b.worlds
        desc.n_cells = b.cells
        desc.n_edges = b.edges
        desc.channel_slots = b.channel_slots
        for name, arr in keep.items():
            ctype = {np.int64: ctypes.c_int64, np.int32: ctypes.c_int32}.get(arr.dtype.type,
                                                                            ctypes.c_double)
            setattr(desc, name, _ptr(arr, ctype))
        handle = ctypes.c_void_p()
        _lib.check(self.lib.cb_bind(ctypes.byref(desc), self.device, ctypes.byref(handle)))
        self.handle = handle
        off = np.zeros(len(_lib.STATE_FIELDS), dtype=np.int64)
        total = np.zeros(1, dtype=np.int64)
        _lib.check(self.lib.cb_state_layout(self.handle, _ptr(off, ctypes.c_int64),
                                            _ptr(total, ctypes.c_int64)))
        self.state_offsets = dict(zip(_lib.STATE_FIELDS, off.tolist(), strict=True))
        self.state_size = int(total[0])
        coff = np.zeros(len(_lib.CONTROL_FIELDS), dtype=np.int64)
        _lib.check(self.lib.cb_control_layout(self.handle, _ptr(coff, ctypes.c_int64),
                                              _ptr(total, ctypes.c_int64)))
        self.control_offsets = dict(zip(_lib.CONTROL_FIELDS, coff.tolist(), strict=True))
        self.control_size = int(total[0])
        if b.channel_block is not None:
            self.set_channel_block(b.channel_block)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.cb_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- packing (host)
    def _shape(self, name):
        b = self.batch
        if name == "channel_gate":
            return (2, b.channel_slots, b.cells)
        if name in CHANNEL:
            return (b.channel_slots, b.cells)
        n = b.cells if name in CELL else b.edges if name in EDGE else b.worlds
        return (3, n) if name in SPECIES_FIELDS else (n,)

    def pack_state(self, state):
        flat = np.zeros(self.state_size)
        for name in _lib.STATE_FIELDS:
            v = np.asarray(state[name], dtype=np.float64)
            shape = self._shape(name)
            if v.shape != shape:
                raise ValueError(f"state field {name}: shape {v.shape}, expected {shape}")
            o = self.state_offsets[name]
            flat[o:o + v.size] = v.reshape(-1)
        return flat

    def unpack_state(self, flat):
        flat = np.asarray(flat)
        out = {}
        for name in _lib.STATE_FIELDS:
            shape = self._shape(name)
            o = self.state_offsets[name]
            out[name] = flat[o:o + int(np.prod(shape))].reshape(shape).copy()
        return out

    def pack_control(self, membrane=1.0, junction=1.0, pump=1.0, channel=1.0):
        b = self.batch
        flat = np.zeros(self.control_size)
        nch = b.channel_slots * b.cells
        for name, value, shape in (("membrane", membrane, (b.cells,)),
                                   ("junction", junction, (b.edges,)),
                                   ("pump", pump, (b.cells,)),
                                   ("channel", channel, (b.channel_slots, b.cells))):
            o = self.control_offsets[name]
            n = int(np.prod(shape))
            flat[o:o + n] = np.broadcast_to(np.asarray(value, dtype=np.float64), shape).reshape(-1)
        del nch
        return flat

    def initial_state(self):
        b = self.batch
        state = {name: np.zeros(self._shape(name)) for name in _lib.STATE_FIELDS}
        state["junction_gate"] = np.asarray(b.gate_initial, dtype=np.float64).copy()
        state["channel_gate"] = np.asarray(b.channel_gate_initial, dtype=np.float64).copy()
        return state

    # ---------------------------------------------------------------- device entry points
    def step(self, state_in, state_out, control, dt, n_steps, status, accepted=None, stream=None,
             method=_lib.METHOD_ARS222):
        """cb_step on device tensors (float64 state/control, int32 status/accepted)."""
        _lib.check(self.lib.cb_step(
            self.handle, int(method), ctypes.c_void_p(state_in.data_ptr()),
            ctypes.c_void_p(state_out.data_ptr()), float(dt),
            ctypes.c_void_p(control.data_ptr()), int(n_steps),
            ctypes.c_void_p(status.data_ptr()),
            None if accepted is None else ctypes.c_void_p(accepted.data_ptr()),
            None if stream is None else ctypes.c_void_p(stream),
        ))  # fmt: skip

    def set_launch(self, kernel, block=1024, occupancy=3):
        """cb_set_launch: the kernel path (_lib.KERNEL_SHARED / KERNEL_PACKED) and CTA shape."""
        _lib.check(self.lib.cb_set_launch(self.handle, int(kernel), int(block), int(occupancy)))

    def get_launch(self):
        k, b, o = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.cb_get_launch(self.handle, ctypes.byref(k), ctypes.byref(b),
                                          ctypes.byref(o)))
        return k.value, b.value, o.value

    def set_sparse_launch(self, block):
        """cb_set_sparse_launch: the ROS2/RK4 kernel's CTA threads (128 or 256; 0: the plan's
        own choice)."""
        _lib.check(self.lib.cb_set_sparse_launch(self.handle, int(block)))

    def get_sparse_launch(self):
        out = ctypes.c_int()
        _lib.check(self.lib.cb_get_sparse_launch(self.handle, ctypes.byref(out)))
        return out.value

    def capture(self, state_in, state_out, control, dt, n_steps, status, launches=1,
                accepted=None, method=_lib.METHOD_ARS222):
        """A CUDA graph of ``launches`` cb_step launches of ``n_steps`` steps each (device
        tensors, as step). Replay it with graph.replay(); the tensors must stay alive. Launches
        alternate state_in -> state_out -> state_in ... (in place when they are the same)."""
        import torch

        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=state_in.device)
        side.wait_stream(torch.cuda.current_stream(state_in.device))
        with torch.cuda.stream(side):  # first launch outside the capture sets kernel attributes
            self.step(state_in, state_out, control, dt, 0, status, accepted,
                      stream=side.cuda_stream, method=method)
        torch.cuda.current_stream(state_in.device).wait_stream(side)
        with torch.cuda.graph(graph):
            stream = torch.cuda.current_stream(state_in.device).cuda_stream
            src, dst = state_in, state_out
            for _ in range(launches):
                self.step(src, dst, control, dt, n_steps, status, accepted, stream=stream,
                          method=method)
                src, dst = dst, src
        return graph

    def step_host(self, state_in, control, dt, n_steps, method=_lib.METHOD_ARS222):
        """cb_step_host on packed host arrays; returns (state, status[W], accepted[W])."""
        src = np.ascontiguousarray(state_in, dtype=np.float64)
        ctl = np.ascontiguousarray(control, dtype=np.float64)
        out = np.empty(self.state_size)
        status = np.zeros(self.batch.worlds, dtype=np.uint32)
        taken = np.zeros(self.batch.worlds, dtype=np.int32)
        _lib.check(self.lib.cb_step_host(
            self.handle, int(method), _ptr(src), _ptr(out), float(dt), _ptr(ctl), int(n_steps),
            _ptr(status, ctypes.c_uint32), _ptr(taken, ctypes.c_int32),
        ))  # fmt: skip
        return out, status, taken

    def balances(self, state_dev, out_dev, stream=None):
        """cb_balances: out_dev [W*8] float64 device tensor."""
        _lib.check(self.lib.cb_balances(
            self.handle, ctypes.c_void_p(state_dev.data_ptr()),
            ctypes.c_void_p(out_dev.data_ptr()),
            None if stream is None else ctypes.c_void_p(stream),
        ))  # fmt: skip

    def device_checks(self, previous_dev, row_dev, steps, material_atol, energy_rtol, failed_dev,
                      values_dev, stream=None):
        """cb_device_checks: the accepted-row checks of row_dev against previous_dev (packed
        float64 device states); failed_dev [W] int32 receives each world's bitmask (bit k:
        CHECKS[k] failed), values_dev [W*12] float64 the diagnostics. steps: the accepted-step
        count, one number for every world, or an int64 device tensor [W] of each world's own
        (cb_device_checks_each)."""
        atol = (ctypes.c_double * 3)(*np.broadcast_to(np.asarray(material_atol, float), 3))
        args = (ctypes.c_void_p(previous_dev.data_ptr()), ctypes.c_void_p(row_dev.data_ptr()))
        tail = (atol, float(energy_rtol), ctypes.c_void_p(failed_dev.data_ptr()),
                ctypes.c_void_p(values_dev.data_ptr()),
                None if stream is None else ctypes.c_void_p(stream))
        if hasattr(steps, "data_ptr"):
            if steps.dtype != _torch_int64() or steps.numel() != self.batch.worlds:
                raise ValueError("per-world steps must be an int64 tensor of one entry per world")
            _lib.check(self.lib.cb_device_checks_each(
                self.handle, *args, ctypes.c_void_p(steps.data_ptr()), *tail))
        else:
            _lib.check(self.lib.cb_device_checks(self.handle, *args, int(steps), *tail))

    def copy_worlds(self, mask_dev, src_dev, dst_dev, stream=None):
        """cb_copy_worlds: every state element of each world with mask_dev[w] != 0 (int32
        device tensor [W]) from src_dev to dst_dev (packed float64 device states)."""
        _lib.check(self.lib.cb_copy_worlds(
            self.handle, ctypes.c_void_p(mask_dev.data_ptr()),
            ctypes.c_void_p(src_dev.data_ptr()), ctypes.c_void_p(dst_dev.data_ptr()),
            None if stream is None else ctypes.c_void_p(stream),
        ))  # fmt: skip

    def set_permeability(self, membrane=None, junction=None, channel=None, stream=None):
        """cb_set_permeability from float64 device tensors (m/s): membrane [3, C], junction
        [3, E], channel [NCH, C]; None keeps the bound values."""

        def ptr(t):
            return None if t is None else ctypes.c_void_p(t.data_ptr())

        for t in (membrane, junction, channel):
            if t is not None and not t.is_contiguous():
                raise ValueError("permeability tensors must be contiguous")
        _lib.check(self.lib.cb_set_permeability(
            self.handle, ptr(membrane), ptr(junction), ptr(channel),
            None if stream is None else ctypes.c_void_p(stream),
        ))  # fmt: skip

    def set_channel_block(self, block):
        """cb_set_channel_block from a worlds.ChannelBlock over the batch's cells (None: remove
        the block). A blocked batch runs on the packed kernel, FP64 ARS(2,2,2) only."""
        if block is None:
            _lib.check(self.lib.cb_set_channel_block(self.handle, 0, None, None, None, None))
            return
        arrays = [np.ascontiguousarray(a, dtype=np.float64) for a in
                  (block.weight, block.k0_mM, block.steepness, block.concentration_mM)]
        _lib.check(self.lib.cb_set_channel_block(
            self.handle, block.modes, *(_ptr(a, ctypes.c_double) for a in arrays)))

    def vjp_workspace_bytes(self, n_steps, method=_lib.METHOD_ARS222):
        out = ctypes.c_size_t()
        _lib.check(self.lib.cb_vjp_workspace_method(self.handle, int(method), int(n_steps),
                                                    ctypes.byref(out)))
        return int(out.value)

    def step_vjp(self, state_in, control, dt, n_steps, cot_out, cot_in, grad_membrane,
                 grad_junction, grad_channel, workspace, status, stream=None,
                 method=_lib.METHOD_ARS222):
        """cb_step_vjp_method on device tensors (METHOD_ARS222 or METHOD_ROS2): cotangent of the
        state after n_steps steps in, of state_in out (may alias); permeability gradients added
        to grad_* (float64 [3C], [3E], [NCH C]); workspace a uint8 tensor of
        vjp_workspace_bytes(n_steps, method); status int32 [W]."""

        def ptr(t):
            return None if t is None else ctypes.c_void_p(t.data_ptr())

        _lib.check(self.lib.cb_step_vjp_method(
            self.handle, int(method), ptr(state_in), float(dt), ptr(control), int(n_steps),
            ptr(cot_out), ptr(cot_in), ptr(grad_membrane), ptr(grad_junction), ptr(grad_channel),
            ptr(workspace), int(workspace.numel()), ptr(status),
            None if stream is None else ctypes.c_void_p(stream),
        ))  # fmt: skip


def checked_step(state, dt, control, tissue):
    """One step with host arrays: (state, valid[W]) as the reference's checked_step returns,
    every world at once. ``control`` is a dict with membrane/junction/pump availabilities."""
    flat = tissue.pack_state(state)
    ctl = tissue.pack_control(**control) if isinstance(control, dict) else control
    out, status, _ = tissue.step_host(flat, ctl, dt, 1)
    return tissue.unpack_state(out), status == 0


def decode_status(bits):
    """Names of the refusal bits of one world's status word."""
    return [name for bit, name in _lib.WORLD_BITS.items() if int(bits) & bit]
