"""Host side of the resolved-field step (cb_field_*): worlds whose cells face an extracellular grid.

Mirrors the reference's model-module protocol for ``cells.model.resolved_pump_tissue@1`` with
outside nodes and faces (src/cells/models/surface_pump.py:124-369):

* ``FieldTissue(worlds)``       ~ ``initial_values(spec)``'s layout binding (cb_field_bind): the
  capacitor components, the free nodes' nested-dissection plan, the parameters on the device;
* ``FieldTissue.initial_state()`` ~ ``initial_values(spec)``'s state (zero increments, the
  junctions' initial gates);
* ``FieldTissue.step(...)``     ~ ``checked_step`` repeated ``n_steps`` times for every world on
  device buffers (cb_field_step); a refused world keeps its last accepted state;
* ``FieldTissue.step_host(...)`` the same with host arrays (cb_field_step_host);
* ``FieldBatch(worlds)``        worlds of different geometries in one batch, as the reference's
  vector windows take them (src/cells/execution/vector_windows.py:348-410: each world its own
  layout, padded to common capacities): one FieldTissue per distinct topology, each with its own
  nested-dissection plan, stepped in turn; states and controls per world.

Every world of a FieldTissue shares one topology (grid, cells' nodes, junction graph);
parameters are per world. State is a dict of NumPy arrays [W, ...] per field
(``_lib.FIELD_STATE_FIELDS``; cell fields [W, 3, N] or [W, N], node fields [W, 3, O] or [W, O],
junction fields [W, 3, E] or [W, E], face fields [W, 3, F] or [W, F]); on the device it is one
packed float64 buffer, species-major ([3][W*X]) within a field.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

SPECIES3 = {"amount_increment": "N", "extracellular_increment": "O", "membrane_transferred": "N",
            "junction_transferred": "E", "face_transferred": "F", "reservoir_supplied": "O"}
SCALAR = {"membrane_dissipated": "N", "junction_dissipated": "E", "face_dissipated": "F",
          "electrode_charge": "O", "reservoir_work": "O", "electrode_work": "O",
          "junction_gate": "E", "pump_cycles": "N", "pump_dissipated": "N",
          "metabolic_work": "N"}
TOPOLOGY = ("side", "cell_node", "sender", "receiver", "face_sender", "face_receiver",
            "reservoir")


def topology_key(world):
    """A world's topology as a hashable key: the fields a FieldTissue's worlds must share."""
    return tuple((name, np.asarray(getattr(world, name)).dtype.str,
                  np.asarray(getattr(world, name)).shape,
                  np.ascontiguousarray(getattr(world, name)).tobytes()) for name in TOPOLOGY)


def group_by_topology(worlds):
    """Index lists of the worlds that share a topology, in order of first appearance; each list
    ascending."""
    groups = {}
    for i, w in enumerate(worlds):
        groups.setdefault(topology_key(w), []).append(i)
    return list(groups.values())


def _same_topology(worlds):
    first = worlds[0]
    for w in worlds[1:]:
        for name in TOPOLOGY:
            if not np.array_equal(np.asarray(getattr(w, name)), np.asarray(getattr(first, name))):
                raise ValueError(f"field worlds of one batch must share their topology ({name})")


class FieldTissue:
    """A batch of field worlds bound on one device (cb_field_bind)."""

    def __init__(self, worlds, device=0):
        if not worlds:
            raise ValueError("no worlds")
        _same_topology(worlds)
        self.lib = _lib.load()
        self.worlds = list(worlds)
        self.device = int(device)
        w0 = worlds[0]
        self.W, self.N, self.O, self.E, self.F = (len(worlds), w0.cells, w0.nodes, w0.edges,
                                                  w0.faces)

        def stack(name, species=False):
            a = np.stack([np.asarray(getattr(w, name), dtype=np.float64) for w in worlds])
            if species:  # [W, 3, X] -> [3, W*X]
                a = np.transpose(a, (1, 0, 2)).reshape(3, -1)
            return np.ascontiguousarray(a.reshape(-1) if not species else a)

        keep = self._keep = {
            "cell_node": np.ascontiguousarray(w0.cell_node, dtype=np.int64),
            "sender": np.ascontiguousarray(w0.sender, dtype=np.int64),
            "receiver": np.ascontiguousarray(w0.receiver, dtype=np.int64),
            "face_sender": np.ascontiguousarray(w0.face_sender, dtype=np.int64),
            "face_receiver": np.ascontiguousarray(w0.face_receiver, dtype=np.int64),
            "reservoir": np.ascontiguousarray(w0.reservoir, dtype=np.uint8),
            "temperature": np.array([w.temperature for w in worlds], dtype=np.float64),
            "pump": np.ascontiguousarray(np.array([w.pump for w in worlds], dtype=np.float64).T),
            "volume": stack("volume"), "area": stack("area"), "capacitance": stack("capacitance"),
            "permeability": stack("permeability", True), "pump_capacity": stack("pump_capacity"),
            "amount": stack("amount", True), "initial_charge": stack("initial_charge"),
            "junction_area": stack("junction_area"),
            "junction_permeability": stack("junction_permeability", True),
            "gate_threshold": stack("gate_threshold"), "gate_minimum": stack("gate_minimum"),
            "outside_volume": stack("outside_volume"),
            "outside_amount": stack("outside_amount", True),
            "outside_charge": stack("outside_charge"), "boundary_V": stack("boundary_V"),
            "face_factor": np.ascontiguousarray(np.transpose(
                np.stack([w.face_factor for w in worlds]), (1, 0, 2)).reshape(3, -1)),
        }  # fmt: skip

        def ptr(name, ctype=ctypes.c_double):
            return keep[name].ctypes.data_as(ctypes.POINTER(ctype))

        d = _lib.FieldDesc()
        d.worlds, d.cells, d.nodes, d.junctions, d.faces = self.W, self.N, self.O, self.E, self.F
        for name in ("cell_node", "face_sender", "face_receiver"):
            setattr(d, name, ptr(name, ctypes.c_int64))
        d.junction_sender = ptr("sender", ctypes.c_int64)
        d.junction_receiver = ptr("receiver", ctypes.c_int64)
        d.reservoir = ptr("reservoir", ctypes.c_uint8)
        for name in ("temperature", "pump", "volume", "area", "capacitance", "permeability",
                     "pump_capacity", "amount", "initial_charge", "junction_area",
                     "junction_permeability", "gate_threshold", "gate_minimum", "outside_volume",
                     "outside_amount", "outside_charge", "boundary_V", "face_factor"):
            setattr(d, name, ptr(name))
        handle = ctypes.c_void_p()
        _lib.check(self.lib.cb_field_bind(ctypes.byref(d), self.device, ctypes.byref(handle)))
        self.handle = handle
        offsets = (ctypes.c_int64 * len(_lib.FIELD_STATE_FIELDS))()
        total = ctypes.c_int64()
        _lib.check(self.lib.cb_field_state_layout(self.handle, offsets, ctypes.byref(total)))
        self.offsets = dict(zip(_lib.FIELD_STATE_FIELDS, list(offsets), strict=True))
        self.state_total = int(total.value)
        self.control_total = int(self.lib.cb_field_control_length(self.handle))

    def info(self):
        """cb_field_info: the solver's sizes (free nodes, fronts, levels, factor / update doubles
        per world, shared memory per CTA, scratch bytes)."""
        out = (ctypes.c_int64 * 8)()
        _lib.check(self.lib.cb_field_info(self.handle, out))
        keys = ("unknowns", "supernodes", "levels", "factor_doubles", "update_doubles",
                "vector_doubles", "smem_bytes", "scratch_bytes")
        return dict(zip(keys, (int(v) for v in out), strict=True))

    def counts(self):
        """cb_field_counts: the last step call's launches, factorisations and solves."""
        out = (ctypes.c_int64 * 3)()
        _lib.check(self.lib.cb_field_counts(self.handle, out))
        return {"launches": int(out[0]), "factorisations": int(out[1]), "solves": int(out[2])}

    def flops(self):
        """cb_field_flops: per world, the flops of one factorisation and of one solve."""
        out = (ctypes.c_double * 2)()
        _lib.check(self.lib.cb_field_flops(self.handle, out))
        return {"factor": float(out[0]), "solve": float(out[1])}

    def level_kinds(self):
        """cb_field_levels: per level of the factor plan (leaves first), 0 when its fronts go one
        per warp, 1 when one per CTA (the separators' group kernels), 2 when one per CTA with the
        wide factor (fronts of 48 columns or more)."""
        n = int(self.lib.cb_field_levels(self.handle, None, 0))
        if n < 0:
            raise RuntimeError("cb_field_levels: null handle")
        out = (ctypes.c_int32 * max(n, 1))()
        self.lib.cb_field_levels(self.handle, out, n)
        return [int(v) for v in out[:n]]

    def launches(self):
        """Kernels launched by the last step call (cb_field_launches)."""
        return int(self.lib.cb_field_launches(self.handle))

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            self.lib.cb_field_free(handle)
            self.handle = None

    def _size(self, letter):
        return {"N": self.N, "O": self.O, "E": self.E, "F": self.F}[letter]

    def initial_state(self):
        out = {}
        for name, x in SPECIES3.items():
            out[name] = np.zeros((self.W, 3, self._size(x)))
        for name, x in SCALAR.items():
            out[name] = np.zeros((self.W, self._size(x)))
        out["junction_gate"] = np.stack([np.asarray(w.gate_initial, dtype=float)
                                         for w in self.worlds])
        return out

    def pack_state(self, state):
        buf = np.zeros(self.state_total)
        for name in _lib.FIELD_STATE_FIELDS:
            a = np.asarray(state[name], dtype=np.float64)
            off = self.offsets[name]
            if name in SPECIES3:
                flat = np.transpose(a, (1, 0, 2)).reshape(-1)
            else:
                flat = a.reshape(-1)
            buf[off:off + flat.size] = flat
        return buf

    def unpack_state(self, buf):
        out = {}
        for name in _lib.FIELD_STATE_FIELDS:
            off = self.offsets[name]
            if name in SPECIES3:
                x = self._size(SPECIES3[name])
                a = buf[off:off + 3 * self.W * x].reshape(3, self.W, x)
                out[name] = np.ascontiguousarray(np.transpose(a, (1, 0, 2)))
            else:
                x = self._size(SCALAR[name])
                out[name] = buf[off:off + self.W * x].reshape(self.W, x).copy()
        return out

    def pack_control(self, membrane=None, junction=None, pump=None):
        """Availabilities [W, N], [W, E], [W, N] (default 1) -> the packed control buffer."""
        def part(v, size):
            return np.ones(self.W * size) if v is None else np.broadcast_to(
                np.asarray(v, dtype=np.float64), (self.W, size)).reshape(-1)

        return np.concatenate((part(membrane, self.N), part(junction, self.E),
                               part(pump, self.N)))

    def step(self, state_in, state_out, control, dt, n_steps, status, taken=None, stream=None):
        """cb_field_step on float64 device tensors (torch): state [state_total], control
        [control_total], status [W] int32, taken [W] int32 or None."""
        _lib.check(self.lib.cb_field_step(
            self.handle, ctypes.c_void_p(state_in.data_ptr()),
            ctypes.c_void_p(state_out.data_ptr()), float(dt), ctypes.c_void_p(control.data_ptr()),
            int(n_steps), ctypes.c_void_p(status.data_ptr()),
            None if taken is None else ctypes.c_void_p(taken.data_ptr()),
            None if stream is None else ctypes.c_void_p(stream),
        ))  # fmt: skip

    def step_host_packed(self, state_in, state_out, control, dt, n_steps, status, taken):
        """cb_field_step_host on packed host buffers (numpy float64 [state_total], control
        [control_total], uint32 / int32 [W]); pinned memory copies fastest."""
        _lib.check(self.lib.cb_field_step_host(
            self.handle, state_in.ctypes.data_as(_lib._d), state_out.ctypes.data_as(_lib._d),
            float(dt), control.ctypes.data_as(_lib._d), int(n_steps),
            status.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            taken.ctypes.data_as(_lib._i32),
        ))  # fmt: skip

    def step_host(self, state, control, dt, n_steps):
        """cb_field_step_host: host arrays in and out. Returns (state dict, status, taken)."""
        src = np.ascontiguousarray(self.pack_state(state))
        dst = np.empty_like(src)
        ctl = np.ascontiguousarray(control, dtype=np.float64)
        status = np.zeros(self.W, dtype=np.uint32)
        taken = np.zeros(self.W, dtype=np.int32)
        _lib.check(self.lib.cb_field_step_host(
            self.handle, src.ctypes.data_as(_lib._d), dst.ctypes.data_as(_lib._d), float(dt),
            ctl.ctypes.data_as(_lib._d), int(n_steps),
            status.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
            taken.ctypes.data_as(_lib._i32),
        ))  # fmt: skip
        return self.unpack_state(dst), status, taken


class FieldBatch:
    """Field worlds of different geometries (grids, tissues, contact graphs) in one batch: the
    worlds grouped by topology (group_by_topology), each group bound as one FieldTissue with its
    own factor plan; a step advances every group in turn on one device. States, controls and the
    per-world status are in the batch's world order."""

    def __init__(self, worlds, device=0):
        if not worlds:
            raise ValueError("no worlds")
        self.worlds = list(worlds)
        self.W = len(self.worlds)
        self.device = int(device)
        self.groups = [(idx, FieldTissue([self.worlds[i] for i in idx], device=device))
                       for idx in group_by_topology(self.worlds)]

    def initial_state(self):
        """One state dict per world (each field [3, X] or [X])."""
        out = [None] * self.W
        for idx, tissue in self.groups:
            st = tissue.initial_state()
            for k, i in enumerate(idx):
                out[i] = {name: a[k].copy() for name, a in st.items()}
        return out

    def step_host(self, states, dt, n_steps, controls=None):
        """n_steps steps of every world (cb_field_step_host per group). states: one dict per
        world; controls: None (every availability 1) or one dict per world with optional
        membrane [N], junction [E] and pump [N] availabilities. Returns (states, status [W],
        taken [W]) in the batch's order; a refused world keeps its last accepted state."""
        if len(states) != self.W or (controls is not None and len(controls) != self.W):
            raise ValueError("one state (and control) per world")
        out = [None] * self.W
        status = np.zeros(self.W, dtype=np.uint32)
        taken = np.zeros(self.W, dtype=np.int32)
        for idx, tissue in self.groups:
            st = {name: np.stack([np.asarray(states[i][name], dtype=np.float64) for i in idx])
                  for name in _lib.FIELD_STATE_FIELDS}
            if controls is None:
                ctl = tissue.pack_control()
            else:
                ctl = tissue.pack_control(*(
                    np.stack([np.broadcast_to(np.asarray(
                        controls[i].get(key, 1.0), dtype=np.float64), (size,)) for i in idx])
                    for key, size in (("membrane", tissue.N), ("junction", tissue.E),
                                      ("pump", tissue.N))))
            new, s, t = tissue.step_host(st, ctl, dt, n_steps)
            for k, i in enumerate(idx):
                out[i] = {name: a[k].copy() for name, a in new.items()}
                status[i], taken[i] = s[k], t[k]
        return out, status, taken
