"""Drop-in for the reference's checked step on its own pytrees.

The reference resolves a model module whose hot entry is
``checked_step(state, dt, control, p, active) -> (state, valid)``
(src/cells/models/surface_pump.py:365-369, src/cells/models/surface_pump_v3.py:3989) on
NamedTuple pytrees: ``state`` of STATE_TYPE (src/cells/models/surface_kinetic.py:36-44 with
src/cells/models/surface_tissue.py:31-45), ``p`` the bound layout, ``control`` a
SurfaceKineticControl (src/cells/execution/schedule.py:18-22), all padded to capacities with
``*_active`` masks. ``DeviceStep(p)`` binds such a layout once (host analysis, upload) and is
then called with the reference's own arguments; it returns a new state of the same type (inputs
are never mutated) and ``valid``, the unchanged state when the step is refused, like the
reference (surface_pump.py:362).

Scope: the held-bath pump-leak tissue — every active cell has exactly one active membrane
patch, every patch faces its world's held bath (a reservoir outside node), no faces, species
Na/K/Cl (+1/+1/-1), the Na/K-ATPase with one set of pump constants per world, and either no
channel population or two per cell (Kv1.5 and/or NaV1.2 of @3's catalogue, one permeant species
each). Other worlds raise ``Unsupported`` at bind; nothing falls back to the CPU.
"""

from __future__ import annotations

import numpy as np

from . import worlds
from .tissue import Tissue

ARS222_ID = "cells.solver.imex_ars222_face_electromigration@1"
N2_ID = "cells.solver.imex_ars222_implicit_conductances@1"
PUMP_FIELDS = ("atp_mM", "adp_mM", "pi_mM", "km_na_mM", "km_k_mM", "km_atp_mM",
               "delta_g0_J_mol")


class Unsupported(ValueError):
    """The layout is outside the device step's scope (module docstring)."""


def _a(p, name):
    return np.asarray(getattr(p, name))


def _active(p, name, size):
    if hasattr(p, name):
        return _a(p, name).astype(bool)
    return np.ones(size, dtype=bool)


class Mapping:
    """Active-entity indices of one reference layout, in the reference's slot order."""

    def __init__(self, p):
        cell_active = _a(p, "active").astype(bool) if hasattr(p, "active") else _a(
            p, "cell_active").astype(bool)
        self.cells = np.flatnonzero(cell_active)
        membrane_active = _active(p, "membrane_active", _a(p, "membrane_cell").size)
        self.membranes = np.flatnonzero(membrane_active)
        junction_active = _active(p, "junction_active", _a(p, "junction_sender").size)
        self.junctions = np.flatnonzero(junction_active)
        reservoir = _a(p, "reservoir").astype(bool)
        outside_active = _active(p, "outside_active", reservoir.size)
        self.baths = np.flatnonzero(reservoir & outside_active)
        # One patch per cell, in cell order.
        owner = _a(p, "membrane_cell")[self.membranes]
        if sorted(owner.tolist()) != self.cells.tolist():
            raise Unsupported("every active cell needs exactly one active membrane patch")
        self.patch_of_cell = self.membranes[np.argsort(owner, kind="stable")]
        outside = _a(p, "membrane_outside")[self.patch_of_cell]
        if self.baths.size != 1 or np.any(outside != self.baths[0]):
            raise Unsupported("every patch must face the world's one held bath")
        if np.any(outside_active & ~reservoir):
            raise Unsupported("finite (unheld) outside nodes need the field solve")
        if hasattr(p, "face_active") and np.any(_a(p, "face_active")):
            raise Unsupported("extracellular faces need the field solve")
        self.bath = int(self.baths[0])
        # Channel populations: the same number per active cell (0 or 2), each with one permeant
        # species; slot q of a cell is its q-th population in the reference's channel order.
        self.nch = 0
        self.channel_index = np.zeros((0, self.cells.size), dtype=np.int64)
        self.channel_species = np.zeros((0, self.cells.size), dtype=np.int64)
        if hasattr(p, "channel_active") and np.any(_a(p, "channel_active")):
            if not all(hasattr(p, f) for f in ("channel_membranes", "channel_laws",
                                               "channel_relative_permeability")):
                raise Unsupported("channel populations need @3's catalogue layout")
            active = np.flatnonzero(_a(p, "channel_active").astype(bool))
            patch = _a(p, "channel_membranes")[active]
            cell_of_patch = _a(p, "membrane_cell")
            owner = cell_of_patch[patch]
            counts = np.bincount(owner, minlength=cell_active.size)[self.cells]
            if np.any(counts != counts[0]) or counts[0] not in (0, 2):
                raise Unsupported("every cell needs the same number (0 or 2) of channel "
                                  "populations")
            self.nch = int(counts[0])
            index = np.zeros((self.nch, self.cells.size), dtype=np.int64)
            slot = np.zeros(cell_active.size, dtype=np.int64)
            local = {int(c): k for k, c in enumerate(self.cells)}
            for j, c in zip(active, owner, strict=True):
                index[slot[c], local[int(c)]] = j
                slot[c] += 1
            self.channel_index = index
        local = -np.ones(cell_active.size, dtype=np.int64)
        local[self.cells] = np.arange(self.cells.size)
        self.sender = local[_a(p, "junction_sender")[self.junctions]]
        self.receiver = local[_a(p, "junction_receiver")[self.junctions]]


def block_from_layout(p, j):
    """The layout's open-channel block (surface_pump_v3.block_initial_values' fields
    channel_block_weight, _k0_mM, _steepness [M, channel] and _concentration_mM [channel]) at the
    populations j [NCH, C], as a worlds.ChannelBlock. The signed steepness is carried as a
    unit-valence blocker on the side of its sign, whose m_k is |steepness|, so the block's
    steepness equals the layout's exactly."""
    steep = _a(p, "channel_block_steepness")[:, j].astype(float)
    weight = _a(p, "channel_block_weight")[:, j].astype(float)
    conc = _a(p, "channel_block_concentration_mM")[j].astype(float)
    modes = weight.shape[0]
    neutral = np.zeros_like(weight)
    neutral[0] = 1.0
    declared = (conc != 0) | np.any(weight != neutral, axis=0)
    side = np.where(np.all(steep >= 0, axis=0), 1, -1)
    if np.any((steep != 0) & (np.sign(steep) != side)):
        raise Unsupported("one population's modes must share their steepness sign")
    return worlds.ChannelBlock(
        declared=declared, weight=weight,
        k0_mM=_a(p, "channel_block_k0_mM")[:, j].astype(float),
        distance=np.abs(steep), modes_declared=np.full(conc.shape, modes),
        valence=np.ones(conc.shape, dtype=np.int64), side=side.astype(np.int64),
        concentration_mM=conc)


# @3 options the device step does not carry, by a layout field each adds where it is declared
# (models/surface_pump_v3.py: FORMS_LAYOUT_FIELDS :179, SHIFT_LAYOUT_FIELDS :210,
# LOOP_LAYOUT_FIELDS :230, ONE_WAY_LAYOUT_FIELDS :287; series junction gates' parameters :6306).
OPTION_FIELDS = {
    "channel_shift_row": "voltage-shifted channel readers (FR-64)",
    "forms_face_active": "forms faces",
    "loop_flux_row": "routed loops",
    "one_way_entity": "one-way flux records",
    "junction_series_parameters": "series junction gates",
}


def refuse_options(p):
    """Raise Unsupported for a layout that declares an option outside the device step: one of
    OPTION_FIELDS, or a present Ca pump (@2's calcium_pump_present, models/surface_pump_v2.py:51)."""
    for name, what in OPTION_FIELDS.items():
        if hasattr(p, name):
            raise Unsupported(f"{what} are not in the device step")
    if hasattr(p, "calcium_pump_present") and np.any(_a(p, "calcium_pump_present")):
        raise Unsupported("Ca pumps are not in the device step")


def world_from_layout(p):
    """One reference layout -> (worlds.World, Mapping)."""
    refuse_options(p)
    m = Mapping(p)
    valence = _a(p, "valence").reshape(-1)
    if not np.array_equal(valence, worlds.VALENCE):
        raise Unsupported("species must be Na, K, Cl with valences +1, +1, -1")
    patch = m.patch_of_cell
    nch = m.nch
    channel = {}
    if nch:
        j = m.channel_index
        laws = _a(p, "channel_laws")[j]
        if np.any(~np.isin(laws, (0, 2))):
            raise Unsupported("channel laws must be Kv1.5 (0) or NaV1.2 (2)")
        rel = _a(p, "channel_relative_permeability")[:, j]  # [S, NCH, C]
        if np.any(np.count_nonzero(rel, axis=0) != 1):
            raise Unsupported("each channel population needs exactly one permeant species")
        species = np.argmax(rel != 0, axis=0)
        m.channel_species = species
        channel = dict(
            channel_code=laws.astype(np.int32),
            channel_species=species.astype(np.int32),
            channel_permeability=(_a(p, "channel_permeability")[j]
                                  * np.take_along_axis(rel, species[None], 0)[0]),
            channel_abundance=_a(p, "channel_abundance")[j].astype(float),
            channel_gate_initial=np.zeros((2, nch, m.cells.size)),
        )
        if hasattr(p, "channel_block_weight"):
            channel["channel_block"] = block_from_layout(p, j)
    if hasattr(p, "pump_present"):
        present = _a(p, "pump_present")[patch].astype(bool)
        stoich = _a(p, "stoichiometry")[:, patch]
        if np.any(stoich[:, present] != worlds.STOICHIOMETRY[:, None]):
            raise Unsupported("pumps must move 3 Na out and 2 K in per cycle")
        if np.any(_a(p, "pump_sodium_species")[patch][present] != worlds.SODIUM) or np.any(
                _a(p, "pump_potassium_species")[patch][present] != worlds.POTASSIUM):
            raise Unsupported("pump roles must be Na (sodium) and K (potassium)")
        capacity = np.where(present, _a(p, "pump_capacity")[patch], 0.0)
        constants = []
        for name in PUMP_FIELDS:
            v = _a(p, "pump_" + name)[patch][present]
            if v.size and np.any(v != v[0]):
                raise Unsupported(f"pump {name} must be one value per world")
            constants.append(float(v[0]) if v.size else 1.0)
    else:
        capacity = np.zeros(m.cells.size)
        constants = [1.5, 0.1, 0.1, 12.0, 0.2, 0.5, -37000.0]
    bath_volume = float(_a(p, "extracellular_volume")[m.bath])
    bath_amount = _a(p, "extracellular_amount_reference")[:, m.bath]
    n = m.cells.size
    world = worlds.World(
        volume=_a(p, "volume")[m.cells].astype(float),
        area=_a(p, "membrane_area")[patch].astype(float),
        capacitance=_a(p, "membrane_capacitance")[patch].astype(float),
        permeability=_a(p, "membrane_permeability")[:, patch].astype(float),
        pump_capacity=capacity.astype(float),
        amount=_a(p, "amount_reference")[:, m.cells].astype(float),
        fixed_charge_fmol=np.zeros(n),
        initial_charge=_a(p, "initial_cell_charge_C")[m.cells].astype(float),
        sender=m.sender,
        receiver=m.receiver,
        junction_area=_a(p, "junction_area")[m.junctions].astype(float),
        junction_permeability=_a(p, "junction_permeability")[:, m.junctions].astype(float),
        gate_threshold=_a(p, "junction_threshold_voltage")[m.junctions].astype(float),
        gate_minimum=_a(p, "junction_minimum")[m.junctions].astype(float),
        gate_initial=np.ones(m.junctions.size),
        temperature=float(_a(p, "temperature")),
        bath_mM=bath_amount / bath_volume,
        bath_volume=bath_volume,
        bath_potential=float(_a(p, "boundary_V")[m.bath]),
        pump=tuple(constants),
        **channel,
    )
    return world, m


# Reference state fields <-> packed fields (one world; the bath at mapping.bath).
_CELL_MAP = (
    ("amount_increment", "amount_increment", "cell"),
    ("membrane_transferred", "membrane_transferred", "patch"),
    ("membrane_dissipated_energy_pJ", "membrane_dissipated", "patch"),
    ("pump_cycles", "pump_cycles", "patch"),
    ("pump_dissipated_energy_pJ", "pump_dissipated", "patch"),
    ("metabolic_work_pJ", "metabolic_work", "patch"),
)
_EDGE_MAP = (
    ("junction_transferred", "junction_transferred"),
    ("junction_dissipated_energy_pJ", "junction_dissipated"),
    ("junction_gate", "junction_gate"),
)
_BATH_MAP = (
    ("reservoir_supplied", "reservoir_supplied"),
    ("electrode_charge_transferred_C", "electrode_charge"),
    ("reservoir_work_pJ", "reservoir_work"),
    ("electrode_work_pJ", "electrode_work"),
)
_ZERO_FIELDS = ("extracellular_amount_increment", "face_transferred",
                "face_dissipated_energy_pJ")


def packed_state(state, m):
    """Reference state (one world) -> packed dict of the device layout."""
    out = {}
    for ref, name, kind in _CELL_MAP:
        v = np.asarray(getattr(state, ref))
        idx = m.cells if kind == "cell" else m.patch_of_cell
        out[name] = v[..., idx].astype(float)
    for ref, name in _EDGE_MAP:
        out[name] = np.asarray(getattr(state, ref))[..., m.junctions].astype(float)
    for ref, name in _BATH_MAP:
        out[name] = np.asarray(getattr(state, ref))[..., m.bath:m.bath + 1].astype(float)
    j, sp = m.channel_index, m.channel_species
    if m.nch:
        out["channel_gate"] = np.asarray(state.channel_gate)[:, j].astype(float)
        out["channel_transferred"] = np.asarray(state.channel_transferred)[sp, j].astype(float)
        out["channel_dissipated"] = np.asarray(
            state.channel_dissipated_energy_pJ)[sp, j].astype(float)
    else:
        c = m.cells.size
        out["channel_gate"] = np.zeros((2, 0, c))
        out["channel_transferred"] = np.zeros((0, c))
        out["channel_dissipated"] = np.zeros((0, c))
    return out


def reference_state(packed, like, m):
    """Packed dict -> a new reference state of like's type (like's padding kept)."""
    fields = {k: np.array(v, copy=True) for k, v in like._asdict().items()}
    for ref, name, kind in _CELL_MAP:
        idx = m.cells if kind == "cell" else m.patch_of_cell
        fields[ref][..., idx] = packed[name]
    for ref, name in _EDGE_MAP:
        fields[ref][..., m.junctions] = packed[name]
    for ref, name in _BATH_MAP:
        fields[ref][..., m.bath:m.bath + 1] = packed[name]
    if m.nch:
        j, sp = m.channel_index, m.channel_species
        fields["channel_gate"][:, j] = packed["channel_gate"]
        fields["channel_transferred"][sp, j] = packed["channel_transferred"]
        fields["channel_dissipated_energy_pJ"][sp, j] = packed["channel_dissipated"]
    return type(like)(**fields)


def layout_solver(p):
    """The IMEX method a bound layout declares: N2 (imex_ars222_implicit_conductances@1) when its
    operator time is a vector (one entry per frozen block, the reference's own static switch,
    numerics/surface_imex.py:94-107), else the plain ARS(2,2,2)."""
    time = getattr(p, "imex_operator_time", None)
    return N2_ID if time is not None and np.shape(time) == (2,) else ARS222_ID


class DeviceStep:
    """checked_step(state, dt, control, p, active) of the held-bath pump tissue on the device.

    Bind once per layout: ``step = DeviceStep(p)``; then ``state, valid = step(state, dt,
    control, p, active)`` as the reference's checked_step. ``solver`` is the layout's IMEX
    method (by default the one the layout declares, layout_solver): ARS(2,2,2)
    (imex_ars222_face_electromigration@1, CB_METHOD_ARS222) or N2
    (imex_ars222_implicit_conductances@1, CB_METHOD_N2)."""

    def __init__(self, p, device=0, solver=None):
        from . import _lib

        solver = layout_solver(p) if solver is None else solver
        if solver not in (ARS222_ID, N2_ID):
            raise Unsupported(f"solver {solver} is not in the device step")
        if hasattr(p, "imex_explicit") and np.asarray(p.imex_explicit).shape[0] != 3:
            raise Unsupported("the layout's tableau is not ARS(2,2,2)")
        self.method = _lib.METHOD_N2 if solver == N2_ID else _lib.METHOD_ARS222
        world, self.mapping = world_from_layout(p)
        self.batch = worlds.pack([world])
        self.tissue = Tissue(self.batch, device=device)

    def __call__(self, state, dt, control, p=None, active=None):
        for name in _ZERO_FIELDS:
            if hasattr(state, name) and np.any(np.asarray(getattr(state, name)) != 0):
                raise Unsupported(f"{name} must stay zero in a held-bath tissue")
        m = self.mapping
        if m.nch:
            moved = np.array(state.channel_transferred, copy=True)
            moved[m.channel_species, m.channel_index] = 0.0
            if np.any(moved != 0):
                raise Unsupported("channel transfer of a non-permeant species must stay zero")
        packed = packed_state(state, m)
        ctl = self.tissue.pack_control(
            membrane=np.asarray(control.membrane)[m.patch_of_cell],
            junction=np.asarray(control.junction)[m.junctions],
            pump=np.asarray(control.pump)[m.patch_of_cell],
            channel=(np.asarray(control.channel)[m.channel_index] if m.nch else 1.0),
        )
        out, status, _ = self.tissue.step_host(self.tissue.pack_state(packed), ctl, float(dt), 1,
                                               method=self.method)
        valid = bool(status[0] == 0)
        new = reference_state(self.tissue.unpack_state(out), state, m)
        return new, np.asarray(valid)

    def close(self):
        self.tissue.close()
