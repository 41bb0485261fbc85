"""Seeded synthetic tissues embedded in a resolved extracellular grid (the spatial-field worlds).

A *field world* is one pump-leak tissue whose cells face finite extracellular nodes instead of
one held bath: a side-by-side square grid of outside nodes (``side`` per side, spacing 10 um),
joined by 4-neighbour faces that carry logarithmic-mean electrodiffusion
(``cells.route.logmean_electrodiffusion@1``); the ring of boundary nodes is held (reservoirs at
the bath's concentrations and 0 V). Cells sit on a square lattice of interior nodes (``stride``
nodes apart, so no two cells share a node and no cell faces the ring), each with one membrane
patch to its node, and 4-neighbour gap junctions between lattice neighbours. Each cell and its
node form one capacitor component; every other interior node is a component of its own. All
are floating (no gauge): Kirchhoff current balance over faces and junctions fixes their
offsets, as the reference's field closure does (numerics/surface_field.py:1-7, :253-361).

The cells' laws are the pump-leak tissue's (worlds.py); the field's declared values, which the
benchmark does not give, are named below. Every world of a batch shares its topology (grid,
lattice and junction graph); parameters are drawn per world. The face conductivity multiplier
is log-normal (sigma 0.5), one per face.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import worlds as W

SPACING_M = 1e-5  # 10 um grid spacing
VOLUME_FRACTION = 0.2  # Not given by the benchmark: declared here.
NODE_VOLUME_PL = VOLUME_FRACTION * SPACING_M**3 * 1e15  # 0.2 pL per node
FACE_AREA_M2 = VOLUME_FRACTION * SPACING_M**2
# Free diffusivities of Na, K, Cl (m^2/s) over a tortuosity of 1.6 (declared here).
DIFFUSIVITY_M2_S = np.array([1.33e-9, 1.96e-9, 2.03e-9]) / 1.6**2
FACE_SIGMA = 0.5


@dataclass
class FieldWorld:
    """One tissue in its extracellular grid, host arrays, world-local indices."""

    side: int
    cells_side: int
    stride: int
    cell_node: np.ndarray  # [N] outside node of each cell's membrane
    volume: np.ndarray  # [N] pL
    area: np.ndarray  # [N] m^2
    capacitance: np.ndarray  # [N] F
    permeability: np.ndarray  # [S, N] m/s
    pump_capacity: np.ndarray  # [N]
    amount: np.ndarray  # [S, N] fmol
    fixed_charge_fmol: np.ndarray  # [N]
    initial_charge: np.ndarray  # [N] C
    sender: np.ndarray  # [E]
    receiver: np.ndarray  # [E]
    junction_area: np.ndarray  # [E]
    junction_permeability: np.ndarray  # [S, E]
    gate_threshold: np.ndarray  # [E]
    gate_minimum: np.ndarray  # [E]
    gate_initial: np.ndarray  # [E]
    outside_volume: np.ndarray  # [O] pL
    outside_amount: np.ndarray  # [S, O] fmol
    outside_fixed_fmol: np.ndarray  # [O]
    outside_charge: np.ndarray  # [O] C
    reservoir: np.ndarray  # [O] bool (the held ring)
    boundary_V: np.ndarray  # [O]
    face_sender: np.ndarray  # [F] outside node
    face_receiver: np.ndarray  # [F]
    face_diffusivity: np.ndarray  # [S, F] m^2/s (free x tortuosity x the face's multiplier)
    face_area: float = FACE_AREA_M2
    face_length: float = SPACING_M
    temperature: float = W.TEMPERATURE_K
    pump: tuple = (W.PUMP_ATP, W.PUMP_ADP, W.PUMP_PI, W.PUMP_KM_NA, W.PUMP_KM_K, W.PUMP_KM_ATP,
                   W.PUMP_DG0)
    position: np.ndarray = field(default_factory=lambda: np.zeros((2, 0)))

    @property
    def cells(self):
        return self.volume.size

    @property
    def edges(self):
        return self.sender.size

    @property
    def nodes(self):
        return self.outside_volume.size

    @property
    def faces(self):
        return self.face_sender.size

    @property
    def face_factor(self):
        """D A / L per species and face (m^3/s), as the reference forms it from the definition
        (models/surface_tissue.py:191)."""
        return self.face_diffusivity * self.face_area / self.face_length


def grid_faces(side):
    """4-neighbour faces of a side-by-side node grid, row-major nodes, each pair once."""
    return W.grid_edges(side, side)


def lattice(side, cells_side, stride):
    """The interior nodes the cells face: a cells_side-square lattice, stride nodes apart,
    centred in the grid and clear of the ring."""
    span = stride * (cells_side - 1)
    first = (side - 1 - span) // 2
    if first < 1 or first + span > side - 2 or stride < 2:
        raise ValueError("the cell lattice must sit inside the held ring with stride >= 2")
    at = first + stride * np.arange(cells_side)
    return (at[None, :] + side * at[:, None]).reshape(-1)


def anchored_background(amount, anchor):
    """The fixed background (charge-equivalent fmol) of nodes whose charge anchor is ``anchor``
    (C), by the reference's anchor rule: fl(fl(anchor / CHARGE_PER_FMOL) - fsum(z n))
    (models/surface_tissue.py:447-474)."""
    return np.array([
        anchor[i] / W.CHARGE_PER_FMOL - math.fsum(z * a for z, a in zip(W.VALENCE, amount[:, i],
                                                                         strict=True))
        for i in range(amount.shape[1])])  # fmt: skip


def field_world(side, cells_side, stride, rng, *, gate=None, junction_sigma=0.0):
    """One field world: a side x side grid, a cells_side x cells_side tissue."""
    n = cells_side * cells_side
    o = side * side
    cell_node = lattice(side, cells_side, stride)
    volume, area, capacitance, permeability, amount, fixed = W._cells(rng, n)
    sender, receiver = W.grid_edges(cells_side, cells_side)
    t = W._assemble(volume, area, capacitance, permeability, amount, fixed, sender, receiver, rng,
                    junction_sigma=junction_sigma, gate=gate)
    ix, iy = np.arange(o) % side, np.arange(o) // side
    ring = (ix == 0) | (iy == 0) | (ix == side - 1) | (iy == side - 1)
    out_volume = np.full(o, NODE_VOLUME_PL)
    out_amount = W.BATH_mM[:, None] * out_volume[None, :]
    # Every charge anchor is exactly zero, so each capacitor component (a cell and its node, or
    # a lone node) is neutral to the bit, as the field's bind requires.
    out_fixed = anchored_background(out_amount, np.zeros(o))
    cell_fixed = anchored_background(t.amount, np.zeros(n))
    fs, fr = grid_faces(side)
    multiplier = np.exp(FACE_SIGMA * rng.standard_normal(fs.size))
    diffusivity = DIFFUSIVITY_M2_S[:, None] * multiplier[None, :]
    cx, cy = cell_node % side, cell_node // side
    return FieldWorld(
        side=side, cells_side=cells_side, stride=stride, cell_node=cell_node,
        volume=t.volume, area=t.area, capacitance=t.capacitance, permeability=t.permeability,
        pump_capacity=t.pump_capacity, amount=t.amount, fixed_charge_fmol=cell_fixed,
        initial_charge=np.zeros(n), sender=t.sender, receiver=t.receiver,
        junction_area=t.junction_area, junction_permeability=t.junction_permeability,
        gate_threshold=t.gate_threshold, gate_minimum=t.gate_minimum,
        gate_initial=t.gate_initial, outside_volume=out_volume, outside_amount=out_amount,
        outside_fixed_fmol=out_fixed, outside_charge=np.zeros(o),
        reservoir=ring, boundary_V=np.zeros(o), face_sender=fs, face_receiver=fr,
        face_diffusivity=diffusivity,
        position=np.stack(((cx + 0.5) / side, (cy + 0.5) / side)),
    )  # fmt: skip


def field_tissues(worlds, side=128, cells_side=32, stride=3, seed=7):
    """The spatial-field benchmark's worlds: each 1024 cells in a 128 x 128 grid."""
    return [field_world(side, cells_side, stride, W.world_rng(seed, w)) for w in range(worlds)]


def reference_definition(world, *, dt, steps, solver="cells.solver.imex_ars222_face_electromigration@1",
                         field_solver="cells.solver.capacitive_reduction_gauged_damped_newton@2",
                         membrane_control=None, junction_control=None, pump_control=None):
    """One FieldWorld as a reference definition dict (schema_version 1, model @1)."""
    n, e, o, nf = world.cells, world.edges, world.nodes, world.faces
    mc = np.ones(n) if membrane_control is None else np.broadcast_to(membrane_control, (n,))
    jc = np.ones(e) if junction_control is None else np.broadcast_to(junction_control, (e,))
    pc = np.ones(n) if pump_control is None else np.broadcast_to(pump_control, (n,))
    atp, adp, pi, km_na, km_k, km_atp, dg0 = world.pump
    sp = W.SPECIES
    cells = [{
        "id": f"cell_{i}",
        "volume_pL": float(world.volume[i]),
        "initial_amount_fmol": {s: float(world.amount[k, i]) for k, s in enumerate(sp)},
        "fixed_charge_equivalent_fmol": float(world.fixed_charge_fmol[i]),
        "initial_charge_C": float(world.initial_charge[i]),
    } for i in range(n)]
    outside = [{
        "id": f"outside_{j}",
        "volume_pL": float(world.outside_volume[j]),
        "initial_amount_fmol": {s: float(world.outside_amount[k, j]) for k, s in enumerate(sp)},
        "fixed_charge_equivalent_fmol": float(world.outside_fixed_fmol[j]),
        "initial_charge_C": float(world.outside_charge[j]),
        "reservoir": bool(world.reservoir[j]),
        "boundary_potential_V": float(world.boundary_V[j]),
    } for j in range(o)]
    membranes = [{
        "id": f"membrane_{i}",
        "inside": f"cell_{i}",
        "outside": f"outside_{int(world.cell_node[i])}",
        "area_m2": float(world.area[i]),
        "capacitance_F": float(world.capacitance[i]),
        "permeability_m_per_s": {s: float(world.permeability[k, i]) for k, s in enumerate(sp)},
        "law": "cells.route.constant_field@1",
        "pump": {
            "id": f"pump_{i}",
            "law": "cells.cycle.nak_atp_mass_action_positive@1",
            "roles": {"sodium": "Na", "potassium": "K"},
            "stoichiometry": {"Na": -3, "K": 2},
            "capacity_fmol_per_s": float(world.pump_capacity[i]),
            "km_na_mM": km_na, "km_k_mM": km_k, "km_atp_mM": km_atp,
            "metabolism": {
                "kind": "cells.fuel_kind.maintained_chemical_reservoirs@1",
                "atp_mM": atp, "adp_mM": adp, "pi_mM": pi, "delta_g0_J_per_mol": dg0,
            },
        },
    } for i in range(n)]  # fmt: skip
    junctions = [{
        "id": f"junction_{k}",
        "sender": f"cell_{int(world.sender[k])}",
        "receiver": f"cell_{int(world.receiver[k])}",
        "area_m2": float(world.junction_area[k]),
        "permeability_m_per_s": {
            s: float(world.junction_permeability[j, k]) for j, s in enumerate(sp)},
        "law": "cells.route.constant_field@1",
        "gate": {
            "law": "cells.junction.junction_voltage_relaxation@1",
            "threshold_voltage_V": float(world.gate_threshold[k]),
            "minimum_open_fraction": float(world.gate_minimum[k]),
            "initial_gate": float(world.gate_initial[k]),
        },
    } for k in range(e)]  # fmt: skip
    faces = [{
        "id": f"face_{f}",
        "sender": f"outside_{int(world.face_sender[f])}",
        "receiver": f"outside_{int(world.face_receiver[f])}",
        "area_m2": float(world.face_area),
        "length_m": float(world.face_length),
        "diffusivity_m2_per_s": {s: float(world.face_diffusivity[k, f]) for k, s in enumerate(sp)},
        "law": "cells.route.logmean_electrodiffusion@1",
    } for f in range(nf)]  # fmt: skip
    end = float(dt * steps)

    def schedule(key, prefix, values):
        return [{key: f"{prefix}_{i}", "schedule": [{"time": 0.0, "availability": float(v)}]}
                for i, v in enumerate(values)]

    return {
        "schema_version": 1,
        "model": {
            "id": "cells.model.resolved_pump_tissue@1",
            "temperature_K": float(world.temperature),
            "species": [{"id": s, "valence": int(z)} for s, z in zip(sp, W.VALENCE, strict=True)],
            "cells": cells,
            "extracellular": outside,
            "membranes": membranes,
            "junctions": junctions,
            "faces": faces,
            "closure": {
                "law": "cells.field_closure.resolved_capacitor_components_current_continuity@1",
                "gauge_reference": None,
            },
        },
        "experiment": {
            "end_time": end,
            "observation_times": [0.0, end],
            "membrane_controls": schedule("membrane_id", "membrane", mc),
            "junction_controls": schedule("junction_id", "junction", jc),
            "pump_controls": schedule("pump_id", "pump", pc),
        },
        "execution": {
            "dt": float(dt),
            "capacity": n,
            "extracellular_capacity": o,
            "membrane_capacity": n,
            "edge_capacity": e,
            "face_capacity": nf,
            "backend": "cpu",
            "jit": True,
            "precision": "float64",
            "solver": solver,
            "field_solver": field_solver,
            "max_steps": int(steps),
            "max_trace_bytes": 536870912,
            "material_balance_atol_fmol": {s: 2e-11 for s in sp},
        },
    }
