"""Generate the golden fixtures under tests/golden/ by running the REFERENCE's own step.

Run in a container that holds the reference source tree (its project root, the directory with
``src/cells``), by hand and never from the test suite (the committed fixtures are what the
tests read; machines without the reference sources only read them):

    python tests/golden/make_golden.py --reference <reference project root>
    CELLS_REFERENCE=<reference project root> python tests/golden/make_golden.py

The reference is a JAX program; jax is absent here, so ``jax_shim/`` (a NumPy stand-in for the
few jax names it touches) goes first on sys.path and the reference's step runs on its own
``xp=np`` branch (models/surface_pump.py:259-362 imex_step, models/surface_pump_v3.py:3547
imex_step, numerics/fixed_step.py:25 rk4_checked_step). Each fixture stores the world (the packed
arrays of cells_b200.worlds) and the reference's state at chosen steps, converted to the packed
layout of oracle/tissue.py (membrane i is cell i's patch; the world has one held bath).

Fixtures:
  ars222_grid4x4.npz     The single 4x4 CPU world (seed 0), ARS(2,2,2), dt 1 ms, 10,000 steps,
                         @1; snapshots at a few early steps and every 500 steps.
  ars222_v3_grid4x4.npz  The same world through @3's imex_step for 200 steps (the live model).
  ars222_gated.npz       A 3x3 world with voltage-gated junctions (minimum 0.1), partial controls
                         and a bath at -4 mV, 400 steps at 1 ms (@1).
  pytrees_gated_padded.npz  The gated world with every capacity 3 above its count: the
                         reference's own layout fields, controls and padded states (60 steps),
                         for the drop-in checked step (cells_b200/model.py).
  rk4_grid4x4.npz        The 4x4 world by RK4 at dt 0.1 ms, 100 steps (@1).
  ars222_v3_channels.npz The 4x4 world (seed 3) with a NaV1.2 (m^3 h) and a Kv1.5 (m h)
                         population per cell, partial channel availabilities, @3, 300 steps.
  ars222_v3_block.npz    A 4x4 world with both populations; 12 of its Na populations blocked by
                         an outside divalent blocker in two modes; @3, 300 steps.
  ars222_v3_block_delaunay.npz  A gated 40-cell Delaunay world with both populations: half the
                         Na populations blocked (outside, two modes), 80% of the K populations
                         (inside, three modes); partial controls; 200 steps.
  pytrees_v3_block_padded.npz  That world's @3 pytrees, capacities 2 above the counts.
  ars222_v3_channels_delaunay.npz  A 40-cell Delaunay world with both populations, gated
                         junctions, partial controls, a -4 mV bath, @3, 200 steps.
  pytrees_v3_channels_padded.npz  That world's @3 pytrees with every capacity 2 above its count
                         (layout, controls, padded states over 40 steps), for the drop-in step.
  n2_grid4x4.npz         The 4x4 world under N2 (@3, implicit slope conductances), 300 steps.
  n2_channels_delaunay.npz  A 40-cell Delaunay world with NaV1.2 and Kv1.5 populations, gated
                         junctions, partial controls, a -4 mV bath, under N2, 200 steps.
  pytrees_n2_padded.npz  That world's @3 pytrees under N2 (capacities 2 above the counts, 40
                         steps), for the drop-in step.
  vector_window.npz      The reference's own vector window (execution/vector_windows.py:348-410)
                         over @3 on three gated 4x4 worlds with per-world step sizes, held
                         controls, observation slots, counts and first steps, one world refused
                         (vmap and scan of the jax stand-in loop over worlds and rows).
  device_checks.npz      The reference's accepted-row device checks (@3) on rows of its own
                         trajectory of a 36-cell gated Delaunay world with channels: accepted
                         rows after 1-120 steps and two planted faults (failed bits, values).
  field_grid10.npz       A 10x10 extracellular grid (held ring) with a 3x3 tissue, @1 ARS(2,2,2)
                         with face electromigration and the factored field, 400 steps at 0.5 ms.
  field_gated14.npz      A 14x14 grid with a 4x4 gated tissue (log-normal junctions), partial
                         controls, 200 steps.
  field_grid24.npz       A 24x24 grid with a 6x6 tissue, 60 steps.
  laws.npz               Point laws on grids of inputs: bernoulli, the pump kinetics and the
                         junction gate rate.
"""

from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _setup(reference):
    sys.path.insert(0, os.path.join(HERE, "jax_shim"))
    sys.path.insert(0, os.path.join(reference, "src"))
    sys.path.insert(0, reference)
    sys.path.insert(0, REPO)


def _state_to_packed(state):
    """Reference STATE_TYPE (one world, held bath at outside slot 0) -> packed dict."""
    return dict(
        amount_increment=np.asarray(state.amount_increment),
        membrane_transferred=np.asarray(state.membrane_transferred),
        membrane_dissipated=np.asarray(state.membrane_dissipated_energy_pJ),
        pump_cycles=np.asarray(state.pump_cycles),
        pump_dissipated=np.asarray(state.pump_dissipated_energy_pJ),
        metabolic_work=np.asarray(state.metabolic_work_pJ),
        junction_transferred=np.asarray(state.junction_transferred),
        junction_dissipated=np.asarray(state.junction_dissipated_energy_pJ),
        junction_gate=np.asarray(state.junction_gate),
        reservoir_supplied=np.asarray(state.reservoir_supplied)[:, :1],
        electrode_charge=np.asarray(state.electrode_charge_transferred_C)[:1],
        reservoir_work=np.asarray(state.reservoir_work_pJ)[:1],
        electrode_work=np.asarray(state.electrode_work_pJ)[:1],
    )


def _channels_to_packed(state, world):
    """@3's channel fields [2, Ch] / [S, Ch] (channel j = cell i * NCH + slot k) -> packed
    [2, NCH, C] and [NCH, C] (the permeant species only)."""
    nch, n = world.channel_slots, world.cells
    j = np.arange(n)[None, :] * nch + np.arange(nch)[:, None]  # [NCH, C]
    species = world.channel_species
    gate = np.asarray(state.channel_gate)[:, j]
    moved = np.asarray(state.channel_transferred)[species, j]
    heat = np.asarray(state.channel_dissipated_energy_pJ)[species, j]
    return dict(channel_gate=gate, channel_transferred=moved, channel_dissipated=heat)


def _batch_arrays(batch):
    from dataclasses import fields

    out = {"batch_" + f.name: getattr(batch, f.name) for f in fields(batch)
           if f.name != "channel_block"}
    if batch.channel_block is not None:
        out.update({"block_" + f.name: getattr(batch.channel_block, f.name)
                    for f in fields(batch.channel_block)})
    return out


LAYOUT_FIELDS = (
    "active", "membrane_active", "membrane_cell", "membrane_outside", "junction_active",
    "junction_sender", "junction_receiver", "reservoir", "outside_active", "face_active",
    "channel_active", "valence", "temperature", "pump_present", "stoichiometry",
    "pump_sodium_species", "pump_potassium_species", "pump_capacity", "pump_atp_mM",
    "pump_adp_mM", "pump_pi_mM", "pump_km_na_mM", "pump_km_k_mM", "pump_km_atp_mM",
    "pump_delta_g0_J_mol", "extracellular_volume", "extracellular_amount_reference", "volume",
    "membrane_area", "membrane_capacitance", "membrane_permeability", "amount_reference",
    "initial_cell_charge_C", "junction_area", "junction_permeability",
    "junction_threshold_voltage", "junction_minimum", "boundary_V", "imex_explicit",
    "imex_operator_time",
)


CHANNEL_LAYOUT_FIELDS = (
    "channel_membranes", "channel_laws", "channel_relative_permeability",
    "channel_permeability", "channel_abundance", "channel_gate_active",
    "channel_block_weight", "channel_block_k0_mM", "channel_block_steepness",
    "channel_block_concentration_mM",
)


def _run_reference_pytrees(world, *, model_id, dt, steps, keep, padding, controls, solver=None):
    """The reference's own pytrees: layout fields, controls and full states (padded slots)."""
    from cells.definitions.specs import parse_spec
    from cells.registry.models import get_model

    from cells_b200 import worlds

    extra = {} if solver is None else {"solver": solver}
    raw = worlds.reference_definition(world, dt=dt, steps=steps, model=model_id,
                                      padding=padding, **controls, **extra)
    spec = parse_spec(raw)
    model = get_model(spec.model)
    state, p = model.initial_values(spec)
    if model_id.endswith("@3"):
        from cells.definitions.surface_pump_v3_spec import control_values
    else:
        from cells.execution.schedule import control_values

    cv = control_values(spec, [0.0])
    control = type(cv)(*(v[0] for v in cv))
    fields = LAYOUT_FIELDS + tuple(f for f in CHANNEL_LAYOUT_FIELDS if hasattr(p, f))
    out = {"layout_" + f: np.asarray(getattr(p, f)) for f in fields}
    out.update({"control_ref_" + f: np.asarray(v) for f, v in control._asdict().items()})
    snaps = []
    for k in range(0, steps + 1):
        if k:
            state, ok = model.imex_step(state, dt, control, p, xp=np)[:2]
            if not bool(ok):
                raise RuntimeError(f"reference refused step {k}")
        if k in keep:
            snaps.append({f: np.asarray(v) for f, v in state._asdict().items()})
    for f in snaps[0]:
        out["refstate_" + f] = np.stack([s_[f] for s_ in snaps])
    out["steps"] = np.asarray(sorted(keep))
    out["dt"] = np.asarray(dt)
    out["state_fields"] = np.asarray(list(snaps[0]))
    return out


def _run(world, *, model_id, dt, steps, keep, solver, controls=None, channels=False):
    from cells.definitions.specs import parse_spec
    from cells.registry.models import get_model

    from cells_b200 import worlds

    controls = controls or {}
    raw = worlds.reference_definition(world, dt=dt, steps=steps, model=model_id, solver=solver,
                                      **controls)
    spec = parse_spec(raw)
    model = get_model(spec.model)
    state, p = model.initial_values(spec)
    if model_id.endswith("@3"):
        from cells.definitions.surface_pump_v3_spec import control_values
    else:
        from cells.execution.schedule import control_values
    cv = control_values(spec, [0.0])
    control = type(cv)(*(v[0] for v in cv))
    def packed(st):
        out = _state_to_packed(st)
        if channels:
            out.update(_channels_to_packed(st, world))
        return out

    snaps, kept = [], []
    if 0 in keep:
        snaps.append(packed(state))
        kept.append(0)
    t0 = time.perf_counter()
    for k in range(1, steps + 1):
        if solver == "rk4":
            state, ok = model.checked_step(state, dt, control, p, p.active)
        else:
            out = model.imex_step(state, dt, control, p, xp=np)
            state, ok = out[0], out[1]
        if not bool(ok):
            raise RuntimeError(f"reference refused step {k}")
        if k in keep:
            snaps.append(packed(state))
            kept.append(k)
    elapsed = time.perf_counter() - t0
    stacked = {"ref_" + key: np.stack([s[key] for s in snaps]) for key in snaps[0]}
    return stacked, np.asarray(kept), elapsed


def _save(name, batch, stacked, kept, *, dt, model_id, solver, elapsed, extra=None):
    path = os.path.join(HERE, name)
    np.savez_compressed(
        path, **_batch_arrays(batch), **stacked, steps=kept, dt=np.asarray(dt),
        model_id=np.asarray(model_id), solver=np.asarray(solver),
        reference_seconds=np.asarray(elapsed), **(extra or {}),
    )  # fmt: skip
    print(f"{name}: {len(kept)} snapshots, reference {elapsed:.1f} s")


def make_trajectories():
    from cells_b200 import worlds

    ars = "cells.solver.imex_ars222_face_electromigration@1"
    world = worlds.single_grid_tissue(0)
    batch = worlds.pack([world])
    keep = {0, 1, 2, 3, 10, 100} | set(range(500, 10001, 500))
    stacked, kept, el = _run(world, model_id="cells.model.resolved_pump_tissue@1", dt=1e-3,
                             steps=10000, keep=keep, solver=ars)
    _save("ars222_grid4x4.npz", batch, stacked, kept, dt=1e-3,
          model_id="cells.model.resolved_pump_tissue@1", solver=ars, elapsed=el)

    keep = {0, 1, 2, 10, 50, 100, 200}
    stacked, kept, el = _run(world, model_id="cells.model.resolved_pump_tissue@3", dt=1e-3,
                             steps=200, keep=keep, solver=ars)
    _save("ars222_v3_grid4x4.npz", batch, stacked, kept, dt=1e-3,
          model_id="cells.model.resolved_pump_tissue@3", solver=ars, elapsed=el)

    gated = worlds.grid_world(3, 3, worlds.world_rng(7, 0), junction_sigma=0.3,
                              gate=(0.015, 0.1, 0.6))
    gated.bath_potential = -0.004
    rng = np.random.default_rng(11)
    controls = dict(
        membrane_control=rng.uniform(0.5, 1.0, gated.cells),
        junction_control=rng.uniform(0.5, 1.0, gated.edges),
        pump_control=rng.uniform(0.5, 1.0, gated.cells),
    )
    batch = worlds.pack([gated])
    keep = {0, 1, 2, 5, 50, 100, 200, 400}
    stacked, kept, el = _run(gated, model_id="cells.model.resolved_pump_tissue@1", dt=1e-3,
                             steps=400, keep=keep, solver=ars, controls=controls)
    _save("ars222_gated.npz", batch, stacked, kept, dt=1e-3,
          model_id="cells.model.resolved_pump_tissue@1", solver=ars, elapsed=el,
          extra={"control_" + k.split("_")[0]: v for k, v in controls.items()})

    # The reference's own padded pytrees (capacities 3 above the counts) for the drop-in step.
    out = _run_reference_pytrees(gated, model_id="cells.model.resolved_pump_tissue@1", dt=1e-3,
                                 steps=60, keep={0, 1, 2, 30, 60}, padding=3, controls=controls)
    np.savez_compressed(os.path.join(HERE, "pytrees_gated_padded.npz"), **out)
    print("pytrees_gated_padded.npz written")

    keep = {0, 1, 2, 10, 50, 100}
    stacked, kept, el = _run(world, model_id="cells.model.resolved_pump_tissue@1", dt=1e-4,
                             steps=100, keep=keep, solver="rk4")
    _save("rk4_grid4x4.npz", worlds.pack([world]), stacked, kept, dt=1e-4,
          model_id="cells.model.resolved_pump_tissue@1", solver="rk4", elapsed=el)


def make_channel_trajectories():
    """@3 (the live model) with voltage-gated Na (NaV1.2 m^3 h) and K (Kv1.5 m h) populations."""
    from cells_b200 import worlds

    ars = "cells.solver.imex_ars222_face_electromigration@1"
    v3 = "cells.model.resolved_pump_tissue@3"
    rng = np.random.default_rng(21)
    world = worlds.with_channels(worlds.grid_world(4, 4, worlds.world_rng(3, 0)), rng,
                                 na=("nav", 2e-10, 0.5), k=("kv", 3e-10, 0.5), sigma=0.3)
    controls = dict(channel_control=rng.uniform(0.5, 1.0, (2, world.cells)))
    keep = {0, 1, 2, 5, 50, 100, 200, 300}
    stacked, kept, el = _run(world, model_id=v3, dt=1e-3, steps=300, keep=keep, solver=ars,
                             controls=controls, channels=True)
    _save("ars222_v3_channels.npz", worlds.pack([world]), stacked, kept, dt=1e-3,
          model_id=v3, solver=ars, elapsed=el, extra={"control_channel": controls[
              "channel_control"]})

    dworld = worlds.with_channels(
        worlds.delaunay_world(40, worlds.world_rng(4, 0), junction_sigma=0.3,
                              gate=(0.02, 0.1, 0.8)), rng,
        na=("nav", 4e-10, 0.4), k=("kv", 5e-10, 0.6), sigma=0.3)
    dworld.bath_potential = -0.004
    controls = dict(
        membrane_control=rng.uniform(0.5, 1.0, dworld.cells),
        junction_control=rng.uniform(0.5, 1.0, dworld.edges),
        pump_control=rng.uniform(0.5, 1.0, dworld.cells),
        channel_control=rng.uniform(0.3, 1.0, (2, dworld.cells)),
    )
    # @3's own padded channel pytrees for the drop-in step.
    out = _run_reference_pytrees(dworld, model_id=v3, dt=1e-3, steps=40, keep={0, 1, 20, 40},
                                 padding=2, controls=controls)
    np.savez_compressed(os.path.join(HERE, "pytrees_v3_channels_padded.npz"), **out)
    print("pytrees_v3_channels_padded.npz written")

    keep = {0, 1, 2, 10, 100, 200}
    stacked, kept, el = _run(dworld, model_id=v3, dt=1e-3, steps=200, keep=keep, solver=ars,
                             controls=controls, channels=True)
    _save("ars222_v3_channels_delaunay.npz", worlds.pack([dworld]), stacked, kept, dt=1e-3,
          model_id=v3, solver=ars, elapsed=el,
          extra={"control_" + k.split("_")[0]: v for k, v in controls.items()})


def make_block_trajectories():
    """@3 with an open-channel block (cells.channel_block.open_channel_block_weighted_modes@1) on
    its channel populations, read at the patch voltage."""
    from cells_b200 import worlds

    ars = "cells.solver.imex_ars222_face_electromigration@1"
    v3 = "cells.model.resolved_pump_tissue@3"
    rng = np.random.default_rng(41)
    world = worlds.with_channels(worlds.grid_world(4, 4, worlds.world_rng(5, 0)), rng,
                                 na=("nav", 2e-10, 0.5), k=("kv", 3e-10, 0.5), sigma=0.3)
    worlds.with_block(world, rng, slot=0, fraction=0.75)
    controls = dict(channel_control=rng.uniform(0.5, 1.0, (2, world.cells)))
    keep = {0, 1, 2, 5, 50, 100, 200, 300}
    stacked, kept, el = _run(world, model_id=v3, dt=1e-3, steps=300, keep=keep, solver=ars,
                             controls=controls, channels=True)
    _save("ars222_v3_block.npz", worlds.pack([world]), stacked, kept, dt=1e-3,
          model_id=v3, solver=ars, elapsed=el, extra={"control_channel": controls[
              "channel_control"]})

    dworld = worlds.with_channels(
        worlds.delaunay_world(40, worlds.world_rng(6, 0), junction_sigma=0.3,
                              gate=(0.02, 0.1, 0.8)), rng,
        na=("nav", 4e-10, 0.4), k=("kv", 5e-10, 0.6), sigma=0.3)
    dworld.bath_potential = -0.004
    worlds.with_block(dworld, rng, slot=0, fraction=0.5)
    worlds.with_block(dworld, rng, slot=1, fraction=0.8, valence=2, side="inside",
                      concentration_mM=(0.2, 1.0),
                      modes=((0.5, 0.05, 0.9), (0.25, 0.5, 0.5), (0.25, 5.0, 0.1)))
    controls = dict(
        membrane_control=rng.uniform(0.5, 1.0, dworld.cells),
        junction_control=rng.uniform(0.5, 1.0, dworld.edges),
        pump_control=rng.uniform(0.5, 1.0, dworld.cells),
        channel_control=rng.uniform(0.3, 1.0, (2, dworld.cells)),
    )
    # @3's own padded pytrees of the blocked world for the drop-in step.
    out = _run_reference_pytrees(dworld, model_id=v3, dt=1e-3, steps=40, keep={0, 1, 20, 40},
                                 padding=2, controls=controls)
    np.savez_compressed(os.path.join(HERE, "pytrees_v3_block_padded.npz"), **out)
    print("pytrees_v3_block_padded.npz written")

    keep = {0, 1, 2, 10, 100, 200}
    stacked, kept, el = _run(dworld, model_id=v3, dt=1e-3, steps=200, keep=keep, solver=ars,
                             controls=controls, channels=True)
    _save("ars222_v3_block_delaunay.npz", worlds.pack([dworld]), stacked, kept, dt=1e-3,
          model_id=v3, solver=ars, elapsed=el,
          extra={"control_" + k.split("_")[0]: v for k, v in controls.items()})


def make_n2_trajectories():
    """@3 under N2 (cells.solver.imex_ars222_implicit_conductances@1): the membranes', channels'
    and junctions' slope conductances implicit, junction gates by their exponential update."""
    from cells_b200 import worlds

    n2 = "cells.solver.imex_ars222_implicit_conductances@1"
    v3 = "cells.model.resolved_pump_tissue@3"
    world = worlds.single_grid_tissue(0)
    keep = {0, 1, 2, 10, 100, 300}
    stacked, kept, el = _run(world, model_id=v3, dt=1e-3, steps=300, keep=keep, solver=n2)
    _save("n2_grid4x4.npz", worlds.pack([world]), stacked, kept, dt=1e-3, model_id=v3,
          solver=n2, elapsed=el)

    rng = np.random.default_rng(31)
    dworld = worlds.with_channels(
        worlds.delaunay_world(40, worlds.world_rng(5, 0), junction_sigma=0.3,
                              gate=(0.02, 0.1, 0.8)), rng,
        na=("nav", 4e-10, 0.4), k=("kv", 5e-10, 0.6), sigma=0.3)
    dworld.bath_potential = -0.004
    controls = dict(
        membrane_control=rng.uniform(0.5, 1.0, dworld.cells),
        junction_control=rng.uniform(0.5, 1.0, dworld.edges),
        pump_control=rng.uniform(0.5, 1.0, dworld.cells),
        channel_control=rng.uniform(0.3, 1.0, (2, dworld.cells)),
    )
    keep = {0, 1, 2, 10, 100, 200}
    stacked, kept, el = _run(dworld, model_id=v3, dt=1e-3, steps=200, keep=keep, solver=n2,
                             controls=controls, channels=True)
    _save("n2_channels_delaunay.npz", worlds.pack([dworld]), stacked, kept, dt=1e-3,
          model_id=v3, solver=n2, elapsed=el,
          extra={"control_" + k.split("_")[0]: v for k, v in controls.items()})
    # @3's own padded pytrees under N2, for the drop-in step.
    out = _run_reference_pytrees(dworld, model_id=v3, dt=1e-3, steps=40, keep={0, 1, 20, 40},
                                 padding=2, controls=controls, solver=n2)
    np.savez_compressed(os.path.join(HERE, "pytrees_n2_padded.npz"), **out)
    print("pytrees_n2_padded.npz written")


def make_checks():
    """The reference's accepted-row device checks (@3's device_checks: surface_pump_checks
    .row_checks with its balances, magnitudes and ledger limits) on rows of its own trajectory
    of a gated Delaunay world with NaV1.2 and Kv1.5 populations: accepted rows at several step
    counts, and rows with planted faults (a material error, a heat that decreases)."""
    from cells.definitions.specs import parse_spec
    from cells.definitions.surface_pump_v3_spec import control_values
    from cells.registry.models import get_model

    from cells_b200 import worlds

    ars = "cells.solver.imex_ars222_face_electromigration@1"
    v3 = "cells.model.resolved_pump_tissue@3"
    rng = np.random.default_rng(41)
    world = worlds.with_channels(
        worlds.delaunay_world(36, worlds.world_rng(6, 0), junction_sigma=0.3,
                              gate=(0.02, 0.1, 0.8)), rng,
        na=("nav", 4e-10, 0.4), k=("kv", 5e-10, 0.6), sigma=0.3)
    world.bath_potential = -0.004
    raw = worlds.reference_definition(world, dt=1e-3, steps=120, model=v3, solver=ars)
    spec = parse_spec(raw)
    model = get_model(spec.model)
    state, p = model.initial_values(spec)
    cv = control_values(spec, [0.0])
    control = type(cv)(*(v[0] for v in cv))
    constants = model.device_check_constants(spec)
    rows = {0: state}
    for k in range(1, 121):
        state, ok = model.imex_step(state, 1e-3, control, p, xp=np)[:2]
        assert bool(ok)
        rows[k] = state
    cases = []
    for k in (1, 2, 10, 60, 120):
        cases.append((rows[k - 1], rows[k], k, "accepted"))
    bad = rows[60]._replace(amount_increment=np.asarray(rows[60].amount_increment).copy())
    bad.amount_increment[1, 3] += 1e-8  # 500 x the 2e-11 fmol material tolerance
    cases.append((rows[59], bad, 60, "material"))
    heat = rows[60]._replace(
        junction_dissipated_energy_pJ=np.asarray(rows[59].junction_dissipated_energy_pJ) - 1e-9)
    cases.append((rows[59], heat, 60, "dissipation"))
    out = {}
    for i, (prev, row, k, label) in enumerate(cases):
        failed, values = model.device_checks(prev, row, p, constants, k)
        for tag, st in (("prev", prev), ("row", row)):
            packed = _state_to_packed(st)
            packed.update(_channels_to_packed(st, world))
            for f, v in packed.items():
                out[f"case{i}_{tag}_{f}"] = v
        out[f"case{i}_steps"] = np.asarray(k)
        out[f"case{i}_label"] = np.asarray(label)
        out[f"case{i}_failed"] = np.asarray(failed)
        out[f"case{i}_values"] = np.asarray(values)
    out["cases"] = np.asarray(len(cases))
    out["material_atol"] = np.asarray(constants.material_atol)
    out["energy_rtol"] = np.asarray(constants.energy_rtol)
    out["checks"] = np.asarray(model.DEVICE_CHECKS)
    out["diagnostics"] = np.asarray(model.DEVICE_DIAGNOSTICS)
    np.savez_compressed(os.path.join(HERE, "device_checks.npz"), **_batch_arrays(
        worlds.pack([world])), **out)
    print("device_checks.npz written:", [c[3] for c in cases])


# The vector window (execution/vector_windows.py:348-410, _vector_window) on three gated 4x4 @3
# worlds: per-world step sizes, held-control indices and observation slots per row, per-world
# counts and first steps; world 1's second control has an availability above 1 (its step is
# refused at the first row that holds it). The same tables as tests/test_windows_gpu.py's
# per-world case.
WINDOW_DT = np.array([[1e-3] * 6, [5e-4] * 6, [1e-3, 2e-3, 1e-3, 2e-3, 1e-3, 2e-3]])
WINDOW_HELD = np.array([[0, 0, 1, 1, 0, 1], [1, 0, 0, 1, 1, 0], [0, 1, 0, 1, 0, 1]])
WINDOW_ROWS = 3
# A row without an observation takes slot WINDOW_ROWS (out of range: dropped), as the reference's
# window plan fills its slot table (vector_windows.py:676).
WINDOW_SLOTS = np.array([[0, 3, 1, 3, 3, 2], [3, 0, 3, 1, 2, 3], [2, 3, 3, 0, 1, 3]])
WINDOW_FIRST = np.array([0, 7, 3])
WINDOW_COUNTS = np.array([6, 6, 4])


def make_windows():
    """The reference's own _vector_window (run through the NumPy jax stand-in: vmap as a loop
    over worlds, scan as a loop over rows) over @3's checked_step and device_checks."""
    import jax

    from cells.definitions.specs import parse_spec
    from cells.definitions.surface_pump_v3_spec import control_values
    from cells.execution import vector_windows as VW
    from cells.registry.models import get_model

    from cells_b200 import worlds

    rng = np.random.default_rng(31)
    ws = [worlds.grid_world(4, 4, worlds.world_rng(31, k), gate=(0.015, 0.2, 1.0))
          for k in range(3)]
    b = worlds.pack(ws)
    membrane = rng.uniform(0.6, 1, b.cells)
    junction = rng.uniform(0.6, 1, b.edges)
    pump = rng.uniform(0.6, 1, b.cells)
    m1 = membrane.copy()
    m1[b.cell_offset[1] + 3] = 1.2
    controls = [(membrane, junction, pump), (m1, junction * 0.9, pump)]
    v3 = "cells.model.resolved_pump_tissue@3"
    states, params, constants, tables = [], [], [], []
    model = None
    for w, world in enumerate(ws):
        c0, c1 = b.cell_offset[w], b.cell_offset[w + 1]
        e0, e1 = b.edge_offset[w], b.edge_offset[w + 1]
        entries = []
        for mem, jun, pmp in controls:
            raw = worlds.reference_definition(
                world, dt=1e-3, steps=10, model=v3, membrane_control=np.minimum(mem[c0:c1], 1.0),
                junction_control=jun[e0:e1], pump_control=pmp[c0:c1])
            spec = parse_spec(raw)
            model = get_model(spec.model)
            cv = control_values(spec, [0.0])
            control = type(cv)(*(np.asarray(v[0]) for v in cv))
            membrane_field = control._fields[0]
            row = np.array(getattr(control, membrane_field), copy=True)
            row[:c1 - c0] = mem[c0:c1]  # an availability above 1 is the step's to refuse
            entries.append(control._replace(**{membrane_field: row}))
        state, p = model.initial_values(spec)
        states.append(state)
        params.append(p)
        constants.append(model.device_check_constants(spec))
        tables.append(jax.tree.map(lambda *v: np.stack(v), *entries))
    stack = lambda trees: jax.tree.map(lambda *v: np.stack([np.asarray(x) for x in v]), *trees)
    state, p, table, const = stack(states), stack(params), stack(tables), stack(constants)
    final, first, bits, maxima, stored = VW._vector_window(
        state, WINDOW_DT, WINDOW_COUNTS, table, WINDOW_HELD, WINDOW_SLOTS, WINDOW_FIRST, p,
        p.active, const, step=model.checked_step, checks=model.device_checks, rows=WINDOW_ROWS)
    out = {"first": np.asarray(first), "bits": np.asarray(bits), "maxima": np.asarray(maxima),
           "dt": WINDOW_DT, "held": WINDOW_HELD, "slots": WINDOW_SLOTS,
           "first_step": WINDOW_FIRST, "counts": WINDOW_COUNTS, "rows": np.asarray(WINDOW_ROWS),
           "material_atol": np.asarray(constants[0].material_atol),
           "energy_rtol": np.asarray(constants[0].energy_rtol)}
    for k, (mem, jun, pmp) in enumerate(controls):
        out[f"control{k}_membrane"], out[f"control{k}_junction"] = mem, jun
        out[f"control{k}_pump"] = pmp
    per_world = lambda tree, w: type(tree)(*(np.asarray(v)[w] for v in tree))
    for w in range(b.worlds):
        for f, v in _state_to_packed(per_world(final, w)).items():
            out[f"final{w}_{f}"] = v
        for r in range(WINDOW_ROWS):
            row = type(stored)(*(np.asarray(v)[w, r] for v in stored))
            for f, v in _state_to_packed(row).items():
                out[f"stored{w}_{r}_{f}"] = v
    np.savez_compressed(os.path.join(HERE, "vector_window.npz"), **_batch_arrays(b), **out)
    print("vector_window.npz written: first", out["first"], "bits", out["bits"])


def make_laws():
    from cells.laws import electrochemistry as ec
    from cells.laws.junctions import junction_voltage_relaxation as jg
    from cells.laws.pumps import nak_atp_mass_action_positive as pump

    x = np.concatenate([
        -np.logspace(-8, np.log10(50), 200)[::-1], [0.0],
        np.logspace(-8, np.log10(50), 200), [-1e-4, 1e-4, -9.999e-5, 9.999e-5],
    ])  # fmt: skip
    b = ec.bernoulli(x, xp=np)
    rng = np.random.default_rng(3)
    n = 500
    na = np.exp(rng.uniform(np.log(0.5), np.log(60.0), n))
    ko = np.exp(rng.uniform(np.log(1.0), np.log(20.0), n))
    mu_na = rng.uniform(-25000.0, 5000.0, n)
    mu_k = rng.uniform(-5000.0, 25000.0, n)
    cap = np.exp(rng.uniform(np.log(1e-3), np.log(0.1), n))
    avail = rng.uniform(0.0, 1.0, n)
    avail[:5] = 0.0
    params = pump.Parameters(cap, 1.5, 0.1, 0.1, 12.0, 0.2, 0.5, -37000.0)
    rates = pump.kinetics(na, ko, mu_na, mu_k, 310.15, params, avail, xp=np)
    v = rng.uniform(-0.12, 0.12, n)
    g = rng.uniform(0.1, 1.0, n)
    thr = rng.uniform(0.0, 0.05, n)
    gate = jg.rhs(g, v, jg.Parameters(thr, 0.1), xp=np)
    np.savez_compressed(
        os.path.join(HERE, "laws.npz"), bernoulli_x=x, bernoulli=b,
        pump_na=na, pump_ko=ko, pump_mu_na=mu_na, pump_mu_k=mu_k, pump_capacity=cap,
        pump_availability=avail, pump_cycles=rates.cycles_fmol_s,
        pump_energy=rates.cycle_free_energy_J_mol, pump_drive=rates.chemical_drive_J_mol,
        gate_g=g, gate_v=v, gate_threshold=thr, gate_rate=gate,
    )  # fmt: skip
    print("laws.npz written")


FIELD_NAMES = dict(
    amount_increment="amount_increment", extracellular_increment="extracellular_amount_increment",
    membrane_transferred="membrane_transferred", junction_transferred="junction_transferred",
    face_transferred="face_transferred", reservoir_supplied="reservoir_supplied",
    membrane_dissipated="membrane_dissipated_energy_pJ",
    junction_dissipated="junction_dissipated_energy_pJ",
    face_dissipated="face_dissipated_energy_pJ", electrode_charge="electrode_charge_transferred_C",
    reservoir_work="reservoir_work_pJ", electrode_work="electrode_work_pJ",
    junction_gate="junction_gate", pump_cycles="pump_cycles",
    pump_dissipated="pump_dissipated_energy_pJ", metabolic_work="metabolic_work_pJ",
)


def _field_world_arrays(world):
    from dataclasses import fields

    return {"fw_" + f.name: np.asarray(getattr(world, f.name)) for f in fields(world)
            if f.name != "pump"} | {"fw_pump": np.asarray(world.pump)}


def _run_field(name, world, *, dt, steps, keep, controls=None):
    """The reference's own step (@1, ARS(2,2,2) face electromigration, factored field) on one
    field world, its states at the keep steps in the oracle's field names."""
    from cells.definitions.specs import parse_spec
    from cells.execution.schedule import control_values
    from cells.registry.models import get_model

    from cells_b200 import field_worlds

    controls = controls or {}
    raw = field_worlds.reference_definition(world, dt=dt, steps=steps, **controls)
    spec = parse_spec(raw)
    model = get_model(spec.model)
    state, p = model.initial_values(spec)
    cv = control_values(spec, [0.0])
    control = type(cv)(*(v[0] for v in cv))
    assert np.array_equal(np.asarray(p.face_factor), world.face_factor)
    snaps = []
    t0 = time.time()
    for k in range(steps + 1):
        if k:
            state, ok = model.imex_step(state, dt, control, p, xp=np)[:2]
            if not bool(ok):
                raise RuntimeError(f"reference refused step {k}")
        if k in keep:
            snaps.append({f: np.asarray(getattr(state, r)) for f, r in FIELD_NAMES.items()})
    out = _field_world_arrays(world)
    out.update({"control_" + k: np.asarray(v) for k, v in
                (("membrane", control.membrane), ("junction", control.junction),
                 ("pump", control.pump))})
    out["dt"], out["steps"] = np.asarray(dt), np.asarray(sorted(keep))
    for f in FIELD_NAMES:
        out["ref_" + f] = np.stack([s[f] for s in snaps])
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(f"{name} written ({steps} steps, {time.time() - t0:.1f} s)")


def make_field_trajectories():
    """Field worlds (cells facing a resolved extracellular grid with a held ring)."""
    from cells_b200 import field_worlds as FW
    from cells_b200 import worlds

    w = FW.field_world(10, 3, 2, worlds.world_rng(11, 0))
    _run_field("field_grid10.npz", w, dt=5e-4, steps=400,
               keep={0, 1, 2, 5, 10, 50, 100, 200, 400})
    rng = np.random.default_rng(12)
    w = FW.field_world(14, 4, 3, worlds.world_rng(12, 0), gate=(0.015, 0.2, 1.0),
                       junction_sigma=0.3)
    controls = dict(membrane_control=rng.uniform(0.6, 1.0, w.cells),
                    junction_control=rng.uniform(0.6, 1.0, w.edges),
                    pump_control=rng.uniform(0.6, 1.0, w.cells))
    _run_field("field_gated14.npz", w, dt=5e-4, steps=200, keep={0, 1, 3, 20, 100, 200},
               controls=controls)
    w = FW.field_world(24, 6, 3, worlds.world_rng(13, 0))
    _run_field("field_grid24.npz", w, dt=5e-4, steps=60, keep={0, 1, 10, 60})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("CELLS_REFERENCE"),
                    help="the reference project's root (or set CELLS_REFERENCE)")
    ap.add_argument("--only", choices=("laws", "trajectories", "channels", "block", "n2",
                                       "checks", "field", "windows"))
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set CELLS_REFERENCE to the reference project's root")
    _setup(args.reference)
    if args.only in (None, "laws"):
        make_laws()
    if args.only in (None, "trajectories"):
        make_trajectories()
    if args.only in (None, "channels"):
        make_channel_trajectories()
    if args.only in (None, "block"):
        make_block_trajectories()
    if args.only in (None, "n2"):
        make_n2_trajectories()
    if args.only in (None, "checks"):
        make_checks()
    if args.only in (None, "field"):
        make_field_trajectories()
    if args.only in (None, "windows"):
        make_windows()


if __name__ == "__main__":
    main()
