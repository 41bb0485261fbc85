"""CPU oracle of the accepted-row device checks for held-bath worlds.

TEST INFRASTRUCTURE ONLY, like oracle/tissue.py.

Restates models/surface_pump_checks.row_checks (:101-192) as @3 calls it (device_checks,
models/surface_pump_v3.py:5572-5597, with device_balances :5556-5569 -> surface_pump_v2
.device_balances :686-709 -> surface_pump_checks.tissue_balances :34-101, and channel_magnitudes
:5243-5258 -> surface_pump.ledger_magnitudes :705-738, ledger_limits :752-800), for worlds whose
every cell faces its world's one held bath and no faces. Per world it returns the twelve checks
in DEVICE_CHECKS order (domain, the ten ledgers of LEDGERS, dissipation) and the twelve
DEVICE_DIAGNOSTICS (each ledger's max |residual|, the energy residual relative to its flows, the
global-charge residual relative to its bound).

Held-bath simplifications (surface_field.bind's components): each cell's capacitor component
holds the bath, so no node is a representative (the capacitor ledger's bound is
CHARGE_ATOL_C + CHARGE_RTOL |charge| alone) and every cell is grounded through the bath (the
global-charge ledger's grounded allowance sums every cell's |z F dn|).
"""

from __future__ import annotations

import numpy as np

from oracle import tissue as T

F, R = T.F, T.R
VALENCE = T.VALENCE
K = T.CHARGE_PER_FMOL
EPS = np.finfo(float).eps
LEDGER_STEP_ROUNDING = 2.5  # models/surface_pump.py:113
COMPONENT_STEP_ROUNDING = 2.5  # numerics/surface_field.py (COMPONENT_STEP_ROUNDING)
GLOBAL_CHARGE_ATOL_C = 3e-25  # models/surface_pump.py:96
GLOBAL_CHARGE_ROUNDING = 256 * EPS  # :97
ENERGY_ATOL_PJ = 2e-8  # models/surface_tissue.py:29
WORK_BOUND_PJ = 3e-12  # ledger_limits' fixed work bounds
DISSIPATION_ATOL_PJ = 1e-12  # models/surface_pump_checks.py:24
CHECKS = ("domain", "local", "outside", "total", "charge", "electrode", "global_charge", "energy",
          "reservoir_work", "electrode_work", "metabolic_work", "dissipation")
DIAGNOSTICS = ("balance_error_fmol", "extracellular_balance_error_fmol",
               "global_balance_error_fmol", "capacitor_charge_error_C", "electrode_charge_error_C",
               "global_charge_error_C", "energy_balance_error_pJ", "reservoir_work_error_pJ",
               "electrode_work_error_pJ", "metabolic_work_error_pJ",
               "energy_balance_relative", "global_charge_bound_ratio")


def _world_max(values, index, worlds):
    out = np.zeros(worlds)
    np.maximum.at(out, index, values)
    return out


def _world_any(values, index, worlds):
    out = np.zeros(worlds, dtype=bool)
    np.logical_or.at(out, index, values)
    return out


def _world_sum(values, index, worlds):
    out = np.zeros(worlds)
    np.add.at(out, index, values)
    return out


def membrane_total(state, b):
    """Membrane transfer with the channels' and the pump's (device_balances' `total`)."""
    moved = state.membrane_transferred.copy()
    idx = np.arange(b.cells)
    for k in range(b.channel_slots):
        moved[b.channel_species[k], idx] += state.channel_transferred[k]
    return moved - T.STOICHIOMETRY[:, None] * state.pump_cycles


def capacitor_charge(state, b, topo):
    """The capacitor ledger per cell: image - initial charge + plate change - charge increment,
    the image C base of the initial charges' solve (tissue_balances' `charge`)."""
    w = topo.cell_world
    base = T.capacitor_potential(b.initial_charge, b, topo)
    image = b.capacitance * base + (-b.capacitance) * b.bath_potential[w]
    n = state.amount_increment
    q = K * ((VALENCE[0] * n[0] + VALENCE[1] * n[1]) + VALENCE[2] * n[2])
    scale = topo.capacitor_scale[w]
    factor = np.sqrt(b.capacitance / scale)
    dp = q / scale / factor / factor
    cap = b.capacitance * dp
    return ((image - b.initial_charge) + cap) - q, dp


def energy(state, b, topo, dp):
    """The energy ledger (pJ) per world: chemical free energy + capacitor energy + heat -
    reservoir and electrode work, with the pump's heat, the channels' heat, less the metabolic
    work (tissue_balances + @2's and @3's device_balances terms)."""
    w = topo.cell_world
    a, d = b.amount_reference, state.amount_increment
    t = b.temperature[w]
    chem = 1e-3 * R * t * np.sum(d * (np.log(a / b.volume) - 1) + (a + d) * np.log1p(d / a),
                                 axis=0)
    v0 = T.capacitor_potential(b.initial_charge, b, topo) - b.bath_potential[w]
    electric = 0.5e12 * (b.capacitance * dp * (2 * v0 + dp))
    cell = (chem + electric + state.membrane_dissipated + state.pump_dissipated
            - state.metabolic_work + np.sum(state.channel_dissipated, axis=0))
    total = _world_sum(cell, w, b.worlds)
    total += _world_sum(state.junction_dissipated, topo.edge_world, b.worlds)
    return total - state.reservoir_work - state.electrode_work


def flows(state, b, topo):
    """The energy bound's flows: sum of |heat and work accumulators| per world."""
    w, e = topo.cell_world, topo.edge_world
    cell = (np.abs(state.membrane_dissipated) + np.abs(state.pump_dissipated)
            + np.abs(state.metabolic_work) + np.sum(np.abs(state.channel_dissipated), axis=0))
    return (_world_sum(cell, w, b.worlds) + _world_sum(np.abs(state.junction_dissipated), e,
                                                        b.worlds)
            + np.abs(state.reservoir_work) + np.abs(state.electrode_work))


def row_checks(previous, row, b, topo, steps, material_atol, energy_rtol):
    """(failed [W, 12] bool, values [W, 12]) for one accepted row and its predecessor."""
    W = b.worlds
    w, ew = topo.cell_world, topo.edge_world
    tol = np.asarray(material_atol, dtype=float)
    rounding = LEDGER_STEP_ROUNDING * EPS * steps
    bal = T.balances(row, b, topo)
    moved_abs = (np.abs(row.membrane_transferred) + np.abs(T.STOICHIOMETRY[:, None] * row.pump_cycles))
    idx = np.arange(b.cells)
    for k in range(b.channel_slots):
        moved_abs[b.channel_species[k], idx] += np.abs(row.channel_transferred[k])
    hj = np.abs(row.junction_transferred)
    mag_local = np.abs(row.amount_increment) + moved_abs
    snd = np.zeros_like(mag_local)
    np.add.at(snd, (slice(None), topo.sender), hj)
    rcv = np.zeros_like(mag_local)
    np.add.at(rcv, (slice(None), topo.receiver), hj)
    mag_local = (mag_local + snd) + rcv
    supplied = np.abs(row.reservoir_supplied)
    mag_outside = np.zeros((3, W))
    np.add.at(mag_outside, (slice(None), w), moved_abs)
    mag_outside = mag_outside + supplied
    mag_total = np.zeros((3, W))
    np.add.at(mag_total, (slice(None), w), np.abs(row.amount_increment))
    mag_total = mag_total + supplied
    co = b.bath_amount / b.bath_volume
    mu = R * b.temperature * np.log(co) + VALENCE[:, None] * F * b.bath_potential
    moved_charge = K * np.sum(np.abs(VALENCE[:, None] * row.reservoir_supplied), axis=0) + np.abs(
        row.electrode_charge)
    mag_rw = np.abs(row.reservoir_work) + 1e-3 * np.sum(np.abs(mu) * supplied, axis=0)
    mag_ew = np.abs(row.electrode_work) + 1e12 * np.abs(b.bath_potential * row.electrode_charge)
    drive = T.chemical_drive(tuple(b.pump[k][w] for k in range(7)), b.temperature[w])
    mag_mw = np.abs(row.metabolic_work) + 1e-3 * np.abs(drive * row.pump_cycles)
    charge_res, dp = capacitor_charge(row, b, topo)
    q = b.initial_charge + K * ((VALENCE[0] * row.amount_increment[0]
                                 + VALENCE[1] * row.amount_increment[1])
                                + VALENCE[2] * row.amount_increment[2])
    e_val = energy(row, b, topo, dp)
    fl = flows(row, b, topo)
    increments = K * np.sum(np.abs(VALENCE[:, None] * row.amount_increment), axis=0)
    grounded = COMPONENT_STEP_ROUNDING * EPS * steps * _world_sum(increments, w, W)
    gc_bound = GLOBAL_CHARGE_ATOL_C + GLOBAL_CHARGE_ROUNDING * moved_charge
    gc_limit = np.maximum(gc_bound + rounding * moved_charge, gc_bound + grounded)
    ledgers = (
        ("cell", bal["local"], tol[:, None] + rounding * mag_local),
        ("world", bal["outside"], tol[:, None] + rounding * mag_outside),
        ("world", bal["total"], tol[:, None] + rounding * mag_total),
        ("cell", charge_res, T.CHARGE_ATOL_C + T.CHARGE_RTOL * np.abs(q)),
        ("world", bal["electrode"], T.CHARGE_ATOL_C + T.CHARGE_RTOL * np.abs(row.electrode_charge)),
        ("world", bal["global_charge"], gc_limit),
        ("world", e_val, ENERGY_ATOL_PJ + energy_rtol * fl),
        ("world", bal["reservoir_work"], WORK_BOUND_PJ + rounding * mag_rw),
        ("world", bal["electrode_work"], WORK_BOUND_PJ + rounding * mag_ew),
        ("cell", bal["metabolic_work"], WORK_BOUND_PJ + rounding * mag_mw),
    )
    failed = np.zeros((W, 12), dtype=bool)  # domain, the ten ledgers, dissipation
    values = np.zeros((W, 12))  # the ten ledgers' max |residual|, the two ratios
    failed[:, 0] = ~T.domain_valid(row, b, topo)
    for k, (kind, value, limit) in enumerate(ledgers, start=1):
        value = np.asarray(value, dtype=float)
        bad = ~np.isfinite(value) | (np.abs(value) > limit)
        mag = np.abs(value)
        if kind == "cell":
            bad = bad.reshape(-1, b.cells) if bad.ndim > 1 else bad[None]
            mag = mag.reshape(-1, b.cells) if mag.ndim > 1 else mag[None]
            failed[:, k] = _world_any(np.any(bad, axis=0), w, W)
            values[:, k - 1] = _world_max(np.max(mag, axis=0), w, W)
        else:
            bad = bad.reshape(-1, W)
            mag = mag.reshape(-1, W)
            failed[:, k] = np.any(bad, axis=0)
            values[:, k - 1] = np.max(mag, axis=0)
    values[:, 10] = np.abs(e_val) / np.maximum(fl, ENERGY_ATOL_PJ)
    values[:, 11] = np.abs(bal["global_charge"]) / gc_limit
    decreasing = np.zeros(W, dtype=bool)
    for name, index in (("membrane_dissipated", w), ("pump_dissipated", w),
                        ("junction_dissipated", ew)):
        v, p_ = getattr(row, name), getattr(previous, name)
        decreasing |= _world_any((v < -DISSIPATION_ATOL_PJ) | (v - p_ < -DISSIPATION_ATOL_PJ),
                                 index, W)
    for k in range(b.channel_slots):
        v, p_ = row.channel_dissipated[k], previous.channel_dissipated[k]
        decreasing |= _world_any((v < -DISSIPATION_ATOL_PJ) | (v - p_ < -DISSIPATION_ATOL_PJ), w, W)
    failed[:, 11] = decreasing
    return failed, values
