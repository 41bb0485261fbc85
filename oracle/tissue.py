"""CPU oracle: a NumPy restatement of the reference's held-bath pump-leak tissue step.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg may import this module, and only as the parity reference or the timed CPU
baseline; the product path (``cells_b200``) never calls it and refuses to run without its CUDA
library.

What it restates (citations are paths inside the reference project):

* point laws: ``bernoulli`` (src/cells/laws/electrochemistry.py:25-32), the constant-field route
  flux ``selective_flux`` (src/cells/laws/junctions/selective.py:28-50), the Na/K-ATPase
  ``kinetics`` and ``chemical_drive`` (src/cells/laws/pumps/nak_atp_mass_action_positive.py:55-98),
  the junction gate ``kinetics``/``rhs`` (src/cells/laws/junctions/junction_voltage_relaxation.py:
  43-67) and their domain predicates;
* the route transport and its scatters (src/cells/numerics/surface_transport.py:298-386);
* the capacitor field closure for a world whose every capacitor component holds its held bath
  (src/cells/numerics/surface_field.py:577-600, :614-855 with no floating offsets), and the IMEX
  operator solve with no faces (src/cells/numerics/surface_imex.py:207-225, :269-278), each in
  the reference's own arithmetic order (diagonal Cholesky factor of the scaled matrix);
* the explicit stage rates (src/cells/models/surface_pump.py:158-240), the ARS(2,2,2) step with
  its ledger bookings (src/cells/models/surface_pump.py:259-362, tableau
  src/cells/numerics/surface_imex.py:47-69), and the checked RK4 of the same right-hand side
  (src/cells/numerics/fixed_step.py:25-71, rates of src/cells/models/surface_kinetic.py:221-410);
* the ledgers (src/cells/models/surface_tissue.py:536-611, src/cells/models/surface_kinetic.py:
  470-482).

Pinned: ``tests/golden/make_golden.py`` runs the reference's own step (models/surface_pump.py
and models/surface_pump_v3.py on their NumPy branch) on seeded worlds and stores trajectories;
``tests/test_oracle_golden.py`` checks this restatement against them.

Layout (packed worlds, see cells_b200/worlds.py): cell arrays are [S, C] or [C], junction arrays
[S, E] or [E], per-world arrays [S, W] or [W]. A world's step is accepted or refused as a whole,
as the reference's ``checked_step`` does (refused: state unchanged, valid False).
"""

from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np

AVOGADRO = 6.02214076e23
F = AVOGADRO * 1.602176634e-19
R = AVOGADRO * 1.380649e-23
MOL_PER_FMOL = 1e-15
CHARGE_PER_FMOL = F * MOL_PER_FMOL
VALENCE = np.array([1.0, 1.0, -1.0])
STOICHIOMETRY = np.array([-3.0, 2.0, 0.0])
SODIUM_PER_CYCLE, POTASSIUM_PER_CYCLE = -3, 2
STANDARD_STATE_mM = 1000.0
MAX_ABS_X = 50.0  # surface_transport.py:20
MAX_ABS_AFFINITY_OVER_RT = 80.0
MAX_ABS_ION_POTENTIAL_OVER_RT = 1600.0
TEMPERATURE_DOMAIN_K = (200.0, 400.0)
MAX_ABS_JUNCTION_V = 0.120
CHARGE_ATOL_C = 3e-25
CHARGE_RTOL = 2e-12
GAMMA = 1.0 - 1.0 / math.sqrt(2.0)
DELTA = 1.0 - 1.0 / (2.0 * GAMMA)

CELL_FIELDS = (
    "amount_increment",  # [S, C]
    "membrane_transferred",  # [S, C]
    "membrane_dissipated",  # [C]
    "pump_cycles",  # [C]
    "pump_dissipated",  # [C]
    "metabolic_work",  # [C]
)
EDGE_FIELDS = ("junction_transferred", "junction_dissipated", "junction_gate")  # [S,E],[E],[E]
WORLD_FIELDS = ("reservoir_supplied", "electrode_charge", "reservoir_work", "electrode_work")
CHANNEL_FIELDS = ("channel_gate", "channel_transferred", "channel_dissipated")  # cell-indexed
EXPLICIT_STEP_BOUND = 1.0  # dt x the Gershgorin membrane rate (surface_pump.py:112)
VOLTAGE_DOMAIN_V = (-0.120, 0.060)  # the channel laws' domain (laws/channels/kv1p5_mh.py:26)
GATE_SERIES_LIMIT = 1e-3  # numerics/exponential_gates.py:33


class State(NamedTuple):
    amount_increment: np.ndarray
    membrane_transferred: np.ndarray
    membrane_dissipated: np.ndarray
    pump_cycles: np.ndarray
    pump_dissipated: np.ndarray
    metabolic_work: np.ndarray
    junction_transferred: np.ndarray
    junction_dissipated: np.ndarray
    junction_gate: np.ndarray
    reservoir_supplied: np.ndarray
    electrode_charge: np.ndarray
    reservoir_work: np.ndarray
    electrode_work: np.ndarray
    channel_gate: np.ndarray  # [2, NCH, C] gate rows (m, h) of each population
    channel_transferred: np.ndarray  # [NCH, C] fmol of the population's permeant species
    channel_dissipated: np.ndarray  # [NCH, C] pJ


class Control(NamedTuple):
    membrane: np.ndarray  # [C] availability of each cell's patch
    junction: np.ndarray  # [E]
    pump: np.ndarray  # [C]
    channel: np.ndarray = None  # [NCH, C]


def initial_state(b):
    c, e, w, nch = b.cells, b.edges, b.worlds, b.channel_slots
    return State(
        np.zeros((3, c)), np.zeros((3, c)), np.zeros(c), np.zeros(c), np.zeros(c), np.zeros(c),
        np.zeros((3, e)), np.zeros(e), b.gate_initial.copy(),
        np.zeros((3, w)), np.zeros(w), np.zeros(w), np.zeros(w),
        np.array(b.channel_gate_initial, dtype=float), np.zeros((nch, c)), np.zeros((nch, c)),
    )  # fmt: skip


def full_control(b, membrane=1.0, junction=1.0, pump=1.0, channel=1.0):
    return Control(
        np.full(b.cells, float(membrane)), np.full(b.edges, float(junction)),
        np.full(b.cells, float(pump)), np.full((b.channel_slots, b.cells), float(channel)),
    )  # fmt: skip


class Topology(NamedTuple):
    """Derived indices: world of each cell/edge, global endpoints, capacitor scale per world."""

    cell_world: np.ndarray
    edge_world: np.ndarray
    sender: np.ndarray
    receiver: np.ndarray
    capacitor_scale: np.ndarray  # [W] sum of the world's patch capacitances (bind's max |C|)


def topology(b):
    cells = np.diff(b.cell_offset)
    edges = np.diff(b.edge_offset)
    cell_world = np.repeat(np.arange(b.worlds), cells)
    edge_world = np.repeat(np.arange(b.worlds), edges)
    base = b.cell_offset[:-1][edge_world]
    scale = np.zeros(b.worlds)
    # surface_field.bind accumulates the held bath's diagonal in membrane order (:327-333); the
    # bath's diagonal is the largest |C| entry (:354), so the scale is that sum.
    np.add.at(scale, cell_world, b.capacitance)
    return Topology(
        cell_world, edge_world, base + b.sender.astype(np.int64),
        base + b.receiver.astype(np.int64), scale,
    )  # fmt: skip


# ---------------------------------------------------------------------------------------------
# Point laws


def bernoulli(x):
    """x/expm1(x) with the reference's series below |x| < 1e-4 (electrochemistry.py:25-32)."""
    small = np.abs(x) < 1e-4
    regular = np.where(small, 1.0, x)
    series_x = np.where(small, x, 0.0)
    series = 1 - series_x / 2 + series_x**2 / 12 - series_x**4 / 720
    with np.errstate(all="ignore"):
        return np.where(small, series, regular / np.expm1(regular))


def route_flux(c_from, c_to, dv, temperature, area, permeability, multiplier):
    """selective_flux with residual 0 and gate 1 (selective.py:28-50), fmol/s, [S, routes]."""
    x = VALENCE[:, None] * F * dv / (R * temperature)
    available = multiplier * (0.0 + (1 - 0.0) * 1.0)
    return (
        area * permeability * available / MOL_PER_FMOL
        * (c_from * bernoulli(-x) - c_to * bernoulli(x))
    )  # fmt: skip


def chemical_drive(pump, temperature):
    """ΔG of hydrolysis at the 1 M standard state (nak_atp_mass_action_positive.py:55-60)."""
    atp, adp, pi, _, _, _, dg0 = pump
    return dg0 + R * temperature * (
        np.log(adp) + np.log(pi) - np.log(atp) - np.log(STANDARD_STATE_mM)
    )


def pump_kinetics(na_in, k_out, mu_na, mu_k, temperature, pump, capacity, availability):
    """Signed cycles (fmol/s), cycle free energy and drive (J/mol) (…positive.py:63-98)."""
    atp, _, _, km_na, km_k, km_atp, _ = pump
    drive = chemical_drive(pump, temperature)
    energy = drive + SODIUM_PER_CYCLE * mu_na + POTASSIUM_PER_CYCLE * mu_k
    a = energy / (R * temperature)
    log_saturation = (
        -np.logaddexp(0.0, 3 * (np.log(km_na) - np.log(na_in)))
        - np.logaddexp(0.0, 2 * (np.log(km_k) - np.log(k_out)))
        - np.logaddexp(0.0, np.log(km_atp) - np.log(atp))
    )
    enabled = (capacity > 0) & (availability > 0)
    safe_capacity = np.where(enabled, capacity, 1.0)
    safe_availability = np.where(enabled, availability, 1.0)
    with np.errstate(all="ignore"):
        magnitude = np.exp(
            np.log(safe_capacity) + np.log(safe_availability) + log_saturation
            + np.maximum(a, 0.0)
        )  # fmt: skip
        departure = np.where(a >= 0, np.expm1(-a), -np.expm1(a))
    cycles = np.where(enabled, magnitude * departure, 0.0)
    return cycles, energy, drive


def pump_domain(na_in, k_out, mu_na, mu_k, temperature, pump, capacity, availability):
    """domain_valid of the pump law (…positive.py:101-148), per route."""
    atp, adp, pi, km_na, km_k, km_atp, dg0 = pump

    def positive(v):
        return np.isfinite(v) & (v > 0)

    valid = positive(na_in) & positive(k_out)
    for v in (atp, adp, pi, km_na, km_k, km_atp):
        valid = valid & positive(v)
    valid = valid & np.isfinite(dg0)
    t_ok = np.isfinite(temperature) & (temperature >= 200.0) & (temperature <= 400.0)
    rt = R * np.where(t_ok, temperature, 298.15)
    valid = valid & t_ok & np.isfinite(capacity) & (capacity >= 0)
    valid = valid & np.isfinite(availability) & (availability >= 0) & (availability <= 1)
    scaled = []
    for mu in (mu_na, mu_k):
        s = mu / rt
        ok = np.isfinite(s) & (np.abs(s) <= MAX_ABS_ION_POTENTIAL_OVER_RT)
        valid = valid & ok
        scaled.append(np.where(ok, s, 0.0))
    affinity = (
        dg0 / rt + np.log(adp) + np.log(pi) - np.log(atp) - np.log(STANDARD_STATE_mM)
        + SODIUM_PER_CYCLE * scaled[0] + POTASSIUM_PER_CYCLE * scaled[1]
    )  # fmt: skip
    return valid & np.isfinite(affinity) & (np.abs(affinity) <= MAX_ABS_AFFINITY_OVER_RT)


def gate_rhs(gate, voltage, threshold, minimum):
    """junction_voltage_relaxation.kinetics/rhs (:43-67)."""
    shift = np.abs(voltage) - threshold
    alpha = 1.3 * np.exp(-77.0 * shift)
    log_beta = np.log(0.065) + 140.0 * shift
    beta = 20.0 * np.exp(-np.logaddexp(0.0, -log_beta))
    return alpha * (1 - gate) - beta * (gate - minimum)


def gate_domain(gate, voltage, threshold, minimum, availability):
    return (
        np.isfinite(threshold) & (threshold >= 0) & (threshold <= MAX_ABS_JUNCTION_V)
        & np.isfinite(minimum) & (minimum >= 0) & (minimum <= 1)
        & np.isfinite(voltage) & (np.abs(voltage) <= MAX_ABS_JUNCTION_V)
        & np.isfinite(gate) & (gate >= minimum) & (gate <= 1)
        & np.isfinite(availability) & (availability >= 0) & (availability <= 1)
    )  # fmt: skip


# ---------------------------------------------------------------------------------------------
# Voltage-gated channel laws (targets [2, ...] and time constants [2, ...] in s; V in volts)

KV1P5, NAV1P2, HH_K_N4 = 0, 2, 100


def kv1p5_kinetics(v):
    """cells.channel.kv1p5_mh@1 (laws/channels/kv1p5_mh.py:29-41)."""

    def sigmoid(value):
        e = np.exp(-np.abs(value))
        return np.where(value >= 0, 1 / (1 + e), e / (1 + e))

    targets = np.stack((sigmoid((v + 0.0060) / 0.0064), sigmoid(-(v + 0.0253) / 0.0035)))
    tau = np.stack((0.008330 - 0.1163 * v, 1.620000 - 15.500 * v))
    return targets, tau


def nav1p2_kinetics(v):
    """cells.channel.nav1p2_m3h_regularized@1 (laws/channels/nav1p2_m3h_regularized.py:22-44)."""
    shifted = (v + 0.025) / 0.009
    activation = 0.182 * 9 * bernoulli(-shifted)
    deactivation = 0.124 * 9 * bernoulli(shifted)
    recovery = 0.024 * 5 * bernoulli(-(v + 0.040) / 0.005)
    inactivation = 0.0091 * 5 * bernoulli((v + 0.065000123) / 0.005)
    targets = np.stack((activation / (activation + deactivation),
                        1 / (1 + np.exp((v + 0.055) / 0.0062))))
    tau = np.stack((0.001 / (activation + deactivation), 0.001 / (recovery + inactivation)))
    return targets, tau


def hh_k_n4_kinetics(v):
    """Hodgkin-Huxley K activation n (Hodgkin and Huxley 1952, J. Physiol. 117:500, rest at
    -65 mV): alpha_n = 0.01 (Vm + 55) / (1 - exp(-(Vm + 55)/10)) and beta_n = 0.125
    exp(-(Vm + 65)/80) per ms, Vm in mV; alpha_n written as 0.1 B(-(Vm + 55)/10) with the
    Bernoulli function, whose removable singularity takes its limit. One gate (row 1 unused)."""
    vm = 1000.0 * v
    alpha = 100.0 * bernoulli(-(vm + 55.0) / 10.0)  # 1/s
    beta = 125.0 * np.exp(-(vm + 65.0) / 80.0)  # 1/s
    targets = np.stack((alpha / (alpha + beta), np.zeros_like(v)))
    tau = np.stack((1.0 / (alpha + beta), np.ones_like(v)))
    return targets, tau


def gate_rows_active(code):
    """[2, ...] rows that relax (channel_gate_active): both for Kv1.5 and NaV1.2, n alone for
    the HH n^4 law."""
    code = np.asarray(code)
    return np.stack((np.ones(code.shape, dtype=bool), code != HH_K_N4))


def channel_kinetics(v, code):
    """Each population's targets and time constants by its law code, [2, NCH, C]."""
    out_t = np.zeros((2, *code.shape))
    out_tau = np.ones((2, *code.shape))
    with np.errstate(all="ignore"):
        for law, fn in ((KV1P5, kv1p5_kinetics), (NAV1P2, nav1p2_kinetics),
                        (HH_K_N4, hh_k_n4_kinetics)):
            mask = code == law
            if np.any(mask):
                t, tau = fn(np.broadcast_to(v, code.shape))
                out_t = np.where(mask[None], t, out_t)
                out_tau = np.where(mask[None], tau, out_tau)
    return out_t, out_tau


def channel_opening(gate, code):
    """m^3 h (NaV1.2), m h (Kv1.5), n^4 (HH), [NCH, C] (sodium_channels.opening)."""
    m, h = gate[0], gate[1]
    return np.where(code == NAV1P2, m**3 * h, np.where(code == HH_K_N4, m**4, m * h))


def channel_domain(v, targets, tau):
    """channel_domain_valid (surface_pump_v3.py:848-858) per population, [NCH, C]."""
    inside = (v >= VOLTAGE_DOMAIN_V[0]) & (v <= VOLTAGE_DOMAIN_V[1])
    kin = np.isfinite(targets) & (targets >= 0) & (targets <= 1) & np.isfinite(tau) & (tau > 0)
    return inside & np.all(kin, axis=0)


def lag_weight(z):
    """1 - (1 - e^-z)/z (numerics/exponential_gates.py:36-41)."""
    small = z < GATE_SERIES_LIMIT
    safe = np.where(small, 1.0, z)
    series = z * (0.5 - z * (1 / 6 - z * (1 / 24 - z / 120)))
    return np.where(small, series, (np.expm1(-safe) + safe) / safe)


def advance_gates(gate, target_start, tau_start, target_end, tau_end, dt):
    """Exponential update with a linearly varying target (numerics/exponential_gates.py:44-51)."""
    z = 0.5 * dt * (1 / tau_start + 1 / tau_end)
    return gate + (target_start - gate) * -np.expm1(-z) + (target_end - target_start) * lag_weight(z)


# ---------------------------------------------------------------------------------------------
# Field closure (held-bath worlds: each cell's one patch faces its world's held bath)


def node_charge(state, b):
    """Cell charge (C): anchor plus F sum_s z n (surface_pump.node_charge, surface_tissue.py:269)."""
    q = CHARGE_PER_FMOL * np.sum(VALENCE[:, None] * state.amount_increment, axis=0)
    return b.initial_charge + q


def capacitor_potential(charge, b, topo):
    """surface_field._capacitor_solve on the cells (surface_field.py:596-600): the scaled
    capacitor matrix is diagonal on the free cells, factor sqrt(c/scale); two substitutions."""
    bath = b.bath_potential[topo.cell_world]
    scale = topo.capacitor_scale[topo.cell_world]
    rhs = (charge - (-b.capacitance) * bath) / scale
    factor = np.sqrt(b.capacitance / scale)
    return rhs / factor / factor


def operator_potential(charge, b, topo):
    """surface_imex.factor_operator/solve_operator with no faces (surface_imex.py:207-225,
    :269-278): Jacobi scale 1/sqrt(c), reduced diagonal (c s) s, Cholesky sqrt of it."""
    bath = b.bath_potential[topo.cell_world]
    s = 1.0 / np.sqrt(b.capacitance)
    factor = np.sqrt(b.capacitance * s * s)
    rhs = (charge - (-b.capacitance) * bath) * s
    phi = rhs / factor / factor * s
    residual = b.capacitance * phi + (-b.capacitance) * bath - charge
    return phi, residual


def capacitor_plate_sum(state, b, topo):
    """Held bath plate charge of the charge-only increment (surface_tissue.capacitor_change,
    :329-393): C dp at the bath row, dp the capacitor solve of z F n in species order."""
    amount = state.amount_increment
    q = CHARGE_PER_FMOL * (VALENCE[0] * amount[0] + VALENCE[1] * amount[1] + VALENCE[2] * amount[2])
    scale = topo.capacitor_scale[topo.cell_world]
    factor = np.sqrt(b.capacitance / scale)
    dp = q / scale / factor / factor
    out = np.zeros(b.worlds)
    np.add.at(out, topo.cell_world, -b.capacitance * dp)
    return out


# ---------------------------------------------------------------------------------------------
# Rates


class Rates(NamedTuple):
    state: State  # d(state)/dt of the explicit stage (surface_pump.explicit_rates)
    valid: np.ndarray  # [W]
    membrane_voltage: np.ndarray  # [C]


def concentrations(state, b):
    ci = (b.amount_reference + state.amount_increment) / b.volume
    co = b.bath_amount / b.bath_volume
    return ci, co


NORMAL = float(np.finfo(np.float64).tiny)


def channel_block(blk, k, v, temperature):
    """The open-channel block of slot k's populations at their patch voltages v [C]
    (laws/channels/open_channel_block.py: dissociation, fractions, unblocked_fraction, slope,
    domain_valid; surface_pump_v3.channel_block :1003-1036 without a voltage shift).
    Returns (u, slope, valid) [C]."""
    steep = blk.steepness[:, k]
    per_volt = steep * (F / (R * temperature))  # exponent_per_volt
    K = blk.k0_mM[:, k] * np.exp(per_volt * v)
    c = blk.concentration_mM[k]
    total = c + K
    theta, free = c / total, K / total
    w = blk.weight[:, k]
    a = np.abs(per_volt)
    num, den = w[0] * free[0], w[0]
    snum = w[0] * a[0] * (theta[0] * free[0])
    for j in range(1, w.shape[0]):
        num = num + w[j] * free[j]
        den = den + w[j]
        snum = snum + w[j] * a[j] * (theta[j] * free[j])
    valid = np.all(np.isfinite(K) & (K >= NORMAL) & np.isfinite(total) & (total >= NORMAL),
                   axis=0)
    return num / den, snum / den, valid


def explicit_rates(state, potential, control, b, topo):
    """surface_pump.explicit_rates (surface_pump.py:158-240) for held-bath worlds."""
    w = topo.cell_world
    ci, co = concentrations(state, b)
    co_c = co[:, w]
    t_c = b.temperature[w]
    bath = b.bath_potential[w]
    rt_c = R * t_c
    dvm = potential - bath
    with np.errstate(all="ignore"):
        jm = route_flux(ci, co_c, dvm, t_c, b.area, b.permeability, control.membrane)
        mu_m = rt_c * (np.log(ci) - np.log(co_c)) + VALENCE[:, None] * F * dvm
        dm = 1e-3 * np.sum(jm * mu_m, axis=0)
        s, r = topo.sender, topo.receiver
        t_e = b.temperature[topo.edge_world]
        dve = potential[s] - potential[r]
        opening = control.junction * state.junction_gate
        jj = route_flux(ci[:, s], ci[:, r], dve, t_e, b.junction_area,
                        b.junction_permeability, opening)
        mu_j = R * t_e * (np.log(ci[:, s]) - np.log(ci[:, r])) + VALENCE[:, None] * F * dve
        dj = 1e-3 * np.sum(jj * mu_j, axis=0)
    # Scatter into cells as transport() does (surface_transport.py:372-375).
    cell = -jm
    send = np.zeros_like(cell)
    np.add.at(send, (slice(None), s), -jj)
    cell = cell + send
    recv = np.zeros_like(cell)
    np.add.at(recv, (slice(None), r), jj)
    cell = cell + recv
    # Pump (kinetic_pump_binding.role_inputs: Na inside, K outside, their Δμ).
    pump = tuple(b.pump[k][w] for k in range(7))
    args = (ci[0], co_c[1], mu_m[0], mu_m[1], t_c, pump, b.pump_capacity, control.pump)
    cycles, energy, drive = pump_kinetics(*args)
    # Channel populations (surface_pump_v3.channel_rates, :937-963): the permeant species'
    # constant-field flux at the patch voltage, open fraction times availability times abundance.
    nch, idx = b.channel_slots, np.arange(b.cells)
    chan, chan_d = np.zeros((nch, b.cells)), np.zeros((nch, b.cells))
    chsum = np.zeros((3, b.cells))
    ch_ok = np.ones(b.cells, dtype=bool)
    block_ok = np.ones(b.cells, dtype=bool)
    if nch:
        opening = channel_opening(state.channel_gate, b.channel_code)
        with np.errstate(all="ignore"):
            for k in range(nch):
                sp = b.channel_species[k]
                x = VALENCE[sp] * F * dvm / (R * t_c)
                available = (opening[k] * control.channel[k]) * (
                    0.0 + (1 - 0.0) * b.channel_abundance[k])
                g = b.area * b.channel_permeability[k] * available / MOL_PER_FMOL
                flux = g * (ci[sp, idx] * bernoulli(-x) - co_c[sp, idx] * bernoulli(x))
                if getattr(b, "channel_block", None) is not None:  # surface_pump_v3.channel_rates :958-960
                    u, _, blk_ok = channel_block(b.channel_block, k, dvm, t_c)
                    flux = flux * u
                    block_ok &= blk_ok
                chan[k] = flux
                chan_d[k] = 1e-3 * flux * mu_m[sp, idx]
                chsum[sp, idx] = chsum[sp, idx] + flux
            targets, tau = channel_kinetics(dvm[None, :], b.channel_code)
        ch_ok = np.all(channel_domain(dvm[None, :], targets, tau), axis=0) & block_ok
        ch_ok &= np.all(np.isfinite(control.channel) & (control.channel >= 0)
                        & (control.channel <= 1), axis=0)
        ch_ok &= np.all(np.isfinite(chan) & np.isfinite(chan_d), axis=0)
    extra = (-STOICHIOMETRY[:, None] * cycles - 0.0) + chsum
    inflow = np.zeros((3, b.worlds))
    np.add.at(inflow, (slice(None), w), jm + extra)
    gate = gate_rhs(state.junction_gate, dve, b.gate_threshold, b.gate_minimum)
    rates = State(
        cell - extra,
        jm,
        dm,
        cycles,
        -1e-3 * cycles * energy,
        -1e-3 * cycles * drive,
        jj,
        dj,
        gate,
        -inflow,
        np.zeros(b.worlds),
        np.zeros(b.worlds),
        np.zeros(b.worlds),
        np.zeros_like(state.channel_gate),
        chan,
        chan_d,
    )
    # Validity per world (transport validity, pump and gate domains, finiteness, controls).
    ok_c = (
        np.all(np.isfinite(ci) & (ci > 0), axis=0) & np.isfinite(potential)
        & np.all(np.abs(VALENCE[:, None] * F * dvm / (R * t_c)) <= MAX_ABS_X, axis=0)
        & np.all(np.isfinite(jm), axis=0) & np.isfinite(dm)
        & pump_domain(*args)
        & np.all(np.isfinite(rates.amount_increment), axis=0)
        & np.isfinite(cycles) & np.isfinite(rates.pump_dissipated)
        & np.isfinite(rates.metabolic_work)
        & (control.membrane >= 0) & (control.membrane <= 1) & np.isfinite(control.membrane)
        & (control.pump >= 0) & (control.pump <= 1) & np.isfinite(control.pump)
        & ch_ok
    )  # fmt: skip
    ok_e = (
        np.all(np.abs(VALENCE[:, None] * F * dve / (R * t_e)) <= MAX_ABS_X, axis=0)
        & np.all(np.isfinite(jj), axis=0) & np.isfinite(dj) & np.isfinite(gate)
        & gate_domain(state.junction_gate, dve, b.gate_threshold, b.gate_minimum,
                      control.junction)
    )  # fmt: skip
    valid = np.ones(b.worlds, dtype=bool)
    np.logical_and.at(valid, w, ok_c)
    np.logical_and.at(valid, topo.edge_world, ok_e)
    valid &= np.all(np.isfinite(inflow), axis=0)
    return Rates(rates, valid, dvm)


def membrane_rate(state, control, b, topo, potential=None):
    """Gershgorin rate (1/s) of membrane charge relaxation at a stage's openings, per world
    (surface_pump_v3.membrane_rate, :4588-4660, with _patch_slopes :4534-4585): max over cells of
    F^2/RT sum z^2 P max(c) A (patch and open populations) over the cell's capacitance. With an
    open-channel block every population enters with its T_V = u G_max + |I_free| slope
    (channel_block_terms :1051-1090) at the stage's potentials, added after the patch's term."""
    if getattr(b, "channel_block", None) is not None:
        return _blocked_membrane_rate(state, control, b, topo, potential)
    w = topo.cell_world
    ci, co = concentrations(state, b)
    largest = np.maximum(ci, co[:, w])
    slope = F * F / (R * b.temperature[w])
    z2 = VALENCE[:, None] ** 2
    terms = z2 * b.permeability * largest
    passive = ((terms[0] + terms[1]) + terms[2]) * control.membrane
    membrane = passive * b.area
    extra = np.zeros(b.cells)
    nch, idx = b.channel_slots, np.arange(b.cells)
    if nch:
        open_fraction = b.channel_abundance * channel_opening(state.channel_gate, b.channel_code)
        for k in range(nch):
            sp = b.channel_species[k]
            ch = (VALENCE[sp] ** 2 * b.channel_permeability[k] * 1.0 * largest[sp, idx]) * (
                open_fraction[k] * control.channel[k])
            extra = extra + ch * b.area
    membrane = membrane + extra
    rate = slope * (0.0 + membrane) / (0.0 + b.capacitance)
    out = np.zeros(b.worlds)
    np.maximum.at(out, w, rate)
    return out


def _blocked_membrane_rate(state, control, b, topo, potential):
    w = topo.cell_world
    ci, co = concentrations(state, b)
    largest = np.maximum(ci, co[:, w])
    t_c = b.temperature[w]
    slope = F * F / (R * t_c)
    z2 = VALENCE[:, None] ** 2
    terms = z2 * b.permeability * largest
    passive = ((terms[0] + terms[1]) + terms[2]) * control.membrane
    membrane = 0.0 + passive * b.area
    dvm = potential - b.bath_potential[w]
    idx = np.arange(b.cells)
    open_fraction = b.channel_abundance * channel_opening(state.channel_gate, b.channel_code)
    blocked = np.zeros(b.cells)
    with np.errstate(all="ignore"):
        for k in range(b.channel_slots):
            sp = b.channel_species[k]
            z = VALENCE[sp]
            ch = (z ** 2 * b.channel_permeability[k] * 1.0 * largest[sp, idx]) * (
                open_fraction[k] * control.channel[k])
            g_max = F * F / (R * t_c) * (ch * b.area)
            x = z * F * dvm / (R * t_c)
            available = (channel_opening(state.channel_gate, b.channel_code)[k]
                         * control.channel[k]) * (0.0 + (1 - 0.0) * b.channel_abundance[k])
            g = b.area * b.channel_permeability[k] * available / MOL_PER_FMOL
            free = g * (ci[sp, idx] * bernoulli(-x) - co[sp, w] * bernoulli(x))
            u, s_u, _ = channel_block(b.channel_block, k, dvm, t_c)
            blocked = blocked + (u * g_max + np.abs(CHARGE_PER_FMOL * (z * free)) * s_u)
    rate = (slope * membrane + blocked) / (0.0 + b.capacitance)
    out = np.zeros(b.worlds)
    np.maximum.at(out, w, rate)
    return out


def _combine(state, dt, terms):
    """state + dt * sum(weight * rates), one term at a time (surface_pump._combine, :252-256)."""
    result = state
    for weight, rates in terms:
        result = State(*(y + (weight * dt) * d for y, d in zip(result, rates, strict=True)))
    return result


def domain_valid(state, b, topo):
    """surface_kinetic.domain_valid + surface_tissue.domain_valid for held-bath worlds."""
    ci = b.amount_reference + state.amount_increment
    ok_c = np.all(np.isfinite(ci) & (ci > 0), axis=0)
    for name in ("membrane_transferred",):
        ok_c &= np.all(np.isfinite(getattr(state, name)), axis=0)
    for name in ("membrane_dissipated", "pump_cycles", "pump_dissipated", "metabolic_work"):
        ok_c &= np.isfinite(getattr(state, name))
    ok_c &= np.all(np.where(b.permeability > 0, True, state.membrane_transferred == 0), axis=0)
    ok_c &= np.where(b.pump_capacity > 0, True, state.pump_cycles == 0)
    if b.channel_slots:
        g = state.channel_gate
        ok_c &= np.all(np.isfinite(g) & (g >= 0) & (g <= 1), axis=(0, 1))
        ok_c &= np.all(np.isfinite(state.channel_transferred), axis=0)
        ok_c &= np.all(np.isfinite(state.channel_dissipated), axis=0)
    ok_e = np.all(np.isfinite(state.junction_transferred), axis=0)
    ok_e &= np.isfinite(state.junction_dissipated) & np.isfinite(state.junction_gate)
    ok_e &= (state.junction_gate >= b.gate_minimum) & (state.junction_gate <= 1)
    ok_e &= np.all(
        np.where(b.junction_permeability > 0, True, state.junction_transferred == 0), axis=0
    )
    valid = np.ones(b.worlds, dtype=bool)
    np.logical_and.at(valid, topo.cell_world, ok_c)
    np.logical_and.at(valid, topo.edge_world, ok_e)
    for name in WORLD_FIELDS:
        v = getattr(state, name)
        valid &= np.isfinite(v) if v.ndim == 1 else np.all(np.isfinite(v), axis=0)
    return valid


def _select(valid, new, old, b, topo):
    out = []
    for field, n, o in zip(State._fields, new, old, strict=True):
        if field in CELL_FIELDS or field in CHANNEL_FIELDS:
            m = valid[topo.cell_world]
        elif field in EDGE_FIELDS:
            m = valid[topo.edge_world]
        else:
            m = valid
        out.append(np.where(m, n, o))
    return State(*out)


def ars222_step(state, dt, control, b, topo=None):
    """One ARS(2,2,2) step (surface_pump.imex_step, surface_pump.py:259-362) for every world.

    With no faces the implicit drift is zero and the operator is the capacitor matrix alone,
    so the stage potentials come from operator_potential. Returns (state, valid[W])."""
    topo = topology(b) if topo is None else topo
    w = topo.cell_world
    e_mat = np.array([[0.0, 0.0, 0.0], [GAMMA, 0.0, 0.0], [DELTA, 1.0 - DELTA, 0.0]])
    bath = b.bath_potential[w]
    nch = b.channel_slots
    charge0 = node_charge(state, b)
    start = capacitor_potential(charge0, b, topo)
    k0 = explicit_rates(state, start, control, b, topo)
    valid = k0.valid.copy()
    # The explicit-stability refusal at each explicit stage (surface_pump_v3.py:3668-3670).
    valid &= dt * membrane_rate(state, control, b, topo, start) <= EXPLICIT_STEP_BOUND
    zero = State(*(np.zeros_like(v) for v in state))
    zero = zero._replace(reservoir_supplied=-zero.reservoir_supplied)  # implicit_rates' -0.0
    rows = gate_rows_active(b.channel_code)
    if nch:  # The start's kinetics (readouts at the start potentials).
        start_kin = channel_kinetics((start - bath)[None, :], b.channel_code)

    def stage_gates(potential, fraction):
        """surface_pump_v3.stage_gates (:3061-3070): exponential update from the step start."""
        kin = channel_kinetics((potential - bath)[None, :], b.channel_code)
        moved = advance_gates(state.channel_gate, start_kin[0], start_kin[1], kin[0], kin[1],
                              fraction * dt)
        ok = np.all(channel_domain((potential - bath)[None, :], *kin), axis=0)
        return np.where(rows, moved, state.channel_gate), ok

    # Stage 1.
    known = _combine(state, dt, [(e_mat[1, 0], k0.state)])
    charge = node_charge(known, b)
    potential, residual = operator_potential(charge, b, topo)
    scale = np.maximum(np.abs(charge), np.abs(b.capacitance * potential
                                               + (-b.capacitance) * b.bath_potential[w]))
    ok = np.isfinite(potential) & (np.abs(residual) <= CHARGE_ATOL_C + CHARGE_RTOL * scale)
    np.logical_and.at(valid, w, ok)
    stage = _combine(known, dt, [(GAMMA, zero)])
    if nch:
        with np.errstate(all="ignore"):
            gate, ok = stage_gates(potential, np.sum(e_mat[1]))
        stage = stage._replace(channel_gate=gate)
        np.logical_and.at(valid, w, ok)
    k1 = explicit_rates(stage, potential, control, b, topo)
    valid &= k1.valid
    valid &= dt * membrane_rate(stage, control, b, topo, potential) <= EXPLICIT_STEP_BOUND
    # Stage 2 (the last): explicit weights delta, 1 - delta; implicit 1 - gamma, gamma (zeros).
    known = _combine(state, dt, [(e_mat[2, 0], k0.state), (e_mat[2, 1], k1.state),
                                 (1.0 - GAMMA, zero)])
    charge = node_charge(known, b)
    potential, residual = operator_potential(charge, b, topo)
    scale = np.maximum(np.abs(charge), np.abs(b.capacitance * potential
                                               + (-b.capacitance) * b.bath_potential[w]))
    ok = np.isfinite(potential) & (np.abs(residual) <= CHARGE_ATOL_C + CHARGE_RTOL * scale)
    np.logical_and.at(valid, w, ok)
    stage = _combine(known, dt, [(GAMMA, zero)])
    if nch:
        with np.errstate(all="ignore"):
            gate, ok = stage_gates(potential, np.sum(e_mat[2]))
        stage = stage._replace(channel_gate=gate)
        np.logical_and.at(valid, w, ok)
    # Ledger bookings of the step (surface_pump.py:338-355).
    applied = (0 + e_mat[2, 0] * k0.state.reservoir_supplied) + e_mat[2, 1] * k1.state.reservoir_supplied
    applied = applied + ((0 + (1.0 - GAMMA) * zero.reservoir_supplied) + GAMMA * zero.reservoir_supplied)
    electrode = capacitor_plate_sum(stage, b, topo) - capacitor_plate_sum(state, b, topo)
    co = b.bath_amount / b.bath_volume
    mu = R * b.temperature * np.log(co) + VALENCE[:, None] * F * b.bath_potential
    stage = stage._replace(
        electrode_charge=state.electrode_charge + electrode,
        reservoir_work=state.reservoir_work + 1e-3 * np.sum(mu * (dt * applied), axis=0),
        electrode_work=state.electrode_work + 1e12 * b.bath_potential * electrode,
    )
    valid &= domain_valid(stage, b, topo)
    return _select(valid, stage, state, b, topo), valid


def readout_rates(state, control, b, topo):
    """surface_kinetic.readouts' derivative (surface_kinetic.py:221-410): the explicit rates
    at the capacitor potentials plus the electrode current and the work rates."""
    w = topo.cell_world
    potential = capacitor_potential(node_charge(state, b), b, topo)
    r = explicit_rates(state, potential, control, b, topo)
    # dphi = capacitor solve of qdot; the bath's electrode current is (C dphi) at its row.
    qdot = CHARGE_PER_FMOL * np.sum(VALENCE[:, None] * r.state.amount_increment, axis=0)
    scale = topo.capacitor_scale[w]
    factor = np.sqrt(b.capacitance / scale)
    dphi = qdot / scale / factor / factor
    electrode = np.zeros(b.worlds)
    np.add.at(electrode, w, -b.capacitance * dphi)
    co = b.bath_amount / b.bath_volume
    mu = R * b.temperature * np.log(co) + VALENCE[:, None] * F * b.bath_potential
    if b.channel_slots:  # readouts' gate rate, (target - g)/tau (surface_kinetic.py:237)
        targets, tau = channel_kinetics((potential - b.bath_potential[w])[None, :],
                                        b.channel_code)
        rate = np.where(gate_rows_active(b.channel_code),
                        (targets - state.channel_gate) / tau, 0.0)
        r = r._replace(state=r.state._replace(channel_gate=rate))
    d = r.state._replace(
        electrode_charge=electrode,
        reservoir_work=1e-3 * np.sum(mu * r.state.reservoir_supplied, axis=0),
        electrode_work=1e12 * b.bath_potential * electrode,
    )
    return d, r.valid


def rk4_step(state, dt, control, b, topo=None):
    """fixed_step.rk4_checked_step (:25-71) over readout_rates."""
    topo = topology(b) if topo is None else topo

    def inc(k, f):
        return State(*(y + f * dt * dy for y, dy in zip(state, k, strict=True)))

    k1, a = readout_rates(state, control, b, topo)
    k2, bb = readout_rates(inc(k1, 0.5), control, b, topo)
    k3, c = readout_rates(inc(k2, 0.5), control, b, topo)
    k4, d = readout_rates(inc(k3, 1.0), control, b, topo)
    new = State(*(
        y + (dt / 6.0) * (p + 2.0 * q + 2.0 * r + s)
        for y, p, q, r, s in zip(state, k1, k2, k3, k4, strict=True)
    ))  # fmt: skip
    ok = a & bb & c & d & domain_valid(new, b, topo)
    return _select(ok, new, state, b, topo), ok


def membrane_voltage(state, b, topo=None):
    topo = topology(b) if topo is None else topo
    v = capacitor_potential(node_charge(state, b), b, topo)
    return v - b.bath_potential[topo.cell_world]


# ---------------------------------------------------------------------------------------------
# Ledgers (the reference's balances(), held-bath worlds)


def balances(state, b, topo=None):
    """Per-world conservation residuals (surface_tissue.balances, :536-611, with the pump and
    junction terms of surface_kinetic.balances, :470-482). Returns a dict of arrays."""
    topo = topology(b) if topo is None else topo
    w = topo.cell_world
    di = state.amount_increment
    moved = state.membrane_transferred
    if b.channel_slots:  # channel_to_membrane (surface_kinetic.py:197-207)
        moved = moved.copy()
        idx = np.arange(b.cells)
        for k in range(b.channel_slots):
            moved[b.channel_species[k], idx] += state.channel_transferred[k]
    total_m = moved - STOICHIOMETRY[:, None] * state.pump_cycles
    local = di + total_m
    send = np.zeros_like(di)
    np.add.at(send, (slice(None), topo.sender), state.junction_transferred)
    recv = np.zeros_like(di)
    np.add.at(recv, (slice(None), topo.receiver), state.junction_transferred)
    local = local + send - recv
    per_world_di = np.zeros((3, b.worlds))
    np.add.at(per_world_di, (slice(None), w), di)
    # Held bath: its increment stays zero; what crossed its patches is supplied.
    outside_moved = np.zeros((3, b.worlds))
    np.add.at(outside_moved, (slice(None), w), total_m)
    outside = -outside_moved - state.reservoir_supplied
    total = per_world_di - state.reservoir_supplied
    cap = capacitor_plate_sum(state, b, topo)
    electrode = state.electrode_charge - cap
    supply_charge = CHARGE_PER_FMOL * np.sum(VALENCE[:, None] * state.reservoir_supplied, axis=0)
    global_charge = state.electrode_charge + supply_charge
    co = b.bath_amount / b.bath_volume
    mu = R * b.temperature * np.log(co) + VALENCE[:, None] * F * b.bath_potential
    reservoir_work = state.reservoir_work - 1e-3 * np.sum(mu * state.reservoir_supplied, axis=0)
    electrode_work = state.electrode_work - 1e12 * b.bath_potential * state.electrode_charge
    drive = chemical_drive(tuple(b.pump[k][w] for k in range(7)), b.temperature[w])
    metabolic = state.metabolic_work + 1e-3 * drive * state.pump_cycles
    return dict(
        local=local, outside=outside, total=total, electrode=electrode,
        global_charge=global_charge, reservoir_work=reservoir_work,
        electrode_work=electrode_work, metabolic_work=metabolic,
    )  # fmt: skip
