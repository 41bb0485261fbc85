"""CPU oracle of the N2 step: ARS(2,2,2) with the membranes', channels' and junctions' slope
conductances implicit (cells.solver.imex_ars222_implicit_conductances@1), for held-bath worlds.

TEST INFRASTRUCTURE ONLY, like oracle/tissue.py: only tests/, __graft_entry__.smoke() and
bench.py's CPU legs may import it; the product path never calls it.

What it restates (paths inside the reference project), for worlds whose every cell has one patch
facing the world's held bath, with no faces and no declared kinds (structure None):

* models/surface_pump_v3.py:3547-3955 imex_step under an N2 ID: the step start's readouts; the
  operator-time prediction of the amounts, channel gates and junction gates at half the step and
  its field (operator_time_conductances, :2961-3029); the frozen slopes dJ/d(dv) of every patch,
  channel population and junction (conductance_weights, route_slope, :2741-2813, with the
  reference's bernoulli_slope, laws/routes/patch_electrodiffusion.py:43-54); their Laplacian beside
  the capacitors, C + gamma dt L (conductance_laplacian :2816-2841, numerics/surface_imex.py
  factor_operator :207-225 on the dense node space of the world's cells and its bath, the bath
  clamped); the explicit remainders J - W dv (explicit_remainder :2925-2946, with the junction
  gates' rate zero); the implicit linear fluxes W dv at each stage's potentials with their heat at
  the stage (implicit_rates :2659-2700, implicit_route_heat :2949-2958); the channel gates and the
  junction gates by their exponential updates (stage_gates, stage_junction_gates :3130-3156);
  the ledger bookings of surface_pump.imex_step;
* the dense Cholesky solve of surface_field.cholesky_solve (:577-593) and
  surface_imex.solve_operator (:269-278), in their arithmetic order, one world at a time.

Under N2 the stage stability rule counts only declared kinds' terms (membrane_rate,
explicit_only), so these worlds have none.

Pinned: tests/golden/make_golden.py runs the reference's own N2 step (@3 on its xp=np branch)
on seeded worlds; tests/test_oracle_n2.py checks this restatement against them.
"""

from __future__ import annotations

import numpy as np

from oracle import tissue as T

F, R = T.F, T.R
VALENCE = T.VALENCE
MOL_PER_FMOL = T.MOL_PER_FMOL
CHARGE_PER_FMOL = T.CHARGE_PER_FMOL
GAMMA, DELTA = T.GAMMA, T.DELTA
N2_ID = "cells.solver.imex_ars222_implicit_conductances@1"
OPERATOR_TIME = 0.5  # the routes' operator time (surface_imex.TABLEAUX[N2_ID].operator_time[1])
SLOPE_SERIES_BELOW = 1e-3  # laws/routes/patch_electrodiffusion.py:40


def bernoulli_slope(x):
    """B'(x), the reference's form (patch_electrodiffusion.bernoulli_slope): the series
    -1/2 + x/6 - x^3/180 below |x| < 1e-3, otherwise e^-|x| forms of (e^x - 1 - x e^x)/(e^x-1)^2."""
    x = np.asarray(x, dtype=float)
    small = np.abs(x) < SLOPE_SERIES_BELOW
    pos = x > 0
    xs = np.where(small, 1.0, x)
    em = np.exp(-np.abs(xs))
    with np.errstate(all="ignore"):
        pos_form = (em * (1.0 - xs) - em * em) / (1.0 - em) ** 2
        neg_form = (em - 1.0 - xs * em) / (em - 1.0) ** 2
    regular = np.where(pos, pos_form, neg_form)
    series = -0.5 + x / 6.0 - x**3 / 180.0
    return np.where(small, series, regular)


def route_slope(c_from, c_to, dv, valence, temperature, area, permeability, available):
    """dJ/d(dv) of the constant-field route flux (fmol/s per V, sender -> receiver)."""
    k = valence * F / (R * temperature)
    x = k * dv
    prefactor = area * permeability * available / MOL_PER_FMOL
    return prefactor * k * (-c_from * bernoulli_slope(-x) - c_to * bernoulli_slope(x))


def junction_kinetics(voltage, threshold, minimum):
    """junction_voltage_relaxation.kinetics (:41-60): (target, relaxation rate 1/s)."""
    shift = np.abs(voltage) - threshold
    alpha = 1.3 * np.exp(-77.0 * shift)
    log_beta = np.log(0.065) + 140.0 * shift
    beta = 20.0 * np.exp(-np.logaddexp(0.0, -log_beta))
    relaxation = alpha + beta
    return (alpha + beta * minimum) / relaxation, relaxation


def conductance_weights(state, potential, control, b, topo):
    """(W_membrane [S, C], W_channel [NCH, C] for each population's permeant species,
    W_junction [S, E]) at a state and node potentials (conductance_weights, :2758-2813)."""
    w = topo.cell_world
    ci, co = T.concentrations(state, b)
    co_c = co[:, w]
    t_c = b.temperature[w]
    dv = potential - b.bath_potential[w]
    z = VALENCE[:, None]
    with np.errstate(all="ignore"):
        membrane = route_slope(ci, co_c, dv, z, t_c, b.area, b.permeability, control.membrane)
        nch, idx = b.channel_slots, np.arange(b.cells)
        channel = np.zeros((nch, b.cells))
        if nch:
            opening = T.channel_opening(state.channel_gate, b.channel_code)
            for k in range(nch):
                sp = b.channel_species[k]
                available = b.channel_abundance[k] * opening[k] * control.channel[k]
                channel[k] = route_slope(ci[sp, idx], co_c[sp, idx], dv, VALENCE[sp], t_c, b.area,
                                         b.channel_permeability[k] * 1.0, available)
        s, r = topo.sender, topo.receiver
        t_e = b.temperature[topo.edge_world]
        junction = route_slope(ci[:, s], ci[:, r], potential[s] - potential[r], z, t_e,
                               b.junction_area, b.junction_permeability,
                               control.junction * state.junction_gate)
    return membrane, channel, junction


def patch_conductance(weights, b):
    """(G_patch [C], G_junction [E]) in S: CHARGE_PER_FMOL sum_s z_s W_s (species in order), a
    patch's channels added into it in slot order (conductance_laplacian, :2816-2841)."""
    membrane, channel, junction = weights
    zw = VALENCE[:, None] * membrane
    g_patch = CHARGE_PER_FMOL * ((zw[0] + zw[1]) + zw[2])
    if b.channel_slots:
        extra = np.zeros(b.cells)
        for k in range(b.channel_slots):
            sp = b.channel_species[k]
            # species_sum over [S] with only the permeant species non-zero.
            terms = np.zeros((3, b.cells))
            terms[sp, np.arange(b.cells)] = VALENCE[sp] * channel[k]
            extra = extra + CHARGE_PER_FMOL * ((terms[0] + terms[1]) + terms[2])
        g_patch = g_patch + extra
    zj = VALENCE[:, None] * junction
    g_junction = CHARGE_PER_FMOL * ((zj[0] + zj[1]) + zj[2])
    return g_patch, g_junction


class Operator:
    """Per-world dense operator (C + gamma dt L on the world's cells and its bath, the bath
    clamped), its Jacobi scale and lower Cholesky factor (surface_imex.factor_operator)."""

    def __init__(self, g_patch, g_junction, coefficient, b, topo):
        self.worlds = []
        self.valid = np.ones(b.worlds, dtype=bool)
        for w in range(b.worlds):
            c0, c1 = b.cell_offset[w], b.cell_offset[w + 1]
            e0, e1 = b.edge_offset[w], b.edge_offset[w + 1]
            n = c1 - c0
            size = n + 1
            cap = np.zeros((size, size))
            for i in range(n):  # surface_field.bind's membrane loop
                c = b.capacitance[c0 + i]
                cap[i, i] += c
                cap[n, n] += c
                cap[i, n] -= c
                cap[n, i] -= c

            def block(g, a, bb):
                parts = []
                for key in ((a, a), (bb, bb), (a, bb), (bb, a)):
                    m = np.zeros((size, size))
                    np.add.at(m, key, g)
                    parts.append(m)
                return ((parts[0] + parts[1]) - parts[2]) - parts[3]

            cells = np.arange(n)
            lap = block(g_patch[c0:c1], cells, np.full(n, n)) + block(
                g_junction[e0:e1], b.sender[e0:e1].astype(np.int64),
                b.receiver[e0:e1].astype(np.int64))
            matrix = cap + coefficient * lap
            free = np.r_[np.ones(n, dtype=bool), False]
            held = np.r_[np.zeros(n), b.bath_potential[w]]
            diagonal = np.where(free, np.diagonal(matrix), 1.0)
            scale = 1.0 / np.sqrt(np.where(diagonal > 0, diagonal, 1.0))
            reduced = np.where(free[:, None] & free[None, :],
                               matrix * scale[:, None] * scale[None, :], 0.0)
            reduced += np.diag((~free).astype(float))
            with np.errstate(all="ignore"):
                try:
                    factor = np.linalg.cholesky(reduced)
                    ok = True
                except np.linalg.LinAlgError:
                    factor, ok = np.full_like(reduced, np.nan), False
            self.valid[w] = ok and np.all(diagonal > 0) and np.all(np.isfinite(factor))
            self.worlds.append((matrix, scale, factor, free, held))

    def solve(self, charge, b):
        """Stage potentials [C], their charge residual [C] and residual scale [C]
        (surface_imex.solve_operator with surface_field.cholesky_solve)."""
        potential = np.zeros(b.cells)
        residual = np.zeros(b.cells)
        scale_out = np.zeros(b.cells)
        for w, (matrix, scale, factor, free, held) in enumerate(self.worlds):
            c0, c1 = b.cell_offset[w], b.cell_offset[w + 1]
            q = np.r_[charge[c0:c1], 0.0]  # the clamped bath's row never enters
            rhs = np.where(free, (q - matrix @ held) * scale, 0.0)
            phi = np.where(free, cholesky_solve(factor, rhs) * scale, held)
            product = matrix @ phi
            residual[c0:c1] = np.where(free, product - q, 0.0)[:-1]
            potential[c0:c1] = phi[:-1]
            scale_out[c0:c1] = np.maximum(np.abs(q), np.abs(product))[:-1]
        return potential, residual, scale_out


def cholesky_solve(factor, rhs):
    """L L^T x = rhs by blocked substitution in 64-row blocks (surface_field.cholesky_solve's
    NumPy branch, in its order)."""
    lower, upper = np.asarray(factor), np.ascontiguousarray(np.asarray(factor).T)
    y = np.array(rhs, dtype=float, copy=True)
    starts = range(0, len(y), 64)
    with np.errstate(all="ignore"):
        for start in starts:
            stop = start + 64
            part = y[start:stop] - lower[start:stop, :start] @ y[:start]
            y[start:stop] = np.linalg.solve(lower[start:stop, start:stop], part)
        for start in reversed(starts):
            stop = start + 64
            part = y[start:stop] - upper[start:stop, stop:] @ y[stop:]
            y[start:stop] = np.linalg.solve(upper[start:stop, start:stop], part)
    return y


def linear_fluxes(weights, potential, b, topo):
    """W dv of every route at the node potentials: (membrane [S, C], channel [NCH, C],
    junction [S, E]) (linear_route_fluxes, :2844-2860)."""
    membrane, channel, junction = weights
    dv = potential - b.bath_potential[topo.cell_world]
    dj = potential[topo.sender] - potential[topo.receiver]
    return membrane * dv, channel * dv, junction * dj


def route_rates(membrane, channel, junction, b, topo):
    """(cells [S, C], bath inflow [S, W]) of route fluxes (route_amount_rates, :2863-2877)."""
    patches = membrane.copy()
    idx = np.arange(b.cells)
    for k in range(b.channel_slots):  # channel_to_membrane: each population onto its patch
        add = np.zeros((3, b.cells))
        add[b.channel_species[k], idx] = channel[k]
        patches = patches + add
    cells_recv = np.zeros((3, b.cells))
    np.add.at(cells_recv, (slice(None), topo.receiver), junction)
    cells_send = np.zeros((3, b.cells))
    np.add.at(cells_send, (slice(None), topo.sender), junction)
    cells_patch = np.zeros((3, b.cells))
    np.add.at(cells_patch, (slice(None), idx), patches)
    cells = (cells_recv - cells_send) - cells_patch
    outside = np.zeros((3, b.worlds))
    np.add.at(outside, (slice(None), topo.cell_world), patches)
    return cells, outside


def delta_mu(state, potential, b, topo):
    """(membrane [S, C], junction [S, E]) electrochemical differences (route_delta_mu)."""
    w = topo.cell_world
    ci, co = T.concentrations(state, b)
    rt = R * b.temperature[w]
    z = VALENCE[:, None]
    dv = potential - b.bath_potential[w]
    with np.errstate(all="ignore"):
        mu_m = rt * (np.log(ci) - np.log(co[:, w])) + z * F * dv
        s, r = topo.sender, topo.receiver
        rte = R * b.temperature[topo.edge_world]
        mu_j = rte * (np.log(ci[:, s]) - np.log(ci[:, r])) + z * F * (potential[s] - potential[r])
    return mu_m, mu_j


def heat_rates(membrane, channel, junction, mu_m, mu_j, b):
    """route_heat_rates (:2900-2910): (membrane [C], channel [NCH, C], junction [E]) pJ/s."""
    hm = membrane * mu_m
    hj = junction * mu_j
    idx = np.arange(b.cells)
    hc = np.zeros((b.channel_slots, b.cells))
    for k in range(b.channel_slots):
        hc[k] = 1e-3 * channel[k] * mu_m[b.channel_species[k], idx]
    return 1e-3 * ((hm[0] + hm[1]) + hm[2]), hc, 1e-3 * ((hj[0] + hj[1]) + hj[2])


def remainder(rates, weights, potential, state, b, topo):
    """explicit_remainder (:2925-2946): the rates less the routes' linear parts at these
    potentials, the junction gates' rate zero ((a))."""
    membrane, channel, junction = linear_fluxes(weights, potential, b, topo)
    cells, outside = route_rates(membrane, channel, junction, b, topo)
    mu_m, mu_j = delta_mu(state, potential, b, topo)
    hm, hc, hj = heat_rates(membrane, channel, junction, mu_m, mu_j, b)
    return rates._replace(
        amount_increment=rates.amount_increment - cells,
        reservoir_supplied=rates.reservoir_supplied - (-outside),
        membrane_transferred=rates.membrane_transferred - membrane,
        junction_transferred=rates.junction_transferred - junction,
        channel_transferred=rates.channel_transferred - channel,
        membrane_dissipated=rates.membrane_dissipated - hm,
        junction_dissipated=rates.junction_dissipated - hj,
        channel_dissipated=rates.channel_dissipated - hc,
        junction_gate=np.zeros_like(rates.junction_gate),
    )


def implicit(weights, potential, state, b, topo):
    """implicit_rates under N2 (:2659-2700): the routes' linear parts at the stage potentials,
    heat zero (set at the stage by implicit_heat)."""
    membrane, channel, junction = linear_fluxes(weights, potential, b, topo)
    cells, outside = route_rates(membrane, channel, junction, b, topo)
    zero = T.State(*(np.zeros_like(v) for v in state))
    return zero._replace(
        amount_increment=cells,
        membrane_transferred=membrane,
        junction_transferred=junction,
        reservoir_supplied=-outside,
        channel_transferred=channel,
    )


def implicit_heat(drift, stage, potential, b, topo):
    """implicit_route_heat (:2949-2958): the linear parts' heat at the stage's concentrations
    and potentials."""
    mu_m, mu_j = delta_mu(stage, potential, b, topo)
    hm, hc, hj = heat_rates(drift.membrane_transferred, drift.channel_transferred,
                            drift.junction_transferred, mu_m, mu_j, b)
    return drift._replace(membrane_dissipated=hm, junction_dissipated=hj, channel_dissipated=hc)


def junction_gates(gate, start, potential, fraction_dt, availability, b, topo):
    """stage_junction_gates (:3130-3156): the exponential update from the start's kinetics to the
    stage's, and the law's domain at the stage per junction."""
    voltage = potential[topo.sender] - potential[topo.receiver]
    target, relaxation = junction_kinetics(voltage, b.gate_threshold, b.gate_minimum)
    with np.errstate(all="ignore"):
        moved = T.advance_gates(gate, start[0], 1.0 / start[1], target, 1.0 / relaxation,
                                fraction_dt)
    ok = T.gate_domain(moved, voltage, b.gate_threshold, b.gate_minimum, availability)
    return moved, ok


def n2_step(state, dt, control, b, topo=None):
    """One N2 step for every world; returns (state, valid[W])."""
    topo = T.topology(b) if topo is None else topo
    w = topo.cell_world
    bath = b.bath_potential[w]
    nch = b.channel_slots
    e_mat = np.array([[0.0, 0.0, 0.0], [GAMMA, 0.0, 0.0], [DELTA, 1.0 - DELTA, 0.0]])
    i_mat = np.array([[0.0, 0.0, 0.0], [0.0, GAMMA, 0.0], [0.0, 1.0 - GAMMA, GAMMA]])
    # The step start (readouts): potentials, whole rates, the channels' and junctions' kinetics.
    start = T.capacitor_potential(T.node_charge(state, b), b, topo)
    whole = T.explicit_rates(state, start, control, b, topo)
    valid = whole.valid.copy()
    rows = T.gate_rows_active(b.channel_code)
    with np.errstate(all="ignore"):
        if nch:
            start_kin = T.channel_kinetics((start - bath)[None, :], b.channel_code)
        start_junction = junction_kinetics(start[topo.sender] - start[topo.receiver],
                                           b.gate_threshold, b.gate_minimum)
        # The operator-time prediction (operator_time_conductances).
        theta = OPERATOR_TIME * dt
        ahead_gate = state.channel_gate
        if nch:
            moved = T.advance_gates(state.channel_gate, start_kin[0], start_kin[1], start_kin[0],
                                    start_kin[1], theta)
            ahead_gate = np.where(rows, moved, state.channel_gate)
        target, relaxation = start_junction
        ahead_junction = state.junction_gate + (target - state.junction_gate) * -np.expm1(
            -relaxation * theta)
        ahead = state._replace(
            amount_increment=state.amount_increment + theta * whole.state.amount_increment,
            channel_gate=ahead_gate, junction_gate=ahead_junction)
        ci, _ = T.concentrations(ahead, b)
        ok_c = np.all(np.isfinite(ci) & (ci > 0), axis=0)
        ahead_potential = T.capacitor_potential(T.node_charge(ahead, b), b, topo)
        ok_c &= np.isfinite(ahead_potential)
        weights = conductance_weights(ahead, ahead_potential, control, b, topo)
        ok_c &= np.all(np.isfinite(weights[0]), axis=0) & np.all(np.isfinite(weights[1]), axis=0)
        ok_e = np.all(np.isfinite(weights[2]), axis=0)
    np.logical_and.at(valid, w, ok_c)
    np.logical_and.at(valid, topo.edge_world, ok_e)
    g_patch, g_junction = patch_conductance(weights, b)
    operator = Operator(g_patch, g_junction, i_mat[-1, -1] * dt, b, topo)
    valid &= operator.valid
    k0 = remainder(whole.state, weights, start, state, b, topo)
    explicit, drifts = [k0], [None]
    potential, stage = start, state
    for i in (1, 2):
        terms = [(e_mat[i, j], explicit[j]) for j in range(i)]
        terms += [(i_mat[i, j], drifts[j]) for j in range(1, i)]
        known = T._combine(state, dt, terms)
        charge = T.node_charge(known, b)
        with np.errstate(all="ignore"):
            potential, residual, scale = operator.solve(charge, b)
        ok = np.isfinite(potential) & (np.abs(residual) <= T.CHARGE_ATOL_C + T.CHARGE_RTOL * scale)
        np.logical_and.at(valid, w, ok)
        drift = implicit(weights, potential, state, b, topo)
        stage = T._combine(known, dt, [(i_mat[i, i], drift)])
        with np.errstate(all="ignore"):
            drift = implicit_heat(drift, stage, potential, b, topo)
        drifts.append(drift)
        stage = T._combine(known, dt, [(i_mat[i, i], drift)])
        fraction = float(np.sum(e_mat[i]))
        if nch:
            with np.errstate(all="ignore"):
                kin = T.channel_kinetics((potential - bath)[None, :], b.channel_code)
                moved = T.advance_gates(state.channel_gate, start_kin[0], start_kin[1], kin[0],
                                        kin[1], fraction * dt)
            ok = np.all(T.channel_domain((potential - bath)[None, :], *kin), axis=0)
            stage = stage._replace(channel_gate=np.where(rows, moved, state.channel_gate))
            np.logical_and.at(valid, w, ok)
        with np.errstate(all="ignore"):
            moved, ok = junction_gates(state.junction_gate, start_junction, potential,
                                       fraction * dt, control.junction, b, topo)
        stage = stage._replace(junction_gate=moved)
        np.logical_and.at(valid, topo.edge_world, ok)
        if i < 2:
            rates = T.explicit_rates(stage, potential, control, b, topo)
            valid &= rates.valid
            explicit.append(remainder(rates.state, weights, potential, stage, b, topo))
    # Ledger bookings (surface_pump.imex_step's, as oracle.tissue.ars222_step).
    applied = sum(e_mat[2, j] * explicit[j].reservoir_supplied for j in range(2))
    applied = applied + sum(i_mat[2, j] * drifts[j].reservoir_supplied for j in (1, 2))
    electrode = T.capacitor_plate_sum(stage, b, topo) - T.capacitor_plate_sum(state, b, topo)
    co = b.bath_amount / b.bath_volume
    mu = R * b.temperature * np.log(co) + VALENCE[:, None] * F * b.bath_potential
    stage = stage._replace(
        electrode_charge=state.electrode_charge + electrode,
        reservoir_work=state.reservoir_work + 1e-3 * np.sum(mu * (dt * applied), axis=0),
        electrode_work=state.electrode_work + 1e12 * b.bath_potential * electrode,
    )
    valid &= T.domain_valid(stage, b, topo)
    return T._select(valid, stage, state, b, topo), valid
