"""CPU oracle of the step's reverse-mode derivative: the discrete adjoint of oracle.tissue's
ARS(2,2,2) step, and loss gradients through a trajectory.

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline leg may import this module; the product path (``cells_b200``) never calls it.

What it differentiates. The reference differentiates this path only forward, by ``jax.jvp`` /
``jax.jacfwd`` of the step (src/cells/analysis/stationary.py:505-514); a loss gradient of a
trajectory would be ``jax.grad`` of the composed steps, i.e. the transposed linearisation of each
step applied in reverse order. This module writes that transposed linearisation by hand for the
held-bath step of oracle.tissue.ars222_step (models/surface_pump.py:259-362):

* the dynamic state is the amount increments n [S, C], the junction gates g [E] and the channel
  gates [2, NCH, C]; the ledgers (transferred, dissipated, cycles, works, reservoir, electrode)
  never feed back into the dynamics, so their cotangents do not enter the parameters' gradients;
* a stage's potential is the capacitor closure V = (Q0 + F sum_s z_s n_s) / C + V_bath, a diagonal
  (self-adjoint) map, so the transposed stage solve is the same diagonal;
* each explicit stage rate is differentiated term by term: the constant-field flux through B(x)
  and its slope B'(x) (the reference's bernoulli_slope, laws/routes/patch_electrodiffusion.py:
  43-54, restated from B(x) = x / (e^x - 1)), the Na/K-ATPase of
  laws/pumps/nak_atp_mass_action_positive.py:63-98 (its magnitude-departure product is
  -M expm1(a) on both branches), the junction gate law of junction_voltage_relaxation.py:43-67,
  the channel laws and openings, and the exponential stage gates of
  numerics/exponential_gates.py:36-51;
* a step a world refused is the identity for that world (its state did not move) and adds
  nothing to the gradients.

Pinned by central finite differences of oracle.tissue.ars222_step (tests/test_oracle_adjoint.py),
which is itself pinned bit for bit to the reference's step.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np

from oracle import tissue as T

F, R = T.F, T.R
VALENCE = T.VALENCE
MOL_PER_FMOL = T.MOL_PER_FMOL
CHARGE_PER_FMOL = T.CHARGE_PER_FMOL


def sigmoid(u):
    e = np.exp(-np.abs(u))
    return np.where(u >= 0, 1.0 / (1.0 + e), e / (1.0 + e))


def bernoulli_slope(x):
    """B'(x) for B(x) = x / expm1(x). Away from 0, with em = expm1(-|x|):
    x > 0: -(1 + em)(x + em) / em^2;  x < 0: (em + |x| (1 + em)) / em^2.
    Below |x| < 1e-2 the Taylor series -1/2 + x/6 - x^3/180 + x^5/5040 - x^7/151200 (from the
    Bernoulli numbers B_1..B_8)."""
    x = np.asarray(x, dtype=float)
    small = np.abs(x) < 1e-2
    ax = np.where(small, 1.0, np.abs(x))
    em = np.expm1(-ax)
    pos = -(1.0 + em) * (ax + em) / (em * em)
    neg = (em + ax * (1.0 + em)) / (em * em)
    x2 = x * x
    series = -0.5 + x * (1.0 / 6.0 + x2 * (-1.0 / 180.0 + x2 * (1.0 / 5040.0 - x2 / 151200.0)))
    return np.where(small, series, np.where(x > 0, pos, neg))


def channel_kinetics_slope(v, code):
    """Voltage derivatives of the channel laws' targets and time constants, [2, NCH, C] each
    (the laws of oracle.tissue.channel_kinetics)."""
    v = np.broadcast_to(v, code.shape)
    dt = np.zeros((2, *code.shape))
    dtau = np.zeros((2, *code.shape))
    B, dB = T.bernoulli, bernoulli_slope
    with np.errstate(all="ignore"):
        # NaV1.2 (laws/channels/nav1p2_m3h_regularized.py:22-44).
        sh = (v + 0.025) / 0.009
        act, dact = 0.182 * 9 * B(-sh), -0.182 * 9 * dB(-sh) / 0.009
        deact, ddeact = 0.124 * 9 * B(sh), 0.124 * 9 * dB(sh) / 0.009
        ur = -(v + 0.040) / 0.005
        rec, drec = 0.024 * 5 * B(ur), -0.024 * 5 * dB(ur) / 0.005
        ui = (v + 0.065000123) / 0.005
        ina, dina = 0.0091 * 5 * B(ui), 0.0091 * 5 * dB(ui) / 0.005
        s, ds = act + deact, dact + ddeact
        t1 = 1 / (1 + np.exp((v + 0.055) / 0.0062))
        q, dq = rec + ina, drec + dina
        nav = (np.stack(((dact * s - act * ds) / (s * s), -t1 * (1 - t1) / 0.0062)),
               np.stack((-0.001 * ds / (s * s), -0.001 * dq / (q * q))))
        # Hodgkin-Huxley K n^4 (alpha_n = 0.1 B(-(Vm + 55)/10) per ms, beta_n, Vm in mV).
        ua = -(1000.0 * v + 55.0) / 10.0
        alpha, dalpha = 100.0 * B(ua), -100.0 * 100.0 * dB(ua)
        beta = 125.0 * np.exp(-(1000.0 * v + 65.0) / 80.0)
        dbeta = -12.5 * beta
        s, ds = alpha + beta, dalpha + dbeta
        zero = np.zeros_like(v)
        hh = (np.stack(((dalpha * beta - alpha * dbeta) / (s * s), zero)),
              np.stack((-ds / (s * s), zero)))
        # Kv1.5 (laws/channels/kv1p5_mh.py:29-41).
        s0 = sigmoid((v + 0.0060) / 0.0064)
        s1 = sigmoid(-(v + 0.0253) / 0.0035)
        kv = (np.stack((s0 * (1 - s0) / 0.0064, -s1 * (1 - s1) / 0.0035)),
              np.stack((np.full_like(v, -0.1163), np.full_like(v, -15.5))))
    for law, (a, b) in ((T.NAV1P2, nav), (T.HH_K_N4, hh), (T.KV1P5, kv)):
        mask = (code == law)[None]
        dt = np.where(mask, a, dt)
        dtau = np.where(mask, b, dtau)
    return dt, dtau


def opening_partials(gate, code):
    """d opening / d m and d opening / d h, [NCH, C] each."""
    m, h = gate[0], gate[1]
    nav = code == T.NAV1P2
    hh = code == T.HH_K_N4
    dm = np.where(nav, 3 * m * m * h, np.where(hh, 4 * m * m * m, h))
    dh = np.where(nav, m * m * m, np.where(hh, 0.0, m))
    return dm, dh


def advance_partials(g, ts, taus, te, taue, h):
    """Partials of advance_gates' g + (ts - g)(1 - e^-z) + (te - ts) lag(z),
    z = h (1/taus + 1/taue) / 2, lag(z) = 1 - (1 - e^-z)/z, with respect to g, ts, taus, te, taue.
    lag'(z) = -(em (1 + z) + z) / z^2 (em = expm1(-z)), its series 1/2 - z/3 + z^2/8 - z^3/30
    below z < 1e-3 (where lag itself is a series)."""
    z = 0.5 * h * (1 / taus + 1 / taue)
    em = np.expm1(-z)
    small = z < T.GATE_SERIES_LIMIT
    zs = np.where(small, 1.0, z)
    ems = np.expm1(-zs)
    lag = np.where(small, z * (0.5 - z * (1 / 6 - z * (1 / 24 - z / 120))), (ems + zs) / zs)
    dlag = np.where(small, 0.5 - z * (1 / 3 - z * (1 / 8 - z / 30)),
                    -(ems * (1 + zs) + zs) / (zs * zs))
    dz = (ts - g) * (1 + em) + (te - ts) * dlag
    return 1 + em, -em - lag, dz * (-0.5 * h / (taus * taus)), lag, dz * (-0.5 * h / (taue * taue))


class Grads(NamedTuple):
    membrane: np.ndarray  # [S, C] d/d membrane permeability (m/s)
    junction: np.ndarray  # [S, E] d/d junction permeability (m/s)
    channel: np.ndarray  # [NCH, C] d/d channel permeability (m/s)


def zero_grads(b):
    return Grads(np.zeros((3, b.cells)), np.zeros((3, b.edges)),
                 np.zeros((b.channel_slots, b.cells)))


def rates_vjp(n, gj, gc, potential, mu_n, mu_g, control, b, topo):
    """Transposed linearisation of explicit_rates' amount and junction-gate rates at one stage
    (n, gj, gc, V), applied to their cotangents mu_n [S, C] and mu_g [E]. Returns
    (lam_c [S, C] on the concentrations, lam_V [C] on the cell potentials, lam_gj [E],
    lam_gc [2, NCH, C], Grads)."""
    w = topo.cell_world
    ci = (b.amount_reference + n) / b.volume
    co = (b.bath_amount / b.bath_volume)[:, w]
    rt = R * b.temperature[w]
    dvm = potential - b.bath_potential[w]
    lam_c = np.zeros_like(ci)
    lam_v = np.zeros(b.cells)
    g_m = np.zeros((3, b.cells))
    # Patch: J_s = A P_s mc (c_s B(-x_s) - co_s B(x_s)) / 1e-15, x_s = z_s F dv / RT;
    # the amount rate takes -J_s.
    for s in range(3):
        z = VALENCE[s]
        x = z * F * dvm / rt
        bp, bm, sp_, sm_ = T.bernoulli(x), T.bernoulli(-x), bernoulli_slope(x), bernoulli_slope(-x)
        pref = b.area * control.membrane / MOL_PER_FMOL
        g = pref * b.permeability[s]
        mu = -mu_n[s]
        lam_c[s] += mu * g * bm
        lam_v += mu * g * (-ci[s] * sm_ - co[s] * sp_) * (z * F / rt)
        g_m[s] += mu * pref * (ci[s] * bm - co[s] * bp)
    # Na/K-ATPase: cycles = -M expm1(a), M = cap avail exp(log_sat); the amount rates take
    # stoichiometry x cycles (Na -3, K +2).
    pump = tuple(b.pump[k][w] for k in range(7))
    atp, _, _, km_na, _, _, _ = pump
    mu_na = rt * (np.log(ci[0]) - np.log(co[0])) + F * dvm
    mu_k = rt * (np.log(ci[1]) - np.log(co[1])) + F * dvm
    cycles, energy, _ = T.pump_kinetics(ci[0], co[1], mu_na, mu_k, b.temperature[w], pump,
                                        b.pump_capacity, control.pump)
    enabled = (b.pump_capacity > 0) & (control.pump > 0)
    a = energy / rt
    u = 3 * (np.log(km_na) - np.log(ci[0]))
    log_sat = (
        -np.logaddexp(0.0, u)
        - np.logaddexp(0.0, 2 * (np.log(pump[4]) - np.log(co[1])))
        - np.logaddexp(0.0, np.log(pump[5]) - np.log(atp))
    )  # fmt: skip
    with np.errstate(all="ignore"):
        mag_a = np.exp(np.log(np.where(enabled, b.pump_capacity, 1.0))
                       + np.log(np.where(enabled, control.pump, 1.0)) + log_sat + a)
    dcda = np.where(enabled, -mag_a, 0.0)
    mu_cyc = -3.0 * mu_n[0] + 2.0 * mu_n[1]
    lam_c[0] += mu_cyc * (cycles * 3 * sigmoid(u) / ci[0] + dcda * (-3.0 / ci[0]))
    lam_c[1] += mu_cyc * (dcda * (2.0 / ci[1]))
    lam_v += mu_cyc * dcda * (-F / rt)
    # Channels: J = A P_ch open ctl ab (c B(-x) - co B(x)) / 1e-15 of the permeant species.
    nch, idx = b.channel_slots, np.arange(b.cells)
    lam_gc = np.zeros((2, nch, b.cells))
    g_ch = np.zeros((nch, b.cells))
    if nch:
        opening = T.channel_opening(gc, b.channel_code)
        dm, dh = opening_partials(gc, b.channel_code)
        for k in range(nch):
            sp = b.channel_species[k]
            z = VALENCE[sp]
            x = z * F * dvm / rt
            bp, bm = T.bernoulli(x), T.bernoulli(-x)
            sp_, sm_ = bernoulli_slope(x), bernoulli_slope(-x)
            c, c_out = ci[sp, idx], co[sp, idx]
            diff = c * bm - c_out * bp
            unit = b.area * control.channel[k] * b.channel_abundance[k] / MOL_PER_FMOL
            g = unit * b.channel_permeability[k] * opening[k]
            mu = -mu_n[sp, idx]
            lam_c[sp, idx] += mu * g * bm
            lam_v += mu * g * (-c * sm_ - c_out * sp_) * (z * F / rt)
            g_ch[k] += mu * unit * opening[k] * diff
            d_open = mu * unit * b.channel_permeability[k] * diff
            lam_gc[0, k] += d_open * dm[k]
            lam_gc[1, k] += d_open * dh[k]
    # Junctions: J_s = A_j P_j,s jc g (c_a B(-x) - c_b B(x)) / 1e-15; sender -J, receiver +J.
    s_, r_ = topo.sender, topo.receiver
    rte = R * b.temperature[topo.edge_world]
    dve = potential[s_] - potential[r_]
    lam_gj = np.zeros(b.edges)
    g_j = np.zeros((3, b.edges))
    d_dv = np.zeros(b.edges)
    for s in range(3):
        z = VALENCE[s]
        x = z * F * dve / rte
        bp, bm = T.bernoulli(x), T.bernoulli(-x)
        sp_, sm_ = bernoulli_slope(x), bernoulli_slope(-x)
        ca, cb = ci[s, s_], ci[s, r_]
        diff = ca * bm - cb * bp
        unit = b.junction_area * control.junction / MOL_PER_FMOL
        g = unit * b.junction_permeability[s] * gj
        xi = mu_n[s, r_] - mu_n[s, s_]
        np.add.at(lam_c[s], s_, xi * g * bm)
        np.add.at(lam_c[s], r_, -xi * g * bp)
        d_dv += xi * g * (-ca * sm_ - cb * sp_) * (z * F / rte)
        lam_gj += xi * unit * b.junction_permeability[s] * diff
        g_j[s] += xi * unit * gj * diff
    # Junction gate rate alpha (1 - g) - beta (g - min), shift = |dv| - threshold.
    shift = np.abs(dve) - b.gate_threshold
    alpha = 1.3 * np.exp(-77.0 * shift)
    sb = sigmoid(np.log(0.065) + 140.0 * shift)
    beta = 20.0 * sb
    lam_gj += mu_g * (-alpha - beta)
    d_dv += mu_g * np.sign(dve) * (-77.0 * alpha * (1 - gj)
                                   - 20.0 * 140.0 * sb * (1 - sb) * (gj - b.gate_minimum))
    np.add.at(lam_v, s_, d_dv)
    np.add.at(lam_v, r_, -d_dv)
    return lam_c, lam_v, lam_gj, lam_gc, Grads(g_m, g_j, g_ch)


def potential_slope(b):
    """dV/dn [S, C]: F z_s / C of the capacitor closure."""
    return VALENCE[:, None] * CHARGE_PER_FMOL / b.capacitance


def step_vjp(state, dt, control, b, topo, cot_amount, cot_gate, cot_channel):
    """Cotangents of the step's start (amounts, junction gates, channel gates) and the
    parameters' gradients, given the cotangents of its end state. Recomputes the step."""
    new, valid = T.ars222_step(state, dt, control, b, topo)
    w = topo.cell_world
    bath = b.bath_potential[w]
    dvdn = potential_slope(b)
    nch = b.channel_slots
    gamma, delta = T.GAMMA, T.DELTA
    frac1 = float(np.sum(np.array([gamma, 0.0, 0.0])))
    frac2 = float(np.sum(np.array([delta, 1.0 - delta, 0.0])))
    n0, gj0, gc0 = state.amount_increment, state.junction_gate, state.channel_gate
    v0 = T.capacitor_potential(T.node_charge(state, b), b, topo)
    k0 = T.explicit_rates(state, v0, control, b, topo).state
    n1 = n0 + (gamma * dt) * k0.amount_increment
    gj1 = gj0 + (gamma * dt) * k0.junction_gate
    stage1 = state._replace(amount_increment=n1, junction_gate=gj1)
    v1 = T.operator_potential(T.node_charge(stage1, b), b, topo)[0]
    n2 = n0 + (delta * dt) * k0.amount_increment
    rows = T.gate_rows_active(b.channel_code)
    gc1 = gc0
    if nch:
        with np.errstate(all="ignore"):
            t0, tau0 = T.channel_kinetics((v0 - bath)[None, :], b.channel_code)
            d_t0, d_tau0 = channel_kinetics_slope((v0 - bath)[None, :], b.channel_code)
            t1, tau1 = T.channel_kinetics((v1 - bath)[None, :], b.channel_code)
            d_t1, d_tau1 = channel_kinetics_slope((v1 - bath)[None, :], b.channel_code)
        gc1 = np.where(rows, T.advance_gates(gc0, t0, tau0, t1, tau1, frac1 * dt), gc0)
    k1 = T.explicit_rates(stage1._replace(channel_gate=gc1), v1, control, b, topo).state
    n2 = n2 + ((1.0 - delta) * dt) * k1.amount_increment
    v2 = T.operator_potential(T.node_charge(state._replace(amount_increment=n2), b), b, topo)[0]

    lam_n2 = cot_amount.copy()
    lam_gc = np.zeros_like(gc0)
    lam_v0 = np.zeros(b.cells)
    if nch:
        with np.errstate(all="ignore"):
            t2, tau2 = T.channel_kinetics((v2 - bath)[None, :], b.channel_code)
            d_t2, d_tau2 = channel_kinetics_slope((v2 - bath)[None, :], b.channel_code)
        pg, pts, ptaus, pte, ptaue = advance_partials(gc0, t0, tau0, t2, tau2, frac2 * dt)
        lam_gc += np.where(rows, cot_channel * pg, cot_channel)
        lam_v0 += np.sum(np.where(rows, cot_channel * (pts * d_t0 + ptaus * d_tau0), 0.0),
                         axis=(0, 1))
        lam_v2 = np.sum(np.where(rows, cot_channel * (pte * d_t2 + ptaue * d_tau2), 0.0),
                        axis=(0, 1))
        lam_n2 = lam_n2 + lam_v2 * dvdn
    lam_n = lam_n2.copy()
    lam_g = cot_gate.copy()
    mu0n, mu1n = (delta * dt) * lam_n2, ((1.0 - delta) * dt) * lam_n2
    mu0g, mu1g = (delta * dt) * cot_gate, ((1.0 - delta) * dt) * cot_gate
    # Stage 1.
    lam_c1, lam_v1, lam_gj1, lam_gc1, g1 = rates_vjp(n1, gj1, gc1, v1, mu1n, mu1g, control, b,
                                                      topo)
    if nch:
        pg, pts, ptaus, pte, ptaue = advance_partials(gc0, t0, tau0, t1, tau1, frac1 * dt)
        lam_gc += np.where(rows, lam_gc1 * pg, lam_gc1)
        lam_v0 += np.sum(np.where(rows, lam_gc1 * (pts * d_t0 + ptaus * d_tau0), 0.0),
                         axis=(0, 1))
        lam_v1 = lam_v1 + np.sum(np.where(rows, lam_gc1 * (pte * d_t1 + ptaue * d_tau1), 0.0),
                                 axis=(0, 1))
    lam_n1 = lam_c1 / b.volume + lam_v1 * dvdn
    lam_n += lam_n1
    lam_g += lam_gj1
    mu0n = mu0n + (gamma * dt) * lam_n1
    mu0g = mu0g + (gamma * dt) * lam_gj1
    # Stage 0.
    lam_c0, lam_v, lam_gj0, lam_gc0, g0 = rates_vjp(n0, gj0, gc0, v0, mu0n, mu0g, control, b,
                                                     topo)
    lam_gc += lam_gc0
    lam_n += lam_c0 / b.volume + (lam_v0 + lam_v) * dvdn
    lam_g += lam_gj0
    grads = Grads(*(x + y for x, y in zip(g0, g1, strict=True)))
    # A refused world: identity, no gradient.
    cm, em = valid[w], valid[topo.edge_world]
    lam_n = np.where(cm, lam_n, cot_amount)
    lam_g = np.where(em, lam_g, cot_gate)
    lam_gc = np.where(cm, lam_gc, cot_channel)
    grads = Grads(np.where(cm, grads.membrane, 0.0), np.where(em, grads.junction, 0.0),
                  np.where(cm, grads.channel, 0.0))
    return (lam_n, lam_g, lam_gc), grads, new, valid


def membrane_voltage(state, b, topo):
    return T.membrane_voltage(state, b, topo)


def voltage_loss(state, b, topo, target):
    """Per-world sum over cells of (V_m - target)^2 (V^2) and its amount cotangent."""
    v = membrane_voltage(state, b, topo)
    d = v - target
    loss = np.zeros(b.worlds)
    np.add.at(loss, topo.cell_world, d * d)
    return loss, 2.0 * d * potential_slope(b)


def trajectory_grad(state, dt, control, b, n_steps, target):
    """Per-world loss of the state after n_steps steps and the permeability gradients of each
    world's loss (every state kept: small cases). Returns (loss [W], Grads, refused steps [W])."""
    topo = T.topology(b)
    states = [state]
    refused = np.zeros(b.worlds, dtype=np.int64)
    for _ in range(n_steps):
        state, valid = T.ars222_step(state, dt, control, b, topo)
        refused += ~valid
        states.append(state)
    loss, cot_n = voltage_loss(state, b, topo, target)
    cot = (cot_n, np.zeros(b.edges), np.zeros_like(state.channel_gate))
    total = zero_grads(b)
    for t in range(n_steps - 1, -1, -1):
        cot, g, _, _ = step_vjp(states[t], dt, control, b, topo, *cot)
        total = Grads(*(x + y for x, y in zip(total, g, strict=True)))
    return loss, total, refused


def trajectory_loss(state, dt, control, b, n_steps, target):
    """Per-world loss after n_steps steps (the forward alone, for finite differences)."""
    topo = T.topology(b)
    for _ in range(n_steps):
        state, _ = T.ars222_step(state, dt, control, b, topo)
    return voltage_loss(state, b, topo, target)[0]
