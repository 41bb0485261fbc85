"""CPU oracle of the ROS2 step's reverse-mode derivative: the discrete adjoint of
oracle.ros2.ros2_step, and loss gradients through a ROS2 trajectory.

TEST INFRASTRUCTURE ONLY, like oracle/adjoint.py: only ``tests/`` and ``bench.py``'s CPU
baseline leg may import it; the product path (``cells_b200``) never calls it.

The step (oracle/ros2.py; Verwer, Spee, Blom and Hundsdorfer's ROS2, gamma = 1 + 1/sqrt(2)):

    W k1 = F(y),  y1 = y + h k1,  W k2 = F(y1) - 2 k1,  y' = y + 3/2 h k1 + 1/2 h k2,

with W = I - gamma h J(y). Its dynamic state is the amount increments n [S, C], the junction
gates g [E] and the channel gates gc [2, NCH, C]; the ledgers never feed back. Per world, W k = r
is, on the dynamic rows,

    M u = K sum_s z_s r_n,s        M = C + gamma h (diag(G_patch) + L(G_junction))  (bath held)
    k_n = r_n + gamma h route_rates(W_m u, W_c u, W_j du)
    k_g = r_g / (1 + gamma h lambda)                       (junction gates)
    k_gc = (r_gc + gamma h cpl u) / (1 + gamma h dec)      (channel gates)

where W_m, W_c, W_j are the routes' slope conductances at y (N2's route_slope), G their charge
sums, lambda the junction gate law's relaxation rate at y, dec = 1/tau and cpl = d/dV of
(target - g)/tau of a channel gate row at y. The reverse of one step, given the cotangent of
y' (dynamic rows):

    kbar1 = 3/2 h ybar',  kbar2 = 1/2 h ybar'
    (rbar2, Jbar) = solve^T(kbar2)        the transposed stage solve: M is symmetric, so
                                          rho_bar = M^-1 ubar is one more solve through the
                                          step's factor; M's own dependence on y gives
                                          G_patch_bar = -gamma h rho_bar u and
                                          G_junction_bar = -gamma h (rho_bar_a - rho_bar_b) du
    kbar1 -= 2 rbar2;  ybar1 = F^T(y1) rbar2;  ybar += ybar1;  kbar1 += h ybar1
    (rbar1, Jbar) += solve^T(kbar1);  ybar += F^T(y) rbar1
    ybar += J^T(y) Jbar                   the slopes', relaxation rates' and couplings'
                                          dependence on y (second derivatives of the laws)

F^T is oracle.adjoint.rates_vjp (the amount and junction-gate rates) plus the channel gate rows
(target - g)/tau. The second derivatives: B''(x) of the Bernoulli function (``curvature``),
the channel laws' target'' and tau'' (``channel_kinetics_curvature``), d lambda/dV of the
junction gate law. A step a world refused is the identity for it and adds nothing.

Pinned by central finite differences of oracle.ros2.ros2_step (tests/test_oracle_ros2_adjoint.py),
which is itself pinned to the reference's RK4 by observed order and by the ledgers.
"""

from __future__ import annotations

import numpy as np

from oracle import adjoint as A
from oracle import n2 as N
from oracle import ros2 as R2
from oracle import tissue as T

F, R = T.F, T.R
K = T.CHARGE_PER_FMOL
VALENCE = T.VALENCE
MOL_PER_FMOL = T.MOL_PER_FMOL
GAMMA = R2.GAMMA
CURVATURE_SERIES_BELOW = 0.1


def curvature(x):
    """B''(x) for B(x) = x / expm1(x). B'' is even (B(-x) = B(x) + x); with a = |x|,
    om = -expm1(-a) = 1 - e^-a:  B'' = (1 - om)(a (2 - om) - 2 om) / om^3. Below a < 0.1 the
    series 1/6 - x^2/60 + x^4/1008 - x^6/21600 + x^8/532224 (from the Bernoulli numbers
    B_2 .. B_10)."""
    x = np.asarray(x, dtype=float)
    a = np.abs(x)
    small = a < CURVATURE_SERIES_BELOW
    aa = np.where(small, 1.0, a)
    om = -np.expm1(-aa)
    closed = (1.0 - om) * (aa * (2.0 - om) - 2.0 * om) / (om * om * om)
    x2 = x * x
    series = 1.0 / 6.0 + x2 * (-1.0 / 60.0 + x2 * (1.0 / 1008.0 + x2 * (-1.0 / 21600.0
                                                                          + x2 / 532224.0)))
    return np.where(small, series, closed)


def slope_partials(c_from, c_to, dv, valence, temperature, area, permeability, available):
    """Partials of route_slope W = p k (-c_from B'(-x) - c_to B'(x)), x = k dv, k = z F/RT,
    p = A P avail / 1e-15: (dW/dc_from, dW/dc_to, dW/d dv, dW/d(P avail) / P ... as the unit
    slope W1 = W / (P avail))."""
    k = valence * F / (R * temperature)
    x = k * dv
    unit = area / MOL_PER_FMOL
    p = unit * permeability * available
    bm, bp = N.bernoulli_slope(-x), N.bernoulli_slope(x)
    d_from = p * k * (-bm)
    d_to = p * k * (-bp)
    d_dv = p * k * k * curvature(x) * (c_from - c_to)
    w1 = unit * k * (-c_from * bm - c_to * bp)  # W per unit (P avail)
    return d_from, d_to, d_dv, w1


def _law_curvature(v, code):
    """Per law and row: (t, t', t'', kappa, kappa', kappa''), kappa = 1/tau, each [2, ...]."""
    B, dB, d2B = T.bernoulli, A.bernoulli_slope, curvature
    zero = np.zeros_like(v)
    out = {}
    with np.errstate(all="ignore"):
        # NaV1.2: m target a/s, tau 0.001/s; h target sigma(-(v + 0.055)/0.0062), tau 0.001/q.
        sh = (v + 0.025) / 0.009
        a, da, d2a = 0.182 * 9 * B(-sh), -0.182 * 9 * dB(-sh) / 0.009, \
            0.182 * 9 * d2B(-sh) / 0.009**2
        d, dd, d2d = 0.124 * 9 * B(sh), 0.124 * 9 * dB(sh) / 0.009, 0.124 * 9 * d2B(sh) / 0.009**2
        s, ds, d2s = a + d, da + dd, d2a + d2d
        t = a / s
        dt_ = (da - t * ds) / s
        d2t = (d2a - 2 * dt_ * ds - t * d2s) / s
        th = 1 / (1 + np.exp((v + 0.055) / 0.0062))
        dth = -th * (1 - th) / 0.0062
        d2th = -dth * (1 - 2 * th) / 0.0062
        ur = -(v + 0.040) / 0.005
        ui = (v + 0.065000123) / 0.005
        q = 0.024 * 5 * B(ur) + 0.0091 * 5 * B(ui)
        dq = -0.024 * 5 * dB(ur) / 0.005 + 0.0091 * 5 * dB(ui) / 0.005
        d2q = 0.024 * 5 * d2B(ur) / 0.005**2 + 0.0091 * 5 * d2B(ui) / 0.005**2
        out[T.NAV1P2] = (np.stack((t, th)), np.stack((dt_, dth)), np.stack((d2t, d2th)),
                         np.stack((1000.0 * s, 1000.0 * q)), np.stack((1000.0 * ds, 1000.0 * dq)),
                         np.stack((1000.0 * d2s, 1000.0 * d2q)))
        # Hodgkin-Huxley K n: alpha 100 B(-(1000 v + 55)/10), beta 125 e^-(1000 v + 65)/80.
        ua = -(1000.0 * v + 55.0) / 10.0
        al, dal, d2al = 100.0 * B(ua), -100.0 * 100.0 * dB(ua), 100.0 * 100.0**2 * d2B(ua)
        be = 125.0 * np.exp(-(1000.0 * v + 65.0) / 80.0)
        dbe, d2be = -12.5 * be, 156.25 * be
        s, ds, d2s = al + be, dal + dbe, d2al + d2be
        t = al / s
        dt_ = (dal - t * ds) / s
        d2t = (d2al - 2 * dt_ * ds - t * d2s) / s
        out[T.HH_K_N4] = (np.stack((t, zero)), np.stack((dt_, zero)), np.stack((d2t, zero)),
                          np.stack((s, zero)), np.stack((ds, zero)), np.stack((d2s, zero)))
        # Kv1.5: sigmoid targets, tau linear in v.
        s0 = A.sigmoid((v + 0.0060) / 0.0064)
        ds0 = s0 * (1 - s0) / 0.0064
        d2s0 = ds0 * (1 - 2 * s0) / 0.0064
        s1 = A.sigmoid(-(v + 0.0253) / 0.0035)
        ds1 = -s1 * (1 - s1) / 0.0035
        d2s1 = -ds1 * (1 - 2 * s1) / 0.0035
        tau = np.stack((0.008330 - 0.1163 * v, 1.620000 - 15.500 * v))
        dtau = np.stack((np.full_like(v, -0.1163), np.full_like(v, -15.5)))
        kap = 1.0 / tau
        dkap = -dtau / (tau * tau)
        d2kap = 2.0 * dtau * dtau / (tau * tau * tau)
        out[T.KV1P5] = (np.stack((s0, s1)), np.stack((ds0, ds1)), np.stack((d2s0, d2s1)),
                        kap, dkap, d2kap)
    return out


def channel_kinetics_curvature(v, code):
    """(t, t', t'', kappa, kappa', kappa'') of every population's gate rows, [2, NCH, C] each,
    kappa = 1/tau (zeros where no law)."""
    v = np.broadcast_to(v, code.shape)
    res = [np.zeros((2, *code.shape)) for _ in range(6)]
    laws = _law_curvature(v, code)
    for law, parts in laws.items():
        mask = (code == law)[None]
        res = [np.where(mask, p, r) for p, r in zip(parts, res, strict=True)]
    return tuple(res)


class Pieces:
    """The step's W-matrix at y (oracle.ros2.Jacobian) plus what the reverse needs: the
    potentials and concentrations at y, the rows' masks and the laws' second derivatives."""

    def __init__(self, state, control, b, topo, h):
        self.jac = R2.Jacobian(state, control, b, topo, h)
        w = topo.cell_world
        self.v = T.capacitor_potential(T.node_charge(state, b), b, topo)
        self.ci = (b.amount_reference + state.amount_increment) / b.volume
        self.co = (b.bath_amount / b.bath_volume)[:, w]
        self.dve = self.v[topo.sender] - self.v[topo.receiver]
        _, relax = N.junction_kinetics(self.dve, b.gate_threshold, b.gate_minimum)
        self.junction_ok = np.isfinite(relax)
        if b.channel_slots:
            vm = (self.v - b.bath_potential[w])[None, :]
            with np.errstate(all="ignore"):
                self.kin = channel_kinetics_curvature(vm, b.channel_code)
            rows = T.gate_rows_active(b.channel_code)
            self.channel_ok = rows & (self.jac.channel_decay != 0.0)


def voltage_rate(jac, rho, b):
    return jac.voltage_rate(rho, b)


def solve_forward(jac, r_n, r_g, r_gc, b, topo):
    """The dynamic rows of k = W^-1 r and the voltage rate u."""
    gh = GAMMA * jac.h
    rho = K * np.sum(VALENCE[:, None] * r_n, axis=0)
    u = jac.voltage_rate(rho, b)
    membrane, channel, junction = jac.weights
    du = u[topo.sender] - u[topo.receiver]
    cells, _ = N.route_rates(membrane * u, channel * u, junction * du, b, topo)
    k_n = r_n + gh * cells
    k_g = r_g / (1.0 + gh * jac.junction_decay)
    k_gc = (r_gc + gh * jac.channel_coupling * u) / (1.0 + gh * jac.channel_decay)
    return k_n, k_g, k_gc, u


class JBar:
    """Cotangents of the W-matrix's pieces: slopes, junction relaxation, channel decay and
    coupling."""

    def __init__(self, b):
        self.wm = np.zeros((3, b.cells))
        self.wc = np.zeros((b.channel_slots, b.cells))
        self.wj = np.zeros((3, b.edges))
        self.lam = np.zeros(b.edges)
        self.dec = np.zeros((2, b.channel_slots, b.cells))
        self.cpl = np.zeros((2, b.channel_slots, b.cells))


def solve_vjp(jac, kbar_n, kbar_g, kbar_gc, u, k_g, k_gc, jb, b, topo):
    """Transposed k = W^-1 r on the dynamic rows: returns (rbar_n, rbar_g, rbar_gc) and adds the
    pieces' cotangents to jb."""
    gh = GAMMA * jac.h
    membrane, channel, junction = jac.weights
    s_, r_ = topo.sender, topo.receiver
    idx = np.arange(b.cells)
    # Gates.
    den_g = 1.0 + gh * jac.junction_decay
    rbar_g = kbar_g / den_g
    jb.lam += -gh * kbar_g * k_g / den_g
    den_c = 1.0 + gh * jac.channel_decay
    rbar_gc = kbar_gc / den_c
    ubar = np.sum(gh * jac.channel_coupling * rbar_gc, axis=(0, 1)) if b.channel_slots else \
        np.zeros(b.cells)
    jb.cpl += gh * u[None, None, :] * rbar_gc
    jb.dec += -gh * kbar_gc * k_gc / den_c
    # Routes: cells = (recv - send) - patches, each route flux phi = W du.
    phim = -gh * kbar_n
    jb.wm += phim * u
    ubar = ubar + np.sum(phim * membrane, axis=0)
    for q in range(b.channel_slots):
        sp = b.channel_species[q]
        phic = -gh * kbar_n[sp, idx]
        jb.wc[q] += phic * u
        ubar = ubar + phic * channel[q]
    du = u[s_] - u[r_]
    phij = gh * (kbar_n[:, r_] - kbar_n[:, s_])
    jb.wj += phij * du
    uj = np.sum(phij * junction, axis=0)
    np.add.at(ubar, s_, uj)
    np.add.at(ubar, r_, -uj)
    # u = M^-1 rho, M symmetric: rho_bar = M^-1 u_bar.
    rho_bar = jac.voltage_rate(ubar, b)
    rbar_n = kbar_n + K * VALENCE[:, None] * rho_bar[None, :]
    gp_bar = -gh * rho_bar * u
    gj_bar = -gh * (rho_bar[s_] - rho_bar[r_]) * du
    jb.wm += K * VALENCE[:, None] * gp_bar[None, :]
    for q in range(b.channel_slots):
        jb.wc[q] += K * VALENCE[b.channel_species[q]] * gp_bar
    jb.wj += K * VALENCE[:, None] * gj_bar[None, :]
    return rbar_n, rbar_g, rbar_gc


def rates_vjp_full(state, control, b, topo, rbar_n, rbar_g, rbar_gc):
    """F^T at a state: (ybar_n, ybar_g, ybar_gc, Grads) of readout_rates' dynamic rows."""
    w = topo.cell_world
    v = T.capacitor_potential(T.node_charge(state, b), b, topo)
    lam_c, lam_v, lam_g, lam_gc, grads = A.rates_vjp(
        state.amount_increment, state.junction_gate, state.channel_gate, v, rbar_n, rbar_g,
        control, b, topo)
    if b.channel_slots:
        vm = (v - b.bath_potential[w])[None, :]
        with np.errstate(all="ignore"):
            t, dt_, _, kap, dkap, _ = channel_kinetics_curvature(vm, b.channel_code)
        rows = T.gate_rows_active(b.channel_code)
        g = state.channel_gate
        # rate = (t - g) kappa: d/dg = -kappa, d/dV = t' kappa + (t - g) kappa'.
        lam_gc = lam_gc + np.where(rows, -kap * rbar_gc, 0.0)
        lam_v = lam_v + np.sum(np.where(rows, (dt_ * kap + (t - g) * dkap) * rbar_gc, 0.0),
                               axis=(0, 1))
    ybar_n = lam_c / b.volume + lam_v * A.potential_slope(b)
    return ybar_n, lam_g, lam_gc, grads


def pieces_vjp(pc, state, control, jb, b, topo):
    """J^T(y): the slopes', relaxation rates', decays' and couplings' dependence on y and on
    the permeabilities. Returns (ybar_n, ybar_g, ybar_gc, Grads)."""
    w = topo.cell_world
    s_, r_ = topo.sender, topo.receiver
    idx = np.arange(b.cells)
    t_c = b.temperature[w]
    dv = pc.v - b.bath_potential[w]
    lam_c = np.zeros((3, b.cells))
    lam_v = np.zeros(b.cells)
    lam_gc = np.zeros_like(state.channel_gate)
    lam_g = np.zeros(b.edges)
    gm = np.zeros((3, b.cells))
    gj = np.zeros((3, b.edges))
    gch = np.zeros((b.channel_slots, b.cells))
    with np.errstate(all="ignore"):
        # Patches.
        for s in range(3):
            d_from, _, d_dv, w1 = slope_partials(pc.ci[s], pc.co[s], dv, VALENCE[s], t_c, b.area,
                                                 b.permeability[s], control.membrane)
            lam_c[s] += jb.wm[s] * d_from
            lam_v += jb.wm[s] * d_dv
            gm[s] += jb.wm[s] * w1 * control.membrane
        # Channels.
        if b.channel_slots:
            opening = T.channel_opening(state.channel_gate, b.channel_code)
            dm, dh = A.opening_partials(state.channel_gate, b.channel_code)
            for q in range(b.channel_slots):
                sp = b.channel_species[q]
                avail = b.channel_abundance[q] * opening[q] * control.channel[q]
                d_from, _, d_dv, w1 = slope_partials(pc.ci[sp, idx], pc.co[sp, idx], dv,
                                                     VALENCE[sp], t_c, b.area,
                                                     b.channel_permeability[q], avail)
                lam_c[sp, idx] += jb.wc[q] * d_from
                lam_v += jb.wc[q] * d_dv
                gch[q] += jb.wc[q] * w1 * avail
                d_open = jb.wc[q] * w1 * b.channel_permeability[q] * b.channel_abundance[q] \
                    * control.channel[q]
                lam_gc[0, q] += d_open * dm[q]
                lam_gc[1, q] += d_open * dh[q]
            # Decay kappa and coupling t' kappa + (t - g) kappa' of the rows in the operator.
            t, dt_, d2t, kap, dkap, d2kap = pc.kin
            g = state.channel_gate
            ok = pc.channel_ok
            lam_v += np.sum(np.where(ok, jb.dec * dkap, 0.0), axis=(0, 1))
            lam_v += np.sum(np.where(ok, jb.cpl * (d2t * kap + 2 * dt_ * dkap + (t - g) * d2kap),
                                     0.0), axis=(0, 1))
            lam_gc += np.where(ok, -jb.cpl * dkap, 0.0)
        # Junctions.
        t_e = b.temperature[topo.edge_world]
        ddv = np.zeros(b.edges)
        avail = control.junction * state.junction_gate
        for s in range(3):
            d_from, d_to, d_dv, w1 = slope_partials(pc.ci[s, s_], pc.ci[s, r_], pc.dve,
                                                    VALENCE[s], t_e, b.junction_area,
                                                    b.junction_permeability[s], avail)
            np.add.at(lam_c[s], s_, jb.wj[s] * d_from)
            np.add.at(lam_c[s], r_, jb.wj[s] * d_to)
            ddv += jb.wj[s] * d_dv
            gj[s] += jb.wj[s] * w1 * avail
            lam_g += jb.wj[s] * w1 * b.junction_permeability[s] * control.junction
        # Relaxation alpha + beta, shift = |dv| - threshold.
        shift = np.abs(pc.dve) - b.gate_threshold
        alpha = 1.3 * np.exp(-77.0 * shift)
        sb = A.sigmoid(np.log(0.065) + 140.0 * shift)
        dlam = np.sign(pc.dve) * (-77.0 * alpha + 20.0 * 140.0 * sb * (1 - sb))
        ddv += np.where(pc.junction_ok, jb.lam * dlam, 0.0)
    np.add.at(lam_v, s_, ddv)
    np.add.at(lam_v, r_, -ddv)
    ybar_n = lam_c / b.volume + lam_v * A.potential_slope(b)
    return ybar_n, lam_g, lam_gc, A.Grads(gm, gj, gch)


def step_vjp(state, dt, control, b, topo, cot_n, cot_g, cot_gc):
    """Cotangents of the step's start (amounts, junction gates, channel gates) and the
    permeabilities' gradients, given the cotangents of its end. Recomputes the step."""
    new, valid = R2.ros2_step(state, dt, control, b, topo)
    h = dt
    pc = Pieces(state, control, b, topo, h)
    jac = pc.jac
    f0, _ = T.readout_rates(state, control, b, topo)
    k1n, k1g, k1gc, u1 = solve_forward(jac, f0.amount_increment, f0.junction_gate,
                                       f0.channel_gate, b, topo)
    trial = state._replace(amount_increment=state.amount_increment + h * k1n,
                           junction_gate=state.junction_gate + h * k1g,
                           channel_gate=state.channel_gate + h * k1gc)
    f1, _ = T.readout_rates(trial, control, b, topo)
    _, k2g, k2gc, u2 = solve_forward(jac, f1.amount_increment - 2.0 * k1n,
                                     f1.junction_gate - 2.0 * k1g,
                                     f1.channel_gate - 2.0 * k1gc, b, topo)
    jb = JBar(b)
    yb_n, yb_g, yb_gc = cot_n.copy(), cot_g.copy(), cot_gc.copy()
    kb1 = [1.5 * h * cot_n, 1.5 * h * cot_g, 1.5 * h * cot_gc]
    kb2 = [0.5 * h * cot_n, 0.5 * h * cot_g, 0.5 * h * cot_gc]
    rb2 = solve_vjp(jac, *kb2, u2, k2g, k2gc, jb, b, topo)
    kb1 = [x - 2.0 * y for x, y in zip(kb1, rb2, strict=True)]
    y1n, y1g, y1gc, g1 = rates_vjp_full(trial, control, b, topo, *rb2)
    yb_n, yb_g, yb_gc = yb_n + y1n, yb_g + y1g, yb_gc + y1gc
    kb1 = [kb1[0] + h * y1n, kb1[1] + h * y1g, kb1[2] + h * y1gc]
    rb1 = solve_vjp(jac, *kb1, u1, k1g, k1gc, jb, b, topo)
    y0n, y0g, y0gc, g0 = rates_vjp_full(state, control, b, topo, *rb1)
    pn, pg, pgc, gp = pieces_vjp(pc, state, control, jb, b, topo)
    lam_n = yb_n + y0n + pn
    lam_g = yb_g + y0g + pg
    lam_gc = yb_gc + y0gc + pgc
    rows = T.gate_rows_active(b.channel_code)
    if b.channel_slots:
        lam_gc = np.where(rows, lam_gc, yb_gc)
    grads = A.Grads(*((x + y) + z for x, y, z in zip(g1, g0, gp, strict=True)))
    w = topo.cell_world
    cm, em = valid[w], valid[topo.edge_world]
    lam_n = np.where(cm, lam_n, cot_n)
    lam_g = np.where(em, lam_g, cot_g)
    lam_gc = np.where(cm, lam_gc, cot_gc)
    grads = A.Grads(np.where(cm, grads.membrane, 0.0), np.where(em, grads.junction, 0.0),
                    np.where(cm, grads.channel, 0.0))
    return (lam_n, lam_g, lam_gc), grads, new, valid


def trajectory_grad(state, dt, control, b, n_steps, target):
    """Per-world loss of the state after n_steps ROS2 steps and the permeability gradients of
    each world's loss (every state kept: small cases). Returns (loss [W], Grads, refused [W])."""
    topo = T.topology(b)
    states = [state]
    refused = np.zeros(b.worlds, dtype=np.int64)
    for _ in range(n_steps):
        state, valid = R2.ros2_step(state, dt, control, b, topo)
        refused += ~valid
        states.append(state)
    loss, cot_n = A.voltage_loss(state, b, topo, target)
    cot = (cot_n, np.zeros(b.edges), np.zeros_like(state.channel_gate))
    total = A.zero_grads(b)
    for t in range(n_steps - 1, -1, -1):
        cot, g, _, _ = step_vjp(states[t], dt, control, b, topo, *cot)
        total = A.Grads(*(x + y for x, y in zip(total, g, strict=True)))
    return loss, total, refused


def trajectory_loss(state, dt, control, b, n_steps, target):
    """Per-world loss after n_steps ROS2 steps (the forward alone, for finite differences)."""
    topo = T.topology(b)
    for _ in range(n_steps):
        state, _ = R2.ros2_step(state, dt, control, b, topo)
    return A.voltage_loss(state, b, topo, target)[0]
