"""CPU oracle of the ROS2 step on held-bath tissues (this library's
``cells_b200.solver.ros2_verwer@1``; the reference has no Rosenbrock method on its tissue path).

TEST INFRASTRUCTURE ONLY, like oracle/tissue.py: only ``tests/`` and ``bench.py``'s CPU baseline
leg may import it, as the parity reference or the timed CPU baseline.

The method is the two-stage, second-order, L-stable Rosenbrock scheme of Verwer, Spee, Blom and
Hundsdorfer (SIAM J. Sci. Comput. 20 (1999) 1456-1480), with gamma = 1 + 1/sqrt(2):

    W k1 = F(y),   W k2 = F(y + h k1) - 2 k1,   y' = y + (3/2) h k1 + (1/2) h k2,
    W = I - gamma h J.

Its order is two for any J (a W-method), so J carries only what makes the step stable and the
ledgers consistent. The stage structure follows the reference's only Rosenbrock integrator
(numerics/rosenbrock_dense.py:123-141: the stage right-hand sides, one factored matrix per step,
stage solves). F is the reference's whole right-hand side (surface_kinetic.readouts' derivative,
models/surface_kinetic.py:221-410, as ``oracle.tissue.readout_rates``); J is:

* the routes' slope conductances at y: every patch's, channel population's and junction's
  dJ/d(dv) (the reference's ``conductance_weights`` with its ``bernoulli_slope``,
  models/surface_pump_v3.py:2741-2813, laws/routes/patch_electrodiffusion.py:43-54), through the
  membrane potential's dependence on the cell's charge, dV/dn_s = z_s F/C. Every row whose rate
  is a route flux (amounts, the transfer ledgers, the bath supply, the heats through dJ/dV mu +
  J z F, the electrode charge and the works) gets the same linearisation, so the ledgers stay
  conserved to rounding. Solving W k = r then reduces to one SPD system per world in the cells'
  voltage rates u, (C + gamma h G) u = K sum_s z_s r_s (G the conductance Laplacian of N2's
  operator, models/surface_pump_v3.py:2816-2841, the bath held), after which each route's rate
  is r + gamma h W du;
* each gate's own relaxation rate on its diagonal (junction gates alpha + beta of
  junction_voltage_relaxation, channel gates 1/tau), and a channel gate's dependence on its
  cell's voltage, d/dV of (target - g)/tau (the channel laws' slopes, as the adjoint oracle
  forms them): k_g = (r_g + gamma h dg'/dV u) / (1 + gamma h lambda). The fast gates (NaV1.2's
  m relaxes in tens of microseconds) are stiff in both, and a W-matrix without the voltage
  coupling loses an order on them;
* zero for the pump (its rates stay explicit in k = r) and for the gates' effect on the fluxes.

The operator is factored once per step at y. ``ros2_step(..., factor32=True)`` restates this
library's CB_METHOD_ROS2_MIXED: the Jacobi-scaled factor rounded to FP32 and both substitutions
in FP32, nothing refined (a W-method keeps its order and its ledgers for any W; the FP32 factor
is the exact factor of a W within FP32 rounding of this one). A world's step is refused (its state kept) when a
rate evaluation is invalid (the reference's RK4 rule, numerics/fixed_step.py:25-71: the trial
state's domain first, then its rates), a slope is not finite, the operator is not positive
definite, or the new state leaves the domain.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sl

from oracle import adjoint as A
from oracle import n2 as N
from oracle import tissue as T

GAMMA = 1.0 + 1.0 / math.sqrt(2.0)
K = T.CHARGE_PER_FMOL
F = T.F
VALENCE = T.VALENCE


class Jacobian:
    """The step's W-matrix pieces at y: route slopes, the factored voltage operator, the gates'
    relaxation rates, and the start fluxes and potential differences the heat rows need."""

    def __init__(self, state, control, b, topo, h, factor32=False):
        self.factor32 = factor32
        w = topo.cell_world
        bath = b.bath_potential[w]
        self.h = h
        potential = T.capacitor_potential(T.node_charge(state, b), b, topo)
        with np.errstate(all="ignore"):
            self.weights = N.conductance_weights(state, potential, control, b, topo)
        membrane, channel, junction = self.weights
        ok_c = np.all(np.isfinite(membrane), axis=0) & np.all(np.isfinite(channel), axis=0)
        ok_e = np.all(np.isfinite(junction), axis=0)
        self.valid = np.ones(b.worlds, dtype=bool)
        np.logical_and.at(self.valid, w, ok_c)
        np.logical_and.at(self.valid, topo.edge_world, ok_e)
        g_patch, g_junction = N.patch_conductance(self.weights, b)
        with np.errstate(all="ignore"):
            self.operator = N.Operator(np.where(np.isfinite(g_patch), g_patch, 0.0),
                                       np.where(np.isfinite(g_junction), g_junction, 0.0),
                                       GAMMA * h, b, topo)
        self.valid &= self.operator.valid
        # Start fluxes and electrochemical differences for the heat rows.
        rates = T.explicit_rates(state, potential, control, b, topo)
        self.jm = rates.state.membrane_transferred
        self.jj = rates.state.junction_transferred
        self.jc = rates.state.channel_transferred
        self.mu_m, self.mu_j = N.delta_mu(state, potential, b, topo)
        # Gate relaxation rates.
        dve = potential[topo.sender] - potential[topo.receiver]
        with np.errstate(all="ignore"):
            _, relaxation = N.junction_kinetics(dve, b.gate_threshold, b.gate_minimum)
        self.junction_decay = np.where(np.isfinite(relaxation), relaxation, 0.0)
        self.channel_decay = np.zeros_like(state.channel_gate)
        self.channel_coupling = np.zeros_like(state.channel_gate)
        if b.channel_slots:
            v = (potential - bath)[None, :]
            with np.errstate(all="ignore"):
                target, tau = T.channel_kinetics(v, b.channel_code)
                dtarget, dtau = A.channel_kinetics_slope(v, b.channel_code)
                # d/dV of (target - g)/tau at y.
                coupling = dtarget / tau - (target - state.channel_gate) * dtau / (tau * tau)
            rows = T.gate_rows_active(b.channel_code)
            ok = rows & np.isfinite(tau) & (tau > 0) & np.isfinite(coupling)
            self.channel_decay = np.where(ok, 1.0 / tau, 0.0)
            self.channel_coupling = np.where(ok, coupling, 0.0)

    def voltage_rate(self, rho, b):
        """u of (C + gamma h G) u = rho per world, the bath held (its rate zero)."""
        u = np.zeros(b.cells)
        for wi, (_, scale, factor, free, _) in enumerate(self.operator.worlds):
            c0, c1 = b.cell_offset[wi], b.cell_offset[wi + 1]
            rhs = np.where(free, np.r_[rho[c0:c1], 0.0] * scale, 0.0)
            with np.errstate(all="ignore"):
                if self.factor32:
                    lower = np.asarray(factor, dtype=np.float32)
                    y = sl.solve_triangular(lower, rhs.astype(np.float32), lower=True)
                    sol = sl.solve_triangular(lower.T, y, lower=False).astype(np.float64)
                else:
                    sol = N.cholesky_solve(factor, rhs)
                x = np.where(free, sol * scale, 0.0)
            u[c0:c1] = x[:-1]
        return u

    def solve(self, r, b, topo):
        """k = W^-1 r for a rate State r."""
        gh = GAMMA * self.h
        rho = K * np.sum(VALENCE[:, None] * r.amount_increment, axis=0)
        u = self.voltage_rate(rho, b)
        membrane, channel, junction = self.weights
        du_e = u[topo.sender] - u[topo.receiver]
        dm, dc, dj = membrane * u, channel * u, junction * du_e  # the routes' dJ/dV du
        cells, outside = N.route_rates(dm, dc, dj, b, topo)
        z = VALENCE[:, None]
        idx = np.arange(b.cells)
        heat_m = 1e-3 * np.sum(dm * self.mu_m + self.jm * (z * F) * u, axis=0)
        heat_j = 1e-3 * np.sum(dj * self.mu_j + self.jj * (z * F) * du_e, axis=0)
        heat_c = np.zeros_like(r.channel_dissipated)
        for q in range(b.channel_slots):
            sp = b.channel_species[q]
            heat_c[q] = 1e-3 * (dc[q] * self.mu_m[sp, idx] + self.jc[q] * (VALENCE[sp] * F) * u)
        supply = -outside
        charge_rate = K * np.sum(z * cells, axis=0)
        electrode = np.zeros(b.worlds)
        np.add.at(electrode, topo.cell_world, -charge_rate)
        co = b.bath_amount / b.bath_volume
        mu_b = T.R * b.temperature * np.log(co) + z * F * b.bath_potential
        return r._replace(
            amount_increment=r.amount_increment + gh * cells,
            membrane_transferred=r.membrane_transferred + gh * dm,
            junction_transferred=r.junction_transferred + gh * dj,
            channel_transferred=r.channel_transferred + gh * dc,
            membrane_dissipated=r.membrane_dissipated + gh * heat_m,
            junction_dissipated=r.junction_dissipated + gh * heat_j,
            channel_dissipated=r.channel_dissipated + gh * heat_c,
            reservoir_supplied=r.reservoir_supplied + gh * supply,
            electrode_charge=r.electrode_charge + gh * electrode,
            reservoir_work=r.reservoir_work + gh * (1e-3 * np.sum(mu_b * supply, axis=0)),
            electrode_work=r.electrode_work + gh * (1e12 * b.bath_potential * electrode),
            junction_gate=r.junction_gate / (1.0 + gh * self.junction_decay),
            channel_gate=(r.channel_gate + gh * self.channel_coupling * u)
            / (1.0 + gh * self.channel_decay),
        )


def _axpy(state, terms):
    """state + sum(weight * rates), one term at a time."""
    out = state
    for weight, rates in terms:
        out = T.State(*(y + weight * d for y, d in zip(out, rates, strict=True)))
    return out


def _minus(a, b, factor):
    return T.State(*(x - factor * y for x, y in zip(a, b, strict=True)))


def ros2_step(state, dt, control, b, topo=None, factor32=False):
    """One ROS2 step for every world; returns (state, valid[W]). factor32: the FP32-factor form."""
    topo = T.topology(b) if topo is None else topo
    valid = T.domain_valid(state, b, topo)
    f0, ok = T.readout_rates(state, control, b, topo)
    valid &= ok
    jac = Jacobian(state, control, b, topo, dt, factor32)
    valid &= jac.valid
    k1 = jac.solve(f0, b, topo)
    trial = _axpy(state, [(dt, k1)])
    valid &= T.domain_valid(trial, b, topo)
    f1, ok = T.readout_rates(trial, control, b, topo)
    valid &= ok
    k2 = jac.solve(_minus(f1, k1, 2.0), b, topo)
    new = _axpy(state, [(1.5 * dt, k1), (0.5 * dt, k2)])
    valid &= T.domain_valid(new, b, topo)
    return T._select(valid, new, state, b, topo), valid
