"""The CPU oracle (oracle/tissue.py) against the reference's own step (golden fixtures).

The fixtures were produced by running the reference's models/surface_pump.py imex_step (and
surface_pump_v3.py's, and fixed_step.rk4_checked_step) on its NumPy branch; see
tests/golden/make_golden.py. The oracle reproduces them to rounding: bitwise for every field but
the electrode ledger, whose plate sum the reference forms with a BLAS product (order unknown).
"""

import numpy as np
import pytest

from conftest import load_golden, scaled_difference
from oracle import tissue as T

TOL = 1e-14  # rounding-level agreement with the reference's own arithmetic


def _controls(z, b):
    full = T.full_control(b)
    return T.Control(*(z["control_" + f] if "control_" + f in z else getattr(full, f)
                       for f in T.Control._fields))


def _replay(name, step, limit=None):
    z, b = load_golden(name)
    topo = T.topology(b)
    ctl = _controls(z, b)
    dt = float(z["dt"])
    st = T.initial_state(b)
    k = 0
    worst = {}
    for idx, target in enumerate(z["steps"]):
        if limit is not None and target > limit:
            break
        while k < target:
            st, ok = step(st, dt, ctl, b, topo)
            assert ok.all(), f"oracle refused step {k} of {name}"
            k += 1
        for f in T.State._fields:
            if "ref_" + f in z:
                worst[f] = max(worst.get(f, 0.0),
                               scaled_difference(getattr(st, f), z["ref_" + f][idx]))
    return worst


@pytest.mark.parametrize("name,limit", [
    ("ars222_grid4x4.npz", 2000),
    ("ars222_v3_grid4x4.npz", None),
    ("ars222_gated.npz", None),
    ("ars222_v3_channels.npz", None),
    ("ars222_v3_channels_delaunay.npz", None),
])
def test_oracle_matches_reference_ars222(name, limit):
    worst = _replay(name, T.ars222_step, limit)
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, bad


def test_oracle_matches_reference_rk4():
    worst = _replay("rk4_grid4x4.npz", T.rk4_step)
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, bad


def test_oracle_point_laws_match_reference():
    z = np.load(__import__("conftest").GOLDEN + "/laws.npz")
    assert np.array_equal(T.bernoulli(z["bernoulli_x"]), z["bernoulli"])
    pump = (1.5, 0.1, 0.1, 12.0, 0.2, 0.5, -37000.0)
    cycles, energy, drive = T.pump_kinetics(
        z["pump_na"], z["pump_ko"], z["pump_mu_na"], z["pump_mu_k"], 310.15, pump,
        z["pump_capacity"], z["pump_availability"])
    assert np.array_equal(cycles, z["pump_cycles"])
    assert np.array_equal(energy, z["pump_energy"])
    rate = T.gate_rhs(z["gate_g"], z["gate_v"], z["gate_threshold"], 0.1)
    assert np.array_equal(rate, z["gate_rate"])


def test_planted_change_is_caught():
    """A coefficient moved by 1e-9 in the oracle must fail the golden comparison (the
    reference's planted-change idea, tests/unit/test_channel_law_kernels.py:9-11)."""
    z, b = load_golden("ars222_grid4x4.npz")
    b.permeability = b.permeability * (1 + 1e-9)
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(100):
        st, _ = T.ars222_step(st, 1e-3, T.full_control(b), b, topo)
    idx = list(z["steps"]).index(100)
    assert scaled_difference(st.amount_increment, z["ref_amount_increment"][idx]) > 1e-12


def test_hh_k_n4_law_matches_its_closed_form():
    """The HH K n^4 law (this package's; the reference has no n^4 law): alpha_n and beta_n of
    Hodgkin and Huxley (1952) at a -65 mV rest, per ms, written out directly."""
    import math

    for v in (-0.1, -0.08, -0.065, -0.0551, -0.04, 0.0, 0.03):
        vm = 1000.0 * v
        a = 0.01 * (vm + 55.0) / (1.0 - math.exp(-(vm + 55.0) / 10.0))
        bta = 0.125 * math.exp(-(vm + 65.0) / 80.0)
        t, tau = T.hh_k_n4_kinetics(np.asarray(v))
        assert abs(float(t[0]) - a / (a + bta)) <= 1e-13
        assert abs(float(tau[0]) - 1e-3 / (a + bta)) <= 1e-13 * 1e-3 / (a + bta)
    t, _ = T.hh_k_n4_kinetics(np.asarray(-0.055))  # removable singularity: alpha = 0.1 / ms
    assert abs(float(t[0]) - 0.1 / (0.1 + 0.125 * math.exp(-10.0 / 80.0))) <= 1e-13


def test_exponential_gate_update_is_second_order():
    """advance_gates with a linearly varying target (numerics/exponential_gates.py): for a smooth
    target g_inf(t) = 0.3 + 50 t and tau(t) = 0.01 + 5 t, halving the step divides the one-step
    error by about 8 (local error O(h^3))."""
    def f(t, g):
        return ((0.3 + 50.0 * t) - g) / (0.01 + 5.0 * t)

    def exact(h, n=4000):
        g, dt = 0.2, h / n
        for i in range(n):  # classical RK4, far finer than h
            t = i * dt
            k1 = f(t, g)
            k2 = f(t + dt / 2, g + dt / 2 * k1)
            k3 = f(t + dt / 2, g + dt / 2 * k2)
            k4 = f(t + dt, g + dt * k3)
            g += dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        return g

    errs = []
    for h in (1e-3, 5e-4, 2.5e-4):
        g = T.advance_gates(np.asarray(0.2), 0.3, 0.01, 0.3 + 50.0 * h, 0.01 + 5.0 * h, h)
        errs.append(abs(float(g) - exact(h)))
    assert errs[0] / errs[1] > 6.0 and errs[1] / errs[2] > 6.0, errs
