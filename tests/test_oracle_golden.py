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
    if "control_membrane" in z:
        return T.Control(z["control_membrane"], z["control_junction"], z["control_pump"])
    return T.full_control(b)


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
            worst[f] = max(worst.get(f, 0.0), scaled_difference(getattr(st, f), z["ref_" + f][idx]))
    return worst


@pytest.mark.parametrize("name,limit", [
    ("ars222_grid4x4.npz", 2000),
    ("ars222_v3_grid4x4.npz", None),
    ("ars222_gated.npz", None),
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
