"""The N2 oracle (oracle/n2.py) against the reference's own N2 step (@3 under
cells.solver.imex_ars222_implicit_conductances@1, run by tests/golden/make_golden.py): every
field bit for bit over the whole trajectory, the electrode ledgers to 1e-15 (the reference sums
the bath's plate charge with BLAS)."""

import numpy as np
import pytest

from conftest import load_golden, scaled_difference
from oracle import n2
from oracle import tissue as T

LOOSE = {"electrode_charge", "electrode_work"}


def control_of(z, b):
    full = T.full_control(b)
    return T.Control(*(z["control_" + f] if "control_" + f in z.files else getattr(full, f)
                       for f in ("membrane", "junction", "pump", "channel")))


@pytest.mark.parametrize("name", ["n2_grid4x4.npz", "n2_channels_delaunay.npz"])
def test_n2_oracle_matches_the_reference_step(name):
    z, b = load_golden(name)
    topo = T.topology(b)
    control = control_of(z, b)
    state, done = T.initial_state(b), 0
    for idx, target in enumerate(z["steps"]):
        while done < target:
            state, valid = n2.n2_step(state, float(z["dt"]), control, b, topo)
            assert valid.all(), done
            done += 1
        for f in T.State._fields:
            if "ref_" + f not in z.files:
                continue
            got, ref = getattr(state, f), z["ref_" + f][idx]
            if f in LOOSE:
                assert scaled_difference(got, ref) <= 1e-15, (f, target)
            else:
                assert np.array_equal(got, ref), (f, target, scaled_difference(got, ref))


def test_n2_keeps_the_ledgers():
    """Material, charge and the works balance after N2 steps as after ARS(2,2,2) ones."""
    z, b = load_golden("n2_channels_delaunay.npz")
    topo = T.topology(b)
    state = T.initial_state(b)
    control = control_of(z, b)
    for _ in range(50):
        state, _ = n2.n2_step(state, 1e-3, control, b, topo)
    res = T.balances(state, b, topo)
    for key in ("local", "outside", "total"):
        assert np.max(np.abs(res[key])) <= 1e-12 * np.max(np.abs(state.amount_increment))
    assert np.max(np.abs(res["electrode"])) <= 1e-26
    assert np.max(np.abs(res["global_charge"])) <= 1e-26


def test_slope_is_the_bernoulli_derivative():
    x = np.concatenate([np.linspace(-30, 30, 301), np.geomspace(1e-9, 1e-2, 40),
                        -np.geomspace(1e-9, 1e-2, 40)])
    h = 1e-6 * np.maximum(np.abs(x), 1e-2)
    fd = (T.bernoulli(x + h) - T.bernoulli(x - h)) / (2 * h)
    assert np.allclose(n2.bernoulli_slope(x), fd, rtol=1e-5, atol=1e-8)
