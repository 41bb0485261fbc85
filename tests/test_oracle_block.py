"""The oracle's open-channel block (oracle/tissue.py: channel_block, the blocked membrane rate)
against the reference's own @3 trajectories with blocked populations
(tests/golden/ars222_v3_block*.npz, made by tests/golden/make_golden.py --only block).

The grid fixture blocks the Na population of 12 of 16 cells by an outside divalent blocker in
two modes; the Delaunay fixture blocks half of the Na populations (outside, two modes) and 80%
of the K populations (inside, three modes), so mode padding, both steepness signs and unblocked
populations in a blocked world all occur. Agreement to rounding, as the unblocked fixtures; the
same replay with the block removed misses the fixtures by far more, so the block is what the
fixtures test.
"""

import numpy as np
import pytest

from cells_b200 import worlds
from conftest import load_golden, scaled_difference
from oracle import tissue as T
from test_oracle_golden import TOL, _controls

FIXTURES = ("ars222_v3_block.npz", "ars222_v3_block_delaunay.npz")


def replay(z, b):
    topo = T.topology(b)
    ctl = _controls(z, b)
    dt = float(z["dt"])
    st, k, worst = T.initial_state(b), 0, {}
    for idx, target in enumerate(z["steps"]):
        while k < target:
            st, ok = T.ars222_step(st, dt, ctl, b, topo)
            assert ok.all(), k
            k += 1
        for f in T.State._fields:
            if "ref_" + f in z:
                worst[f] = max(worst.get(f, 0.0),
                               scaled_difference(getattr(st, f), z["ref_" + f][idx]))
    return worst


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_block_matches_the_reference(name):
    z, b = load_golden(name)
    assert b.channel_block is not None and b.channel_block.declared.any()
    worst = replay(z, b)
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, bad


@pytest.mark.parametrize("name", FIXTURES)
def test_fixture_depends_on_the_block(name):
    z, b = load_golden(name)
    b.channel_block = None
    worst = replay(z, b)
    assert worst["channel_transferred"] > 1e-3, worst["channel_transferred"]


def test_block_law_limits():
    """u = 1 and slope 0 exactly with no blocker; u -> K/(c+K) for one mode; the slope bound
    equals |du/dV| for one mode (central difference)."""
    n = 5
    v = np.linspace(-0.09, 0.03, n)
    blk = worlds.unblocked(1, n, 2)
    u, s, ok = T.channel_block(blk, 0, v, 310.0)
    assert np.all(u == 1.0) and np.all(s == 0.0) and ok.all()
    blk.weight[0, 0] = 1.0
    blk.k0_mM[0, 0] = 3.0
    blk.distance[0, 0] = 0.8
    blk.valence[0], blk.side[0], blk.concentration_mM[0] = 2, 1, 1.5
    u, s, ok = T.channel_block(blk, 0, v, 310.0)
    a = 1.6 * T.F / (T.R * 310.0)
    K = 3.0 * np.exp(a * v)
    np.testing.assert_allclose(u, K / (1.5 + K), rtol=1e-15)
    h = 1e-6
    up, _, _ = T.channel_block(blk, 0, v + h, 310.0)
    um, _, _ = T.channel_block(blk, 0, v - h, 310.0)
    np.testing.assert_allclose(s, np.abs(up - um) / (2 * h), rtol=1e-6)
