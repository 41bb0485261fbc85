"""The device RK4 step (cb_step with CB_METHOD_RK4: the reference's reference-run method,
numerics/fixed_step.py:25-71, over the held-bath step's whole right-hand side) against the
reference's own RK4 trajectory (tests/golden/rk4_grid4x4.npz, made by running the reference's
rk4_checked_step) and the oracle's RK4 (oracle/tissue.py: rk4_step, pinned bit for bit to that
fixture), at the plain step's tolerance: every field within 1e-10 scaled difference.
"""

import numpy as np
import pytest

from cells_b200 import _lib, worlds
from cells_b200.tissue import Tissue, decode_status
from conftest import load_golden, scaled_difference
from gpu_util import oracle_state
from oracle import tissue as T
from test_ros2_gpu import run, uneven_batch

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_rk4_matches_the_reference_trajectory(cuda):
    z, b = load_golden("rk4_grid4x4.npz")
    tissue = Tissue(b)
    control = tissue.pack_control()
    state, done, worst = tissue.initial_state(), 0, {}
    for idx, target in enumerate(z["steps"]):
        if target > done:
            state, status, taken = run(cuda, tissue, state, control, float(z["dt"]),
                                       [int(target - done)], method=_lib.METHOD_RK4)
            assert status[0] == 0, decode_status(status[0])
            assert taken[0] == target - done
            done = int(target)
        for f in T.State._fields:
            if "ref_" + f in z.files:
                worst[f] = max(worst.get(f, 0.0), scaled_difference(state[f], z["ref_" + f][idx]))
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, (bad, worst)


def test_rk4_matches_the_oracle_on_uneven_worlds(cuda):
    """Delaunay worlds of 16-700 cells with NaV1.2 + HH K populations, gated junctions and random
    partial controls: 200 steps of 20 us (inside RK4's stability bound for the fast gates) in two
    launches; a fused launch equals one-step launches bit for bit."""
    b, rng = uneven_batch(63)
    tissue = Tissue(b)
    mem, jun = rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges)
    pmp, chn = rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells))
    control = tissue.pack_control(mem, jun, pmp, chn)
    got, status, taken = run(cuda, tissue, tissue.initial_state(), control, 2e-5, [80, 120],
                             method=_lib.METHOD_RK4)
    assert np.all(status == 0), [decode_status(s) for s in status]
    topo = T.topology(b)
    st = T.initial_state(b)
    ctl = T.Control(mem, jun, pmp, chn)
    for _ in range(200):
        st, ok = T.rk4_step(st, 2e-5, ctl, b, topo)
        assert ok.all()
    bad = {f: d for f, r in oracle_state(st).items() if (d := scaled_difference(got[f], r)) > TOL}
    assert not bad, bad
    single, s2, _ = run(cuda, tissue, tissue.initial_state(), control, 2e-5, [1] * 20,
                        method=_lib.METHOD_RK4)
    fused, s1, _ = run(cuda, tissue, tissue.initial_state(), control, 2e-5, [20],
                       method=_lib.METHOD_RK4)
    assert np.all(s1 == 0) and np.all(s2 == 0)
    for f in fused:
        assert np.array_equal(fused[f], single[f]), f


def test_rk4_refusal_keeps_the_state(cuda):
    b = worlds.pack([worlds.single_grid_tissue(0), worlds.single_grid_tissue(1)])
    tissue = Tissue(b)
    membrane = np.ones(b.cells)
    membrane[3] = -0.5  # world 0: a negative availability
    start = tissue.initial_state()
    got, status, taken = run(cuda, tissue, start, tissue.pack_control(membrane=membrane), 1e-4,
                             [5], method=_lib.METHOD_RK4)
    assert status[0] & 8 and status[1] == 0
    assert taken[0] == 0 and taken[1] == 5
    assert np.array_equal(got["amount_increment"][:, :16], start["amount_increment"][:, :16])
