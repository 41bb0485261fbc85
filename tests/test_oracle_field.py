"""The resolved-field oracle (oracle/field.py) against the reference's own step on field worlds
(tests/golden/field_*.npz: cells facing a 10x10, 14x14 or 24x24 extracellular grid with a held
ring, @1 ARS(2,2,2) with face electromigration and the factored field solver).

The restatement follows the reference's arithmetic order, so every field is expected bit for
bit; the test allows 1e-15 scaled difference (BLAS may block a product differently on another
host). BLAS runs on one thread, as the reference pins it (execution/blas_threads.py:28-45): a
threaded dense product or solve changes the last bits with the thread count.
"""

import numpy as np
import pytest
import threadpoolctl

from conftest import load_field_golden, scaled_difference
from oracle import field as OF

TOL = 1e-15


@pytest.fixture(autouse=True)
def one_blas_thread():
    with threadpoolctl.threadpool_limits(limits=1, user_api="blas"):
        yield


@pytest.mark.parametrize("name", ["field_grid10.npz", "field_gated14.npz", "field_grid24.npz"])
def test_field_oracle_matches_the_reference(name):
    z, w = load_field_golden(name)
    tp = OF.bind(w)
    control = OF.Control(z["control_membrane"], z["control_junction"], z["control_pump"])
    dt = float(z["dt"])
    state, done, worst = OF.initial_state(w), 0, {}
    for idx, target in enumerate(z["steps"]):
        while done < target:
            state, ok = OF.imex_step(state, dt, control, w, tp)
            assert ok, done
            done += 1
        for f in OF.FieldState._fields:
            worst[f] = max(worst.get(f, 0.0), scaled_difference(getattr(state, f),
                                                                z["ref_" + f][idx]))
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, bad


def test_field_components_and_incidences():
    """bind's reduction on the 10x10 world: one floating component per interior node (each cell
    joins its node's), representatives at the nodes, the ring held."""
    _, w = load_field_golden("field_grid10.npz")
    tp = OF.bind(w)
    interior = int(np.sum(~w.reservoir))
    assert tp.basis.shape == (w.cells + w.nodes, interior)
    assert np.all(tp.basis.sum(axis=0) >= 1)
    assert np.all(tp.fixed[w.cells + np.flatnonzero(w.reservoir)])
    assert not np.any(tp.fixed[:w.cells])
    # Each face touches at most two components; a face between two ring nodes touches none.
    assert np.all(np.abs(tp.face_incidence).sum(axis=0) <= 2)


def test_field_step_refuses_an_invalid_control_and_keeps_the_state():
    z, w = load_field_golden("field_grid10.npz")
    tp = OF.bind(w)
    control = OF.Control(np.full(w.cells, 1.2), np.ones(w.edges), np.ones(w.cells))
    start = OF.initial_state(w)
    state, ok = OF.imex_step(start, 5e-4, control, w, tp)
    assert not ok
    for a, b in zip(state, start, strict=True):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["field_grid10.npz", "field_gated14.npz"])
def test_sparse_restatement_matches_the_reference(name):
    """bind(w, sparse=True): the same algebra in scipy.sparse containers with sparse LU solves
    (what the 128x128 benchmark grid needs) reproduces the reference's trajectories to rounding
    accumulated over the runs (1e-11 scaled over up to 200 steps, ten times inside the device
    bar)."""
    z, w = load_field_golden(name)
    tp = OF.bind(w, sparse=True)
    control = OF.Control(z["control_membrane"], z["control_junction"], z["control_pump"])
    dt = float(z["dt"])
    state, done, worst = OF.initial_state(w), 0, {}
    for idx, target in enumerate(z["steps"]):
        while done < target:
            state, ok = OF.imex_step(state, dt, control, w, tp)
            assert ok, done
            done += 1
        for f in OF.FieldState._fields:
            worst[f] = max(worst.get(f, 0.0), scaled_difference(getattr(state, f),
                                                                z["ref_" + f][idx]))
    bad = {k: v for k, v in worst.items() if v > 1e-11}
    assert not bad, (bad, worst)
