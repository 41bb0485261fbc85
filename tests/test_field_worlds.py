"""Host-side logic of the field worlds (cells_b200/field_worlds.py, cells_b200/field.py): the
lattice and the held ring, the zero charge anchors that keep every capacitor component neutral,
the shared-topology rule of a batch, and the reference definition's face factors."""

import numpy as np
import pytest

from cells_b200 import field_worlds as FW
from cells_b200 import worlds as W
from cells_b200.field import FieldTissue


def test_lattice_sits_inside_the_ring():
    nodes = FW.lattice(128, 32, 3)
    x, y = nodes % 128, nodes // 128
    assert nodes.size == 1024 and np.unique(nodes).size == 1024
    assert x.min() >= 1 and y.min() >= 1 and x.max() <= 126 and y.max() <= 126
    # no two cells share a face (stride 3)
    assert np.min(np.diff(np.unique(x))) == 3
    with pytest.raises(ValueError):
        FW.lattice(10, 5, 2)  # runs into the ring
    with pytest.raises(ValueError):
        FW.lattice(20, 3, 1)  # stride 1: neighbouring cells


def test_field_world_shapes_and_neutral_components():
    w = FW.field_world(12, 3, 3, W.world_rng(5, 0))
    assert (w.cells, w.nodes, w.faces, w.edges) == (9, 144, 2 * 12 * 11, 12)
    ring = w.reservoir
    assert ring.sum() == 4 * 11 and not np.any(ring[w.cell_node])
    # every anchor exactly zero: a cell and its node, and each lone node, carry no net charge
    assert np.all(w.initial_charge == 0.0) and np.all(w.outside_charge == 0.0)
    # the backgrounds cancel the ions' charge to the anchor rule's rounding (a few ulp of the
    # ionic sum, ~1e-24 C)
    z = W.VALENCE
    assert np.allclose(W.CHARGE_PER_FMOL * (z @ w.amount + w.fixed_charge_fmol), 0.0, atol=1e-22)
    assert np.allclose(W.CHARGE_PER_FMOL * (z @ w.outside_amount + w.outside_fixed_fmol), 0.0,
                       atol=1e-22)
    assert np.all(w.face_factor > 0)
    # the ring at the bath's concentrations, every node at the same volume
    assert np.allclose(w.outside_amount / w.outside_volume, W.BATH_mM[:, None])


def test_reference_definition_writes_the_grid():
    w = FW.field_world(10, 3, 2, W.world_rng(11, 0))
    d = FW.reference_definition(w, dt=5e-4, steps=4)
    m = d["model"]
    assert len(m["cells"]) == 9 and len(m["extracellular"]) == 100 and len(m["faces"]) == 180
    assert sum(o["reservoir"] for o in m["extracellular"]) == 36
    face = m["faces"][7]
    factor = np.asarray([face["diffusivity_m2_per_s"][s] for s in W.SPECIES]) * face["area_m2"] \
        / face["length_m"]
    assert np.array_equal(factor, w.face_factor[:, 7])
    assert m["membranes"][4]["outside"] == f"outside_{int(w.cell_node[4])}"
    assert d["execution"]["extracellular_capacity"] == 100


def test_a_batch_shares_one_topology():
    a = FW.field_world(10, 3, 2, W.world_rng(1, 0))
    b = FW.field_world(12, 3, 2, W.world_rng(1, 1))
    with pytest.raises(ValueError, match="share their topology"):
        FieldTissue([a, b])


def test_field_worlds_group_by_topology():
    """FieldBatch's grouping: worlds of one grid, tissue and contact graph share a group whatever
    their parameters; the groups keep first-appearance order and each lists its worlds ascending."""
    from cells_b200 import field as FD

    a = [FW.field_world(16, 4, 3, W.world_rng(3, k)) for k in range(3)]
    b = FW.field_world(12, 3, 3, W.world_rng(3, 9))
    gated = FW.field_world(16, 4, 3, W.world_rng(3, 7), gate=(0.015, 0.2, 1.0),
                           junction_sigma=0.3)
    assert FD.group_by_topology([a[0], b, a[1], gated, a[2]]) == [[0, 2, 3, 4], [1]]
    assert FD.group_by_topology([b]) == [[0]]
    assert FD.topology_key(a[0]) == FD.topology_key(a[2]) != FD.topology_key(b)
