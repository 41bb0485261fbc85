"""The drop-in checked step's host side (cells_b200/model.py) on the reference's own padded
pytrees: layout -> packed world, state round trips, refusals of out-of-scope layouts."""

import numpy as np
import pytest

from cells_b200 import model
from conftest import load_golden
from pytree_util import load_pytrees


def test_layout_maps_to_the_same_world():
    _, p, _, _ = load_pytrees()
    world, m = model.world_from_layout(p)
    _, b = load_golden("ars222_gated.npz")
    ref = b.world(0)
    assert m.cells.tolist() == list(range(9)) and m.bath == 0
    for name in ("volume", "area", "capacitance", "permeability", "pump_capacity",
                 "junction_area", "junction_permeability", "gate_threshold", "gate_minimum",
                 "initial_charge"):
        assert np.array_equal(getattr(world, name), getattr(ref, name)), name
    assert np.array_equal(world.sender, ref.sender)
    assert np.array_equal(world.receiver, ref.receiver)
    assert np.allclose(world.amount, ref.amount, rtol=0, atol=0)
    assert world.bath_potential == ref.bath_potential
    assert world.pump == ref.pump


def test_channel_layout_maps_to_the_same_world():
    _, p, _, _ = load_pytrees("pytrees_v3_channels_padded.npz")
    world, m = model.world_from_layout(p)
    _, b = load_golden("ars222_v3_channels_delaunay.npz")
    ref = b.world(0)
    assert m.nch == 2
    for name in ("channel_code", "channel_species", "channel_permeability",
                 "channel_abundance", "permeability", "junction_permeability", "sender"):
        assert np.array_equal(getattr(world, name), getattr(ref, name)), name


def test_block_layout_maps_to_the_same_block():
    """The reference's block layout fields of a padded @3 layout give the block of the world
    they were made from: the same weights, K(0), concentrations and signed steepness."""
    _, p, _, _ = load_pytrees("pytrees_v3_block_padded.npz")
    world, m = model.world_from_layout(p)
    _, b = load_golden("ars222_v3_block_delaunay.npz")
    got, want = world.channel_block, b.channel_block
    assert got is not None and got.modes == want.modes
    for name in ("weight", "k0_mM", "concentration_mM", "steepness"):
        assert np.array_equal(getattr(got, name), getattr(want, name)), name
    assert np.array_equal(got.declared, want.declared)


@pytest.mark.parametrize("name", ["pytrees_gated_padded.npz", "pytrees_v3_channels_padded.npz",
                                  "pytrees_v3_block_padded.npz"])
def test_state_round_trip_keeps_padding(name):
    _, p, _, states = load_pytrees(name)
    _, m = model.world_from_layout(p)
    for st in states:
        packed = model.packed_state(st, m)
        back = model.reference_state(packed, st, m)
        for f in st._fields:
            assert np.array_equal(np.asarray(getattr(back, f)), np.asarray(getattr(st, f))), f


def test_out_of_scope_layouts_are_refused():
    _, p, _, _ = load_pytrees()
    faces = np.asarray(p.face_active).copy()
    faces[0] = True
    with pytest.raises(model.Unsupported):
        model.world_from_layout(p._replace(face_active=faces))
    channels = np.ones(max(1, np.asarray(p.channel_active).size), dtype=bool)
    with pytest.raises(model.Unsupported):
        model.world_from_layout(p._replace(channel_active=channels))
    outside = np.asarray(p.outside_active).copy()
    outside[1] = True  # a finite, unheld outside node
    with pytest.raises(model.Unsupported):
        model.world_from_layout(p._replace(outside_active=outside))


def test_layouts_with_other_options_are_refused():
    """A layout that declares an option outside the device step (a voltage shift, forms faces,
    loops, one-way records, series junction gates, a present Ca pump) is refused, so the stub
    keeps the reference's own step for it."""
    from collections import namedtuple

    _, p, _, _ = load_pytrees("pytrees_v3_block_padded.npz")
    for field in model.OPTION_FIELDS:
        With = namedtuple("Layout", (*p._fields, field))
        with pytest.raises(model.Unsupported):
            model.world_from_layout(With(*p, np.zeros(1)))
    With = namedtuple("Layout", (*p._fields, "calcium_pump_present"))
    model.world_from_layout(With(*p, np.zeros(3, dtype=bool)))  # declared slots, none present
    with pytest.raises(model.Unsupported, match="Ca pumps"):
        model.world_from_layout(With(*p, np.array([False, True, False])))


def test_layout_declares_its_solver():
    _, p, _, _ = load_pytrees("pytrees_n2_padded.npz")
    assert model.layout_solver(p) == model.N2_ID
    world, m = model.world_from_layout(p)
    assert m.nch == 2
    _, p1, _, _ = load_pytrees()
    assert model.layout_solver(p1) == model.ARS222_ID
