"""Synthetic tissue generators and packing (cells_b200/worlds.py)."""

import math

import numpy as np

from cells_b200 import worlds


def test_grid_world_shape_and_units():
    w = worlds.single_grid_tissue(0)
    assert w.cells == 16 and w.edges == 24
    assert np.allclose(w.area, 4 * math.pi * 25e-12)
    assert np.allclose(w.capacitance, 0.01 * w.area)
    assert np.allclose(w.volume, 4 / 3 * math.pi * 125e-18 * 1e15)
    conc = w.amount / w.volume
    assert np.all((conc[0] >= 10) & (conc[0] <= 15))
    assert np.all((conc[1] >= 130) & (conc[1] <= 145))
    assert np.all((conc[2] >= 5) & (conc[2] <= 20))
    # Fixed anions set for electroneutrality: the anchor charge is rounding-level.
    assert np.all(np.abs(w.initial_charge) < 1e-23)  # a few ulps of the ionic charge


def test_seeded_worlds_are_reproducible_and_independent():
    a = worlds.grid_tissues(3, side=4, seed=5)
    b = worlds.grid_tissues(3, side=4, seed=5)
    for x, y in zip(a, b, strict=True):
        assert np.array_equal(x.permeability, y.permeability)
    assert not np.array_equal(a[0].permeability, a[1].permeability)


def test_delaunay_world_degree():
    w = worlds.delaunay_world(400, worlds.world_rng(3, 0))
    deg = 2 * w.edges / w.cells
    assert 5.0 < deg < 6.2
    assert np.all(w.sender < w.receiver)


def test_pack_roundtrip():
    ws = [worlds.grid_world(3, 4, worlds.world_rng(1, k)) for k in range(3)]
    b = worlds.pack(ws)
    assert b.worlds == 3 and b.cells == 36 and b.edges == 3 * 17
    back = b.world(1)
    assert np.array_equal(back.permeability, ws[1].permeability)
    assert np.array_equal(back.sender, ws[1].sender)


def test_uneven_sizes_log_uniform():
    sizes = worlds.uneven_sizes(1024)
    assert sizes.min() >= 32 and sizes.max() <= 4096
    assert 600 < sizes.mean() < 1100
