"""Seeded synthetic pump-leak tissues, packed structure-of-arrays for the device step.

A *world* is one tissue: N cells, each with one membrane patch facing a held bath (a reservoir
outside node clamped at a boundary potential), E gap junctions between cells, Na/K/Cl with
valences +1/+1/-1, a Na/K-ATPase on every patch, and junction gates of the reference's
voltage-relaxation law. Worlds never interact. A *batch* packs W worlds of possibly different
sizes back to back: world w owns cells ``cell_offset[w]:cell_offset[w+1]`` and junctions
``edge_offset[w]:edge_offset[w+1]``; junction endpoints are world-local cell indices.

Units follow the reference's definition schema (models/surface_tissue.py:135-257): volumes in
pL, amounts in fmol, areas in m^2, permeabilities in m/s, capacitances in F, temperature in K,
potentials in V. Pump parameters follow laws/pumps/nak_atp_mass_action_positive.py:36-50.

The shapes are the pump-leak tissues of the benchmark suite: a square grid with 4-neighbour
junctions (16 cells for the single CPU world, 16x16 for the batched plain step), and Delaunay
contact graphs of Poisson-disk points for uneven batches. ``reference_definition`` writes one
world in the reference's JSON schema so that its own parser and step can run it.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SPECIES = ("Na", "K", "Cl")
VALENCE = np.array([1.0, 1.0, -1.0])
SODIUM, POTASSIUM = 0, 1
STOICHIOMETRY = np.array([-3.0, 2.0, 0.0])  # Inward-positive per cycle (Na out, K in).

# Constants of laws/electrochemistry.py:11-15 (same expressions, so the same doubles).
AVOGADRO = 6.02214076e23
F = AVOGADRO * 1.602176634e-19
R = AVOGADRO * 1.380649e-23
MOL_PER_FMOL = 1e-15
CHARGE_PER_FMOL = F * MOL_PER_FMOL

# The benchmark tissue's laws (cm/s figures converted to m/s).
CELL_RADIUS_M = 5e-6
SPECIFIC_CAPACITANCE_F_M2 = 0.01  # 1 uF/cm^2
TEMPERATURE_K = 310.15  # 37 C
BATH_mM = np.array([145.0, 5.0, 110.0])
BATH_VOLUME_PL = 1.0e4
LEAK_MEDIAN_M_S = np.array([1e-12, 1e-10, 1e-11])  # P_Na 1e-10, P_K 1e-8, P_Cl 1e-9 cm/s
LEAK_SIGMA = 0.3
JUNCTION_M_S = 1e-9  # 1e-7 cm/s
JUNCTION_AREA_M2 = 1e-11  # Not given by the benchmark: declared here.
INITIAL_mM_RANGES = np.array([[10.0, 15.0], [130.0, 145.0], [5.0, 20.0]])
# Pump constants of the reference's configs/resolved_pump_tissue.json. The benchmark gives no pump
# capacity; that file's density (0.02 fmol/s on 4e-10 m^2) is about 300 times the Na leak of the
# benchmark's permeabilities and drives its tissues toward -150 mV. Declared here: a density
# that balances those leaks, resting the tissues at -70 to -80 mV.
PUMP_CAPACITY_PER_M2 = 5e5
PUMP_KM_NA, PUMP_KM_K, PUMP_KM_ATP = 12.0, 0.2, 0.5
PUMP_ATP, PUMP_ADP, PUMP_PI = 1.5, 0.1, 0.1
PUMP_DG0 = -37000.0


@dataclass
class World:
    """One tissue, host arrays, world-local indices."""

    volume: np.ndarray  # [N] pL
    area: np.ndarray  # [N] m^2 (the cell's one membrane patch)
    capacitance: np.ndarray  # [N] F
    permeability: np.ndarray  # [S, N] m/s
    pump_capacity: np.ndarray  # [N] fmol cycles/s
    amount: np.ndarray  # [S, N] fmol, initial
    fixed_charge_fmol: np.ndarray  # [N] fixed background, charge-equivalent fmol
    initial_charge: np.ndarray  # [N] C
    sender: np.ndarray  # [E] int
    receiver: np.ndarray  # [E] int
    junction_area: np.ndarray  # [E] m^2
    junction_permeability: np.ndarray  # [S, E] m/s
    gate_threshold: np.ndarray  # [E] V
    gate_minimum: np.ndarray  # [E]
    gate_initial: np.ndarray  # [E]
    temperature: float = TEMPERATURE_K
    # Voltage-gated channel populations: NCH slots per cell ([NCH, N]; NCH = 0 for none).
    # Law codes: 0 Kv1.5 m h, 2 NaV1.2 m^3 h (the reference's catalogue codes), 100 the
    # Hodgkin-Huxley K n^4 law of this package (channels.HH_K_N4).
    channel_code: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), dtype=np.int32))
    channel_species: np.ndarray = field(default_factory=lambda: np.zeros((0, 0), dtype=np.int32))
    channel_permeability: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))
    channel_abundance: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))
    channel_gate_initial: np.ndarray = field(default_factory=lambda: np.zeros((2, 0, 0)))
    bath_mM: np.ndarray = field(default_factory=lambda: BATH_mM.copy())
    # The populations' open-channel block ([M, NCH, N] modes), or None for none.
    channel_block: ChannelBlock | None = None
    # Cell centres in the unit square ([2, N]), for spatial patterns over the tissue (the
    # adjoint benchmark's voltage target); empty when the builder has no geometry.
    position: np.ndarray = field(default_factory=lambda: np.zeros((2, 0)))
    bath_volume: float = BATH_VOLUME_PL
    bath_potential: float = 0.0
    pump: tuple = (PUMP_ATP, PUMP_ADP, PUMP_PI, PUMP_KM_NA, PUMP_KM_K, PUMP_KM_ATP, PUMP_DG0)

    @property
    def cells(self):
        return self.volume.size

    @property
    def edges(self):
        return self.sender.size

    @property
    def channel_slots(self):
        return int(self.channel_code.shape[0]) if self.channel_code.size else 0


BLOCK_LAW_ID = "cells.channel_block.open_channel_block_weighted_modes@1"
BLOCK_SIDES = {"outside": 1, "inside": -1}  # s in a_k = s sgn(z_B) m_k F/(R T)


@dataclass
class ChannelBlock:
    """Open-channel block of the channel populations (the reference's FR-51 block,
    laws/channels/open_channel_block.py), over the cells of one world or a batch. Arrays
    [M, NCH, N] per mode slot, [NCH, N] per population. A population that declares no block holds
    weights (1, 0, ...), K(0) 1, distance 0 and concentration 0, the reference's layout for it
    (surface_pump_v3.block_initial_values :599-615), so its u is exactly 1; mode slots past a
    population's own modes hold weight 0, K(0) 1, distance 0."""

    declared: np.ndarray          # [NCH, N] bool: the population declares a block
    weight: np.ndarray            # [M, NCH, N]
    k0_mM: np.ndarray             # [M, NCH, N]
    distance: np.ndarray          # [M, NCH, N] electrical distance delta_k (or, for a unit
                                  # valence, the effective valence m_k)
    modes_declared: np.ndarray    # [NCH, N] int: the population's own mode count
    valence: np.ndarray           # [NCH, N] int: the blocker's valence z_B
    side: np.ndarray              # [NCH, N] int: +1 outside, -1 inside
    concentration_mM: np.ndarray  # [NCH, N]

    @property
    def modes(self):
        return int(self.weight.shape[0])

    @property
    def steepness(self):
        """[M, NCH, N] the signed steepness s sgn(z_B) |z_B| delta_k (ChannelBlock.steepness of
        definitions/surface_pump_v3_spec.py, in its order of operations)."""
        sign = self.side * np.where(self.valence > 0, 1, -1)
        return sign * (np.abs(self.valence) * self.distance)

    def cells(self, a, b):
        """The block of cells a..b (a view)."""
        return ChannelBlock(self.declared[:, a:b], self.weight[..., a:b], self.k0_mM[..., a:b],
                            self.distance[..., a:b], self.modes_declared[:, a:b],
                            self.valence[:, a:b], self.side[:, a:b],
                            self.concentration_mM[:, a:b])

    def padded(self, modes):
        """The same block with ``modes`` mode slots (>= its own)."""
        extra = modes - self.modes
        if extra == 0:
            return self
        shape = (extra,) + self.weight.shape[1:]
        return ChannelBlock(self.declared,
                            np.concatenate([self.weight, np.zeros(shape)]),
                            np.concatenate([self.k0_mM, np.ones(shape)]),
                            np.concatenate([self.distance, np.zeros(shape)]),
                            self.modes_declared, self.valence, self.side, self.concentration_mM)


def unblocked(nch, n, modes=1):
    """The layout of populations that declare no block."""
    weight = np.zeros((modes, nch, n))
    weight[0] = 1.0
    return ChannelBlock(np.zeros((nch, n), dtype=bool), weight, np.ones((modes, nch, n)),
                        np.zeros((modes, nch, n)), np.zeros((nch, n), dtype=np.int64),
                        np.ones((nch, n), dtype=np.int64), np.ones((nch, n), dtype=np.int64),
                        np.zeros((nch, n)))


def with_block(world, rng, *, slot=0, fraction=1.0, valence=2, side="outside",
               concentration_mM=(0.5, 2.0), modes=((0.625, 3.0, 0.8), (0.375, 30.0, 0.4))):
    """Block the population in ``slot`` of a fraction of the cells by a held blocker of the given
    valence and side (the default: an outside divalent blocker, Mg2+-like): concentration
    log-uniform in ``concentration_mM``; ``modes`` as (weight, K(0) mM, electrical distance),
    each K(0) scaled per cell by a log-uniform factor in [0.5, 2]. The weights must sum to 1."""
    nch, n = world.channel_slots, world.cells
    if nch == 0:
        raise ValueError("the world has no channel populations")
    m = len(modes)
    if world.channel_block is None:
        blk = unblocked(nch, n, m)
    else:  # another slot's block is kept; the mode axis grows to the larger count
        old = world.channel_block
        blk = old.padded(max(m, old.modes))
        blk = ChannelBlock(*(np.array(getattr(blk, f)) for f in (
            "declared", "weight", "k0_mM", "distance", "modes_declared", "valence", "side",
            "concentration_mM")))
    cells = rng.random(n) < fraction
    lo, hi = np.log(concentration_mM[0]), np.log(concentration_mM[1])
    conc = np.exp(rng.uniform(lo, hi, n))
    scale = np.exp(rng.uniform(np.log(0.5), np.log(2.0), (m, n)))
    for i in np.flatnonzero(cells):
        blk.declared[slot, i] = True
        blk.modes_declared[slot, i] = m
        blk.valence[slot, i] = valence
        blk.side[slot, i] = BLOCK_SIDES[side]
        blk.concentration_mM[slot, i] = conc[i]
        blk.weight[:, slot, i], blk.k0_mM[:, slot, i], blk.distance[:, slot, i] = 0.0, 1.0, 0.0
        for k, (w, k0, delta) in enumerate(modes):
            blk.weight[k, slot, i] = w
            blk.k0_mM[k, slot, i] = k0 * scale[k, i]
            blk.distance[k, slot, i] = delta
    world.channel_block = blk
    return world


def block_declaration(block, k, i):
    """The reference's declaration of the block of population k of cell i (the channel entry's
    "block" key, definitions/surface_pump_v3_spec.parse_block), or None."""
    if block is None or not block.declared[k, i]:
        return None
    side = {v: key for key, v in BLOCK_SIDES.items()}[int(block.side[k, i])]
    return {
        "law": BLOCK_LAW_ID,
        "blocker": {"id": f"blocker_{k}_{i}", "valence": int(block.valence[k, i]),
                    "side": side, "concentration_mM": float(block.concentration_mM[k, i])},
        "modes": [{"weight": float(block.weight[j, k, i]), "k0_mM": float(block.k0_mM[j, k, i]),
                   "electrical_distance": float(block.distance[j, k, i])}
                  for j in range(int(block.modes_declared[k, i]))],
    }


CHANNEL_LAW_IDS = {
    0: "cells.channel.kv1p5_mh@1",
    2: "cells.channel.nav1p2_m3h_regularized@1",
    100: "cells_b200.channel.hh_k_n4@1",
}


def with_channels(world, rng, *, na=("nav", 2e-10, 0.5), k=("kv", 3e-10, 0.5), sigma=0.0):
    """Give every cell a Na population and a K population. ``na``/``k``: (law, permeability
    m/s, abundance); laws "nav" (NaV1.2 m^3 h), "kv" (Kv1.5 m h) or "hh" (HH K n^4). Initial gates
    at the laws' steady state near -60 mV, as fixed values."""
    n = world.cells
    codes = {"nav": 2, "kv": 0, "hh": 100}
    gate0 = {"nav": (0.05, 0.6), "kv": (0.2, 0.7), "hh": (0.32, 0.0)}
    code = np.array([[codes[na[0]]] * n, [codes[k[0]]] * n], dtype=np.int32)
    species = np.array([[SODIUM] * n, [POTASSIUM] * n], dtype=np.int32)
    perm = np.array([[na[1]] * n, [k[1]] * n], dtype=float)
    if sigma:
        perm = perm * np.exp(sigma * rng.standard_normal(perm.shape))
    abundance = np.array([[na[2]] * n, [k[2]] * n], dtype=float)
    gates = np.zeros((2, 2, n))
    for slot, law in enumerate((na[0], k[0])):
        gates[0, slot], gates[1, slot] = gate0[law]
    world.channel_code, world.channel_species = code, species
    world.channel_permeability, world.channel_abundance = perm, abundance
    world.channel_gate_initial = gates
    return world


def anchor_charge(amount, fixed):
    """Charge anchor (C) as the reference's definition check forms it
    (models/surface_tissue.py:484-486): F * fsum(fixed, z n)."""
    out = np.empty(amount.shape[1])
    for i in range(amount.shape[1]):
        terms = [z * a for z, a in zip(VALENCE, amount[:, i], strict=True)]
        out[i] = CHARGE_PER_FMOL * math.fsum((float(fixed[i]), *terms))
    return out


def grid_edges(nx, ny):
    """4-neighbour junctions of an nx-by-ny grid, row-major cells, each pair once."""
    senders, receivers = [], []
    for y in range(ny):
        for x in range(nx):
            i = y * nx + x
            if x + 1 < nx:
                senders.append(i)
                receivers.append(i + 1)
            if y + 1 < ny:
                senders.append(i)
                receivers.append(i + nx)
    return np.asarray(senders, dtype=np.int64), np.asarray(receivers, dtype=np.int64)


def _cells(rng, n):
    radius = CELL_RADIUS_M
    area = np.full(n, 4.0 * math.pi * radius**2)
    volume = np.full(n, 4.0 / 3.0 * math.pi * radius**3 * 1e15)  # m^3 -> pL
    capacitance = SPECIFIC_CAPACITANCE_F_M2 * area
    permeability = LEAK_MEDIAN_M_S[:, None] * np.exp(LEAK_SIGMA * rng.standard_normal((3, n)))
    lo, hi = INITIAL_mM_RANGES[:, 0:1], INITIAL_mM_RANGES[:, 1:2]
    conc = lo + (hi - lo) * rng.random((3, n))
    amount = conc * volume
    # Fixed anions set for electroneutrality: the background cancels the mobile ions' charge.
    fixed = -(VALENCE @ amount)
    return volume, area, capacitance, permeability, amount, fixed


def grid_world(nx, ny, rng, *, junction_sigma=0.0, gate=None):
    """A pump-leak tissue on an nx-by-ny grid (the benchmark's square tissues)."""
    n = nx * ny
    volume, area, capacitance, permeability, amount, fixed = _cells(rng, n)
    sender, receiver = grid_edges(nx, ny)
    world = _assemble(
        volume, area, capacitance, permeability, amount, fixed, sender, receiver, rng,
        junction_sigma=junction_sigma, gate=gate,
    )  # fmt: skip
    ix, iy = np.arange(n) % nx, np.arange(n) // nx
    world.position = np.stack(((ix + 0.5) / nx, (iy + 0.5) / ny))
    return world


def _assemble(
    volume, area, capacitance, permeability, amount, fixed, sender, receiver, rng, *,
    junction_sigma, gate,
):  # fmt: skip
    e = sender.size
    jp = np.full((3, e), JUNCTION_M_S)
    if junction_sigma:
        jp = jp * np.exp(junction_sigma * rng.standard_normal(e))[None, :]
    if gate is None:  # Pinned open: minimum open fraction 1 keeps g = 1 exactly.
        threshold, minimum, initial = np.full(e, 0.015), np.ones(e), np.ones(e)
    else:
        threshold, minimum, initial = (np.full(e, v) for v in gate)
    return World(
        volume=volume,
        area=area,
        capacitance=capacitance,
        permeability=permeability,
        pump_capacity=PUMP_CAPACITY_PER_M2 * area,
        amount=amount,
        fixed_charge_fmol=fixed,
        initial_charge=anchor_charge(amount, fixed),
        sender=sender,
        receiver=receiver,
        junction_area=np.full(e, JUNCTION_AREA_M2),
        junction_permeability=jp,
        gate_threshold=threshold,
        gate_minimum=minimum,
        gate_initial=initial,
    )


def poisson_disk(rng, n):
    """n blue-noise points in the unit square with a minimum spacing: a jittered m-by-m grid
    (each point uniform within the central 0.7 of its grid cell, so any two points are at least
    0.3 cell apart), m = ceil(sqrt(1.3 n)), of which a random n are kept. Vectorised, so a batch
    of a million cells builds in seconds."""
    m = int(math.ceil(math.sqrt(1.3 * n)))
    ix, iy = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    jitter = 0.15 + 0.7 * rng.random((2, m * m))
    pts = np.stack(((ix.ravel() + jitter[0]) / m, (iy.ravel() + jitter[1]) / m), axis=1)
    keep = rng.choice(m * m, size=n, replace=False)
    return pts[np.sort(keep)]


def delaunay_edges(points):
    from scipy.spatial import Delaunay

    tri = Delaunay(points)
    pairs = set()
    for a, b, c in tri.simplices:
        for u, v in ((a, b), (b, c), (a, c)):
            pairs.add((min(u, v), max(u, v)))
    pairs = np.asarray(sorted(pairs), dtype=np.int64)
    return pairs[:, 0], pairs[:, 1]


def delaunay_world(n, rng, *, junction_sigma=0.3, gate=None):
    """A pump-leak tissue whose contact graph is the Delaunay triangulation of Poisson-disk
    points (mean degree about 6), junction permeabilities log-normal."""
    volume, area, capacitance, permeability, amount, fixed = _cells(rng, n)
    points = poisson_disk(rng, n)
    sender, receiver = delaunay_edges(points)
    world = _assemble(
        volume, area, capacitance, permeability, amount, fixed, sender, receiver, rng,
        junction_sigma=junction_sigma, gate=gate,
    )  # fmt: skip
    world.position = points.T.copy()
    return world


def world_rng(seed, world):
    """Independent stream per (seed, world id)."""
    return np.random.default_rng([int(seed), int(world)])


def single_grid_tissue(seed=0):
    """The single CPU world: 16 cells on a 4x4 grid."""
    return grid_world(4, 4, world_rng(seed, 0))


def grid_tissues(worlds, side=16, seed=1):
    """The batched plain step: ``worlds`` independent side-by-side grid tissues."""
    return [grid_world(side, side, world_rng(seed, w)) for w in range(worlds)]


def uneven_sizes(worlds, lo=32, hi=4096, seed=2):
    rng = np.random.default_rng([int(seed), 1 << 20])
    return np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), worlds))).astype(np.int64)


def uneven_world(w, size, seed=2, channels=None):
    """World w (of cell count ``size``) of the uneven batch, as delaunay_tissues builds it."""
    rng = world_rng(seed, w)
    world = delaunay_world(int(size), rng)
    if channels is not None:
        world = with_channels(world, rng, **channels)
    return world


def delaunay_tissues(worlds, lo=32, hi=4096, seed=2, channels=None):
    """Uneven batch: cell counts log-uniform in [lo, hi], Delaunay contact graphs, log-normal
    junction permeabilities; worlds ordered largest first (work items pack consecutive worlds).
    ``channels``: None, or with_channels' keywords (a Na and a K population per cell)."""
    sizes = np.sort(uneven_sizes(worlds, lo, hi, seed))[::-1]
    return [uneven_world(w, n, seed, channels) for w, n in enumerate(sizes)]


# The uneven batch's channel populations: NaV1.2 (m^3 h) and Hodgkin-Huxley K (n^4), log-normal
# permeabilities (sigma 0.3); values declared here (the benchmark names the laws, not densities).
UNEVEN_CHANNELS = dict(na=("nav", 1e-9, 0.5), k=("hh", 5e-10, 0.5), sigma=0.3)


# --------------------------------------------------------------------------------------------
# Packing


@dataclass
class Batch:
    """W worlds packed back to back (structure of arrays, float64 unless noted)."""

    cell_offset: np.ndarray  # [W+1] int64
    edge_offset: np.ndarray  # [W+1] int64
    temperature: np.ndarray  # [W]
    bath_amount: np.ndarray  # [S, W] fmol (held reservoir reference amounts)
    bath_volume: np.ndarray  # [W] pL
    bath_potential: np.ndarray  # [W] V
    pump: np.ndarray  # [7, W]: atp, adp, pi, km_na, km_k, km_atp (mM), delta_g0 (J/mol)
    volume: np.ndarray  # [C]
    area: np.ndarray  # [C]
    capacitance: np.ndarray  # [C]
    permeability: np.ndarray  # [S, C]
    pump_capacity: np.ndarray  # [C]
    amount_reference: np.ndarray  # [S, C]
    initial_charge: np.ndarray  # [C]
    sender: np.ndarray  # [E] int32, world-local
    receiver: np.ndarray  # [E] int32, world-local
    junction_area: np.ndarray  # [E]
    junction_permeability: np.ndarray  # [S, E]
    gate_threshold: np.ndarray  # [E]
    gate_minimum: np.ndarray  # [E]
    gate_initial: np.ndarray  # [E]
    channel_code: np.ndarray = None  # [NCH, C] int32 (NCH = 0: no channel populations)
    channel_species: np.ndarray = None  # [NCH, C] int32
    channel_permeability: np.ndarray = None  # [NCH, C] m/s (max permeability x relative)
    channel_abundance: np.ndarray = None  # [NCH, C]
    channel_gate_initial: np.ndarray = None  # [2, NCH, C]
    position: np.ndarray = None  # [2, C] cell centres in each world's unit square (zeros: none)
    channel_block: ChannelBlock | None = None  # over the batch's cells; None: no block

    def __post_init__(self):
        c = self.cells
        if self.channel_code is None:
            self.channel_code = np.zeros((0, c), dtype=np.int32)
            self.channel_species = np.zeros((0, c), dtype=np.int32)
            self.channel_permeability = np.zeros((0, c))
            self.channel_abundance = np.zeros((0, c))
            self.channel_gate_initial = np.zeros((2, 0, c))
        if self.position is None:
            self.position = np.zeros((2, c))

    @property
    def channel_slots(self):
        return int(self.channel_code.shape[0])

    @property
    def worlds(self):
        return self.cell_offset.size - 1

    @property
    def cells(self):
        return int(self.cell_offset[-1])

    @property
    def edges(self):
        return int(self.edge_offset[-1])

    def world(self, w):
        """World w back as a World (host views)."""
        c0, c1 = self.cell_offset[w], self.cell_offset[w + 1]
        e0, e1 = self.edge_offset[w], self.edge_offset[w + 1]
        return World(
            volume=self.volume[c0:c1],
            area=self.area[c0:c1],
            capacitance=self.capacitance[c0:c1],
            permeability=self.permeability[:, c0:c1],
            pump_capacity=self.pump_capacity[c0:c1],
            amount=self.amount_reference[:, c0:c1],
            fixed_charge_fmol=-(VALENCE @ self.amount_reference[:, c0:c1]),
            initial_charge=self.initial_charge[c0:c1],
            sender=self.sender[e0:e1].astype(np.int64),
            receiver=self.receiver[e0:e1].astype(np.int64),
            junction_area=self.junction_area[e0:e1],
            junction_permeability=self.junction_permeability[:, e0:e1],
            gate_threshold=self.gate_threshold[e0:e1],
            gate_minimum=self.gate_minimum[e0:e1],
            gate_initial=self.gate_initial[e0:e1],
            temperature=float(self.temperature[w]),
            channel_code=self.channel_code[:, c0:c1],
            channel_species=self.channel_species[:, c0:c1],
            channel_permeability=self.channel_permeability[:, c0:c1],
            channel_abundance=self.channel_abundance[:, c0:c1],
            channel_gate_initial=self.channel_gate_initial[:, :, c0:c1],
            position=self.position[:, c0:c1],
            channel_block=(None if self.channel_block is None
                           else self.channel_block.cells(c0, c1)),
            bath_mM=self.bath_amount[:, w] / self.bath_volume[w],
            bath_volume=float(self.bath_volume[w]),
            bath_potential=float(self.bath_potential[w]),
            pump=tuple(float(v) for v in self.pump[:, w]),
        )


def pack(worlds):
    """Pack a list of World into one Batch."""
    cells = np.array([w.cells for w in worlds], dtype=np.int64)
    edges = np.array([w.edges for w in worlds], dtype=np.int64)
    slots = {w.channel_slots for w in worlds}
    if len(slots) != 1:
        raise ValueError("every world of a batch needs the same number of channel slots")
    nch = slots.pop()
    cat = np.concatenate

    def cells_of(name):
        return cat([getattr(w, name) for w in worlds], axis=-1)

    return Batch(
        cell_offset=np.r_[0, np.cumsum(cells)].astype(np.int64),
        edge_offset=np.r_[0, np.cumsum(edges)].astype(np.int64),
        temperature=np.array([w.temperature for w in worlds]),
        bath_amount=np.stack([w.bath_mM * w.bath_volume for w in worlds], axis=1),
        bath_volume=np.array([w.bath_volume for w in worlds]),
        bath_potential=np.array([w.bath_potential for w in worlds]),
        pump=np.array([w.pump for w in worlds], dtype=float).T.copy(),
        volume=cells_of("volume"),
        area=cells_of("area"),
        capacitance=cells_of("capacitance"),
        permeability=cells_of("permeability"),
        pump_capacity=cells_of("pump_capacity"),
        amount_reference=cells_of("amount"),
        initial_charge=cells_of("initial_charge"),
        sender=cells_of("sender").astype(np.int32),
        receiver=cells_of("receiver").astype(np.int32),
        junction_area=cells_of("junction_area"),
        junction_permeability=cells_of("junction_permeability"),
        gate_threshold=cells_of("gate_threshold"),
        gate_minimum=cells_of("gate_minimum"),
        gate_initial=cells_of("gate_initial"),
        channel_code=(cells_of("channel_code").astype(np.int32) if nch
                      else np.zeros((0, int(cells.sum())), dtype=np.int32)),
        channel_species=(cells_of("channel_species").astype(np.int32) if nch
                         else np.zeros((0, int(cells.sum())), dtype=np.int32)),
        channel_permeability=(cells_of("channel_permeability") if nch
                              else np.zeros((0, int(cells.sum())))),
        channel_abundance=(cells_of("channel_abundance") if nch
                           else np.zeros((0, int(cells.sum())))),
        channel_gate_initial=(cells_of("channel_gate_initial") if nch
                              else np.zeros((2, 0, int(cells.sum())))),
        position=cat([w.position if w.position.shape == (2, w.cells) else np.zeros((2, w.cells))
                      for w in worlds], axis=1),
        channel_block=_pack_blocks(worlds, nch),
    )


def _pack_blocks(worlds, nch):
    """The worlds' blocks over the batch's cells (padded to the most modes), or None where no
    world declares one."""
    blocks = [w.channel_block for w in worlds]
    if all(b is None for b in blocks):
        return None
    modes = max(b.modes for b in blocks if b is not None)
    parts = [(unblocked(nch, w.cells, modes) if b is None else b.padded(modes))
             for w, b in zip(worlds, blocks, strict=True)]
    cat = np.concatenate
    return ChannelBlock(*(cat([getattr(p, f) for p in parts], axis=-1) for f in
                          ("declared", "weight", "k0_mM", "distance", "modes_declared",
                           "valence", "side", "concentration_mM")))


# --------------------------------------------------------------------------------------------
# The adjoint benchmark's voltage target

TARGET_BASELINE_V = -0.050
TARGET_BUMP_V = 0.020
TARGET_BUMPS = 3
TARGET_WIDTH = 0.15  # Gaussian sigma in units of the tissue's side (not given: declared here)


def voltage_target(batch, seed=4):
    """A smooth membrane-voltage pattern per cell (V): -50 mV plus three Gaussian bumps of
    20 mV over each world's unit square, bump centres uniform in [0.2, 0.8]^2 from a per-world
    stream."""
    out = np.full(batch.cells, TARGET_BASELINE_V)
    for w in range(batch.worlds):
        c0, c1 = batch.cell_offset[w], batch.cell_offset[w + 1]
        rng = np.random.default_rng([int(seed), int(w), 7])
        centres = rng.uniform(0.2, 0.8, (TARGET_BUMPS, 2))
        xy = batch.position[:, c0:c1]
        for cx, cy in centres:
            r2 = (xy[0] - cx) ** 2 + (xy[1] - cy) ** 2
            out[c0:c1] += TARGET_BUMP_V * np.exp(-r2 / (2 * TARGET_WIDTH**2))
    return out


# --------------------------------------------------------------------------------------------
# The reference's definition schema (configs/resolved_pump_tissue.json's fields)


def reference_definition(world, *, dt, steps, model="cells.model.resolved_pump_tissue@1",
                         solver="cells.solver.imex_ars222_face_electromigration@1",
                         membrane_control=None, junction_control=None, pump_control=None,
                         channel_control=None, padding=0):
    """One World as a reference definition dict (schema_version 1). ``padding`` adds that many
    inactive slots to every capacity (the reference pads its arrays to capacities)."""
    n, e = world.cells, world.edges
    mc = np.ones(n) if membrane_control is None else np.broadcast_to(membrane_control, (n,))
    jc = np.ones(e) if junction_control is None else np.broadcast_to(junction_control, (e,))
    pc = np.ones(n) if pump_control is None else np.broadcast_to(pump_control, (n,))
    atp, adp, pi, km_na, km_k, km_atp, dg0 = world.pump
    bath_amount = world.bath_mM * world.bath_volume
    bath_fixed = -float(VALENCE @ bath_amount)
    cells = []
    for i in range(n):
        cells.append({
            "id": f"cell_{i}",
            "volume_pL": float(world.volume[i]),
            "initial_amount_fmol": {s: float(world.amount[k, i]) for k, s in enumerate(SPECIES)},
            "fixed_charge_equivalent_fmol": float(world.fixed_charge_fmol[i]),
            "initial_charge_C": float(world.initial_charge[i]),
        })
    bath = {
        "id": "bath",
        "volume_pL": float(world.bath_volume),
        "initial_amount_fmol": {s: float(bath_amount[k]) for k, s in enumerate(SPECIES)},
        "fixed_charge_equivalent_fmol": bath_fixed,
        "initial_charge_C": float(anchor_charge(bath_amount[:, None], [bath_fixed])[0]),
        "reservoir": True,
        "boundary_potential_V": float(world.bath_potential),
    }
    membranes = []
    for i in range(n):
        membranes.append({
            "id": f"membrane_{i}",
            "inside": f"cell_{i}",
            "outside": "bath",
            "area_m2": float(world.area[i]),
            "capacitance_F": float(world.capacitance[i]),
            "permeability_m_per_s": {
                s: float(world.permeability[k, i]) for k, s in enumerate(SPECIES)
            },
            "law": "cells.route.constant_field@1",
            "pump": {
                "id": f"pump_{i}",
                "law": "cells.cycle.nak_atp_mass_action_positive@1",
                "roles": {"sodium": "Na", "potassium": "K"},
                "stoichiometry": {"Na": -3, "K": 2},
                "capacity_fmol_per_s": float(world.pump_capacity[i]),
                "km_na_mM": km_na,
                "km_k_mM": km_k,
                "km_atp_mM": km_atp,
                "metabolism": {
                    "kind": "cells.fuel_kind.maintained_chemical_reservoirs@1",
                    "atp_mM": atp,
                    "adp_mM": adp,
                    "pi_mM": pi,
                    "delta_g0_J_per_mol": dg0,
                },
            },
        })
    junctions = []
    for k in range(e):
        junctions.append({
            "id": f"junction_{k}",
            "sender": f"cell_{int(world.sender[k])}",
            "receiver": f"cell_{int(world.receiver[k])}",
            "area_m2": float(world.junction_area[k]),
            "permeability_m_per_s": {
                s: float(world.junction_permeability[j, k]) for j, s in enumerate(SPECIES)
            },
            "law": "cells.route.constant_field@1",
            "gate": {
                "law": "cells.junction.junction_voltage_relaxation@1",
                "threshold_voltage_V": float(world.gate_threshold[k]),
                "minimum_open_fraction": float(world.gate_minimum[k]),
                "initial_gate": float(world.gate_initial[k]),
            },
        })
    end = float(dt * steps)
    v3 = model.endswith("@3")
    out = {
        "schema_version": 1,
        "model": {
            "id": model,
            "temperature_K": float(world.temperature),
            "species": [{"id": s, "valence": int(z)} for s, z in zip(SPECIES, VALENCE, strict=True)],
            "cells": cells,
            "extracellular": [bath],
            "membranes": membranes,
            "junctions": junctions,
            "faces": [],
            "closure": {
                "law": "cells.field_closure.resolved_capacitor_components_current_continuity@1",
                "gauge_reference": None,
            },
        },
        "experiment": {
            "end_time": end,
            "observation_times": [0.0, end],
            "membrane_controls": [
                {"membrane_id": f"membrane_{i}", "schedule": [{"time": 0.0, "availability": float(mc[i])}]}
                for i in range(n)
            ],
            "junction_controls": [
                {"junction_id": f"junction_{k}", "schedule": [{"time": 0.0, "availability": float(jc[k])}]}
                for k in range(e)
            ],
            "pump_controls": [
                {"pump_id": f"pump_{i}", "schedule": [{"time": 0.0, "availability": float(pc[i])}]}
                for i in range(n)
            ],
        },
        "execution": {
            "dt": float(dt),
            "capacity": n + padding,
            "extracellular_capacity": 1 + padding,
            "membrane_capacity": n + padding,
            "edge_capacity": e + padding,
            "face_capacity": padding,
            "backend": "cpu",
            "jit": True,
            "precision": "float64",
            "solver": solver,
            "field_solver": "cells.solver.capacitive_reduction_gauged_damped_newton@2",
            "max_steps": int(steps),
            "max_trace_bytes": 536870912,
            "material_balance_atol_fmol": {s: 2e-11 for s in SPECIES},
        },
    }
    if v3:  # @3 declares its channel populations and (absent) Ca pumps explicitly.
        chs = []
        nch = world.channel_slots
        cc = (np.ones((nch, n)) if channel_control is None
              else np.broadcast_to(channel_control, (nch, n)))
        for i in range(n):
            for k in range(nch):
                code = int(world.channel_code[k, i])
                if code not in (0, 2):
                    raise ValueError("the reference's catalogue has no law with code " + str(code))
                chs.append({
                    "id": f"channel_{k}_{i}",
                    "membrane_id": f"membrane_{i}",
                    "kinetic_law": CHANNEL_LAW_IDS[code],
                    "max_permeability_m_per_s": float(world.channel_permeability[k, i]),
                    "abundance": float(world.channel_abundance[k, i]),
                    "initial_gate": [float(world.channel_gate_initial[0, k, i]),
                                     float(world.channel_gate_initial[1, k, i])],
                    "permeant_ions": [{"species_id": SPECIES[int(world.channel_species[k, i])],
                                       "relative_permeability": 1.0}],
                })
                block = block_declaration(world.channel_block, k, i)
                if block is not None:
                    chs[-1]["block"] = block
        out["model"]["channels"] = chs
        out["experiment"]["channel_controls"] = [
            {"channel_id": f"channel_{k}_{i}",
             "schedule": [{"time": 0.0, "availability": float(cc[k, i])}]}
            for i in range(n) for k in range(nch)
        ]
        out["execution"]["channel_capacity"] = len(chs) + (padding if chs or padding else 0)
        for membrane in out["model"]["membranes"]:
            membrane["calcium_pump"] = None
        out["experiment"]["calcium_pump_controls"] = []
    return out
