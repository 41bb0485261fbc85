"""The packed persistent kernel (uneven and large worlds, a device work queue): parity with the
reference's trajectories and the oracle, per-world refusal inside a work item, and agreement
with the one-world-per-CTA kernel. Tolerances as tests/test_step_gpu.py: 1e-10 scaled difference
per field."""

import numpy as np
import pytest

from cells_b200 import worlds
from cells_b200.tissue import Tissue, decode_status
from conftest import load_golden, scaled_difference
from gpu_util import oracle_state, run_device
from oracle import tissue as T

pytestmark = pytest.mark.gpu
TRAJECTORY_TOL = 1e-10


@pytest.fixture
def packed(monkeypatch):
    monkeypatch.setenv("CELLS_B200_KERNEL", "packed")


@pytest.mark.parametrize("name", ["ars222_grid4x4.npz", "ars222_gated.npz",
                                  "ars222_v3_channels_delaunay.npz"])
def test_packed_matches_reference_trajectory(cuda, packed, name):
    z, b = load_golden(name)
    tissue = Tissue(b)
    control = tissue.pack_control(**{
        f: z["control_" + f] for f in ("membrane", "junction", "pump", "channel")
        if "control_" + f in z})
    state, done, worst = tissue.initial_state(), 0, {}
    for idx, target in enumerate(z["steps"]):
        if target > done:
            state, status, _ = run_device(cuda, tissue, state, control, float(z["dt"]),
                                          int(target - done))
            assert np.all(status == 0)
            done = int(target)
        for f in T.State._fields:
            if "ref_" + f in z:
                worst[f] = max(worst.get(f, 0.0), scaled_difference(state[f], z["ref_" + f][idx]))
    bad = {k: v for k, v in worst.items() if v > TRAJECTORY_TOL}
    assert not bad, bad


def test_packed_uneven_large_worlds_match_oracle(cuda, packed):
    """Worlds of 32 to 3000 cells (Delaunay), several packed per item, HH channels, random
    availabilities, against the oracle."""
    rng = np.random.default_rng(31)
    sizes = (40, 33, 1500, 77, 3000, 256, 64, 900)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(14, k),
                                                     junction_sigma=0.3), rng,
                               na=("nav", 3e-10, 0.5), k=("hh", 6e-10, 0.5), sigma=0.3)
          for k, n in enumerate(sizes)]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    ctl = T.Control(rng.uniform(0.5, 1, b.cells), rng.uniform(0.5, 1, b.edges),
                    rng.uniform(0.5, 1, b.cells), rng.uniform(0.3, 1, (2, b.cells)))
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(60):
        st, ok = T.ars222_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
    got, status, taken = run_device(cuda, tissue, tissue.initial_state(),
                                    tissue.pack_control(*ctl), 1e-3, 60, chunks=[25, 35])
    assert np.all(status == 0), [decode_status(x) for x in status]
    assert np.all(taken == 35)
    for f, ref in oracle_state(st).items():
        assert scaled_difference(got[f], ref) <= TRAJECTORY_TOL, f


def test_packed_refuses_one_world_and_advances_its_item(cuda, packed):
    ws = worlds.grid_tissues(4, side=6, seed=9)
    b = worlds.pack(ws)
    tissue = Tissue(b)
    mc = np.ones(b.cells)
    mc[b.cell_offset[2] + 3] = 2.0  # world 2: an availability outside [0, 1]
    start = tissue.initial_state()
    got, status, taken = run_device(cuda, tissue, start, tissue.pack_control(membrane=mc),
                                    1e-3, 4)
    assert list(taken) == [4, 4, 0, 4]
    assert "control" in decode_status(status[2])
    cs = slice(b.cell_offset[2], b.cell_offset[3])
    assert np.array_equal(got["amount_increment"][:, cs], start["amount_increment"][:, cs])


def test_packed_and_shared_kernels_agree(cuda, monkeypatch):
    b = worlds.pack(worlds.grid_tissues(12, side=16, seed=4))
    monkeypatch.setenv("CELLS_B200_KERNEL", "shared")
    shared = Tissue(b)
    monkeypatch.setenv("CELLS_B200_KERNEL", "packed")
    packed = Tissue(b)
    a, _, _ = run_device(cuda, shared, shared.initial_state(), shared.pack_control(), 1e-3, 50)
    c, _, _ = run_device(cuda, packed, packed.initial_state(), packed.pack_control(), 1e-3, 50)
    for f in a:
        # Cell and junction arithmetic is the same; world sums use other (fixed) orders.
        assert scaled_difference(c[f], a[f]) <= 1e-13, f
    assert np.array_equal(a["junction_gate"], c["junction_gate"])


def test_packed_repeat_runs_are_bit_identical(cuda, packed):
    rng = np.random.default_rng(5)
    ws = [worlds.delaunay_world(int(n), worlds.world_rng(15, k))
          for k, n in enumerate(rng.integers(32, 600, 20))]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    a, _, _ = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(), 1e-3, 20)
    c, _, _ = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(), 1e-3, 20)
    for f in a:
        assert np.array_equal(a[f], c[f]), f


def test_graph_replay_equals_direct_launches(cuda):
    """The step captured in a CUDA graph (three fused launches) replays the same bits as the same
    launches issued directly, on both kernel paths."""
    torch = cuda
    from cells_b200 import _lib

    b = worlds.pack(worlds.grid_tissues(6, side=16, seed=6))
    tissue = Tissue(b)
    dev = torch.device("cuda")
    ctl = torch.from_numpy(tissue.pack_control()).to(dev)
    for kernel, block, occ in ((_lib.KERNEL_SHARED, 256, 3), (_lib.KERNEL_PACKED, 512, 1)):
        tissue.set_launch(kernel, block, occ)
        start = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
        direct = start.clone()
        status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
        for _ in range(3):
            tissue.step(direct, direct, ctl, 1e-3, 7, status)
        graphed = start.clone()
        gstatus = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
        graph = tissue.capture(graphed, graphed, ctl, 1e-3, 7, gstatus, launches=3)
        graphed.copy_(start)
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(direct, graphed)
        assert int(gstatus.abs().max()) == 0
        del graph


def test_autotune_selects_a_feasible_configuration(cuda):
    torch = cuda
    from cells_b200 import _lib, autotune

    ws = worlds.delaunay_tissues(12, lo=32, hi=900, seed=8)
    tissue = Tissue(worlds.pack(ws))
    dev = torch.device("cuda")
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    ctl = torch.from_numpy(tissue.pack_control()).to(dev)
    best, timings = autotune.tune(tissue, state, ctl, 1e-3, steps=5, repeats=1)
    assert best in timings and timings[best] == min(timings.values())
    assert tissue.get_launch()[0] == best[0]
    assert any(k[0] == _lib.KERNEL_PACKED for k in timings)
    got, status, _ = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(),
                                1e-3, 10)
    assert np.all(status == 0)
