"""Parity of the device step (cb_step, ARS(2,2,2), FP64) with the reference and the oracle.

Tolerances (written here, from the benchmark's FP64 contract): every state field within 1e-10
scaled difference (max |a-b| / max |ref|) of the reference's own trajectory over the whole run;
ledgers conserved to 1e-12 relative every step; graph indexing bit-exact (world results do not
depend on batch position or launch count, and repeat bit for bit).
"""

import numpy as np
import pytest

from cells_b200 import worlds
from cells_b200.tissue import Tissue, decode_status
from conftest import load_golden, scaled_difference
from gpu_util import oracle_state, run_device
from oracle import tissue as T

pytestmark = pytest.mark.gpu
TRAJECTORY_TOL = 1e-10
LEDGER_TOL = 1e-12


def _golden_replay(torch, name):
    z, b = load_golden(name)
    tissue = Tissue(b)
    control = tissue.pack_control(**{
        f: z["control_" + f] for f in ("membrane", "junction", "pump", "channel")
        if "control_" + f in z})
    state = tissue.initial_state()
    done = 0
    worst = {}
    for idx, target in enumerate(z["steps"]):
        if target > done:
            state, status, taken = run_device(torch, tissue, state, control, float(z["dt"]),
                                              int(target - done))
            assert np.all(status == 0), decode_status(status[0])
            assert np.all(taken == target - done)
            done = int(target)
        for f in T.State._fields:
            if "ref_" + f in z:
                worst[f] = max(worst.get(f, 0.0),
                               scaled_difference(state[f], z["ref_" + f][idx]))
    return worst


@pytest.mark.parametrize("name", ["ars222_grid4x4.npz", "ars222_v3_grid4x4.npz",
                                  "ars222_gated.npz", "ars222_v3_channels.npz",
                                  "ars222_v3_channels_delaunay.npz"])
def test_device_matches_reference_trajectory(cuda, name):
    worst = _golden_replay(cuda, name)
    bad = {k: v for k, v in worst.items() if v > TRAJECTORY_TOL}
    assert not bad, bad


def _batch(n_worlds, side, seed=1):
    return worlds.pack(worlds.grid_tissues(n_worlds, side=side, seed=seed))


def test_device_matches_oracle_batched_grid(cuda):
    b = _batch(24, 16)  # the batched plain step's 16x16 tissues
    tissue = Tissue(b)
    ctl = T.full_control(b)
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(150):
        st, ok = T.ars222_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
    got, status, _ = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(),
                                1e-3, 150, chunks=[50, 100])
    assert np.all(status == 0)
    for f, ref in oracle_state(st).items():
        assert scaled_difference(got[f], ref) <= TRAJECTORY_TOL, f


def test_device_matches_oracle_delaunay(cuda):
    ws = [worlds.delaunay_world(n, worlds.world_rng(9, k), junction_sigma=0.3,
                                gate=(0.02, 0.2, 0.9)) for k, n in enumerate((40, 97, 200))]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    rng = np.random.default_rng(4)
    mc, jc, pc = rng.uniform(0.3, 1, b.cells), rng.uniform(0.3, 1, b.edges), rng.uniform(0.3, 1, b.cells)
    ctl = T.Control(mc, jc, pc)
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(120):
        st, ok = T.ars222_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
    got, status, _ = run_device(cuda, tissue, tissue.initial_state(),
                                tissue.pack_control(mc, jc, pc), 1e-3, 120)
    assert np.all(status == 0)
    for f, ref in oracle_state(st).items():
        assert scaled_difference(got[f], ref) <= TRAJECTORY_TOL, f


def test_fused_launches_equal_single_steps_bitwise(cuda):
    b = _batch(6, 16)
    tissue = Tissue(b)
    ctl = tissue.pack_control()
    a, _, _ = run_device(cuda, tissue, tissue.initial_state(), ctl, 1e-3, 40)
    c, _, _ = run_device(cuda, tissue, tissue.initial_state(), ctl, 1e-3, 40, chunks=[1] * 40)
    for f in a:
        assert np.array_equal(a[f], c[f]), f


def test_world_results_do_not_depend_on_batch_position(cuda):
    ws = worlds.grid_tissues(5, side=16, seed=3)
    whole = Tissue(worlds.pack(ws))
    alone = Tissue(worlds.pack([ws[3]]))
    a, _, _ = run_device(cuda, whole, whole.initial_state(), whole.pack_control(), 1e-3, 30)
    c, _, _ = run_device(cuda, alone, alone.initial_state(), alone.pack_control(), 1e-3, 30)
    b = whole.batch
    cs = slice(b.cell_offset[3], b.cell_offset[4])
    es = slice(b.edge_offset[3], b.edge_offset[4])
    assert np.array_equal(a["amount_increment"][:, cs], c["amount_increment"])
    assert np.array_equal(a["junction_transferred"][:, es], c["junction_transferred"])
    assert np.array_equal(a["electrode_charge"][3:4], c["electrode_charge"])


def test_repeat_runs_are_bit_identical(cuda):
    b = _batch(8, 16, seed=8)
    tissue = Tissue(b)
    a, _, _ = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(), 1e-3, 25)
    c, _, _ = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(), 1e-3, 25)
    for f in a:
        assert np.array_equal(a[f], c[f]), f


def test_refused_world_keeps_its_state_and_others_advance(cuda):
    b = _batch(3, 8)
    tissue = Tissue(b)
    mc = np.ones(b.cells)
    mc[b.cell_offset[1]] = 1.5  # an availability outside [0, 1] in world 1
    start = tissue.initial_state()
    got, status, taken = run_device(cuda, tissue, start, tissue.pack_control(membrane=mc),
                                    1e-3, 5)
    assert status[0] == 0 and status[2] == 0
    assert "control" in decode_status(status[1])
    assert list(taken) == [5, 0, 5]
    cs = slice(b.cell_offset[1], b.cell_offset[2])
    assert np.array_equal(got["amount_increment"][:, cs], start["amount_increment"][:, cs])
    assert np.any(got["amount_increment"][:, : b.cell_offset[1]] != 0)


def test_host_entry_point_equals_device_entry_point(cuda):
    b = _batch(4, 16)
    tissue = Tissue(b)
    ctl = tissue.pack_control()
    dev, _, _ = run_device(cuda, tissue, tissue.initial_state(), ctl, 1e-3, 12)
    out, status, taken = tissue.step_host(tissue.pack_state(tissue.initial_state()), ctl, 1e-3, 12)
    host = tissue.unpack_state(out)
    assert np.all(status == 0) and np.all(taken == 12)
    for f in dev:
        assert np.array_equal(dev[f], host[f]), f


@pytest.mark.parametrize("method", [0, 1])
def test_chunked_host_entry_point_equals_device_entry_point(cuda, method):
    """cb_step_host on 37 worlds (four uneven chunks on four streams) with NaV1.2 + Kv1.5
    populations and one world refused (a membrane availability above 1): state, status and
    accepted steps equal cb_step's bit for bit, FP64 and mixed."""
    rng = np.random.default_rng(19)
    ws = [worlds.with_channels(worlds.grid_world(16, 16, worlds.world_rng(19, k)), rng,
                               sigma=0.3) for k in range(37)]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    membrane = np.ones(b.cells)
    membrane[b.cell_offset[20] + 5] = 1.3
    ctl = tissue.pack_control(membrane=membrane)
    dev = cuda.device("cuda", tissue.device)
    src = cuda.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    out = cuda.empty_like(src)
    c = cuda.from_numpy(ctl).to(dev)
    st = cuda.zeros(b.worlds, dtype=cuda.int32, device=dev)
    tk = cuda.zeros(b.worlds, dtype=cuda.int32, device=dev)
    tissue.step(src, out, c, 1e-3, 15, st, tk, method=method)
    cuda.cuda.synchronize(dev)
    want = tissue.unpack_state(out.cpu().numpy())
    got_out, status, taken = tissue.step_host(tissue.pack_state(tissue.initial_state()), ctl,
                                              1e-3, 15, method=method)
    got = tissue.unpack_state(got_out)
    assert np.array_equal(status, st.cpu().numpy().astype(np.uint32))
    assert np.array_equal(taken, tk.cpu().numpy())
    assert status[20] != 0 and np.count_nonzero(status) == 1
    for f in want:
        assert np.array_equal(want[f], got[f]), f


def test_full_size_batched_plain_step_conserves_ledgers(cuda):
    """4096 worlds of 16x16 cells (the batched plain step's full size): every step's ledgers
    within 1e-12 relative (device balances), all worlds accepted."""
    torch = cuda
    b = worlds.pack(worlds.grid_tissues(4096, side=16, seed=1))
    tissue = Tissue(b)
    dev = torch.device("cuda")
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    ctl = torch.from_numpy(tissue.pack_control()).to(dev)
    status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
    out = torch.zeros(b.worlds * 8, dtype=torch.float64, device=dev)
    scale_amount = float(np.max(np.abs(b.amount_reference)))
    for _ in range(10):
        tissue.step(state, state, ctl, 1e-3, 2, status)
        tissue.balances(state, out)
        res = out.view(b.worlds, 8).cpu().numpy()
        assert int(status.abs().max()) == 0
        assert res[:, :3].max() <= LEDGER_TOL * scale_amount
        host = tissue.unpack_state(state.cpu().numpy())
        ec = np.abs(host["electrode_charge"]).max()
        assert res[:, 3].max() <= LEDGER_TOL * ec and res[:, 4].max() <= LEDGER_TOL * ec
        for k, f in ((5, "reservoir_work"), (7, "metabolic_work")):
            assert res[:, k].max() <= LEDGER_TOL * np.abs(host[f]).max(), f


def test_device_balances_match_oracle_balances(cuda):
    b = _batch(5, 16, seed=2)
    tissue = Tissue(b)
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(30):
        st, _ = T.ars222_step(st, 1e-3, T.full_control(b), b, topo)
    torch = cuda
    dev = torch.device("cuda")
    s = torch.from_numpy(tissue.pack_state(oracle_state(st))).to(dev)
    out = torch.zeros(b.worlds * 8, dtype=torch.float64, device=dev)
    tissue.balances(s, out)
    res = out.view(b.worlds, 8).cpu().numpy()
    ref = T.balances(st, b, topo)
    scale = np.max(np.abs(b.amount_reference))
    assert np.all(res[:, 0] <= 1e-12 * scale)
    assert np.allclose(res[:, 7], np.max(np.abs(ref["metabolic_work"].reshape(b.worlds, -1)),
                                         axis=1), rtol=0, atol=1e-9 * np.abs(st.metabolic_work).max())


@pytest.mark.parametrize("name", ["pytrees_gated_padded.npz", "pytrees_v3_channels_padded.npz",
                                  "pytrees_n2_padded.npz", "pytrees_v3_block_padded.npz"])
def test_drop_in_checked_step_on_reference_pytrees(cuda, name):
    """model.DeviceStep called with the reference's own padded state, control and layout, step
    by step, against the reference's trajectory (@1; @3 with channels; @3 under N2, which the
    layout declares; @3 with blocked populations); padded slots stay untouched."""
    from cells_b200 import model
    from pytree_util import load_pytrees

    z, p, control, states = load_pytrees(name)
    step = model.DeviceStep(p)
    state = states[0]
    steps = list(z["steps"])
    done = 0
    for idx, target in enumerate(steps):
        while done < target:
            state, valid = step(state, float(z["dt"]), control, p, p.active)
            assert bool(valid)
            done += 1
        ref = states[idx]
        assert type(state) is type(ref)
        for f in ref._fields:
            got, want = np.asarray(getattr(state, f)), np.asarray(getattr(ref, f))
            assert got.shape == want.shape, f
            assert scaled_difference(got, want) <= TRAJECTORY_TOL, f
    pad = ~np.asarray(p.active).astype(bool)
    assert np.all(np.asarray(state.amount_increment)[:, pad] == 0)
    step.close()


def test_device_matches_oracle_with_hh_channels(cuda):
    """Uneven Delaunay worlds with a NaV1.2 (m^3 h) and a Hodgkin-Huxley K (n^4) population per
    cell (the n^4 law is this library's; its oracle is oracle/tissue.py), random availabilities."""
    rng = np.random.default_rng(17)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(12, k),
                                                     junction_sigma=0.3), rng,
                               na=("nav", 3e-10, 0.5), k=("hh", 6e-10, 0.5), sigma=0.3)
          for k, n in enumerate((33, 120, 250))]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    ctl = T.Control(rng.uniform(0.5, 1, b.cells), rng.uniform(0.5, 1, b.edges),
                    rng.uniform(0.5, 1, b.cells), rng.uniform(0.3, 1, (2, b.cells)))
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(150):
        st, ok = T.ars222_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
    got, status, _ = run_device(cuda, tissue, tissue.initial_state(),
                                tissue.pack_control(*ctl), 1e-3, 150, chunks=[70, 80])
    assert np.all(status == 0), [decode_status(x) for x in status]
    for f, ref in oracle_state(st).items():
        assert scaled_difference(got[f], ref) <= TRAJECTORY_TOL, f


def test_stiff_channel_world_is_refused(cuda):
    """A population whose slope conductance makes dt x G/C exceed 1 refuses the step (the
    explicit-stability rule of surface_pump_v3.membrane_rate); its neighbour world advances."""
    rng = np.random.default_rng(2)
    ws = [worlds.with_channels(worlds.grid_world(4, 4, worlds.world_rng(1, k)), rng)
          for k in range(2)]
    ws[1].channel_permeability = ws[1].channel_permeability * 1e5
    b = worlds.pack(ws)
    tissue = Tissue(b)
    topo = T.topology(b)
    _, ok = T.ars222_step(T.initial_state(b), 1e-3, T.full_control(b), b, topo)
    assert list(ok) == [True, False]  # the oracle refuses it too
    got, status, taken = run_device(cuda, tissue, tissue.initial_state(), tissue.pack_control(),
                                    1e-3, 3)
    assert status[0] == 0 and "stiff" in decode_status(status[1])
    assert list(taken) == [3, 0]
