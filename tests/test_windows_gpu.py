"""The window runner (cells_b200/windows.py: steps with per-row device checks, the reference's
vector window, src/cells/execution/vector_windows.py:348-410) against the same window built from
the oracle's step and checks (oracle/tissue.py, oracle/checks.py).

Three gated worlds, six rows of 1 ms under a two-entry held-control table; world 1's second
control has an availability above 1 (its step is refused at the first row that holds it, row 3),
world 2 takes only four rows. Failing rows and bits equal; final states and stored rows within
1e-10 scaled difference; the energy diagnostics' maxima to 1e-8.
"""

import numpy as np
import pytest

from cells_b200 import windows, worlds
from cells_b200.tissue import Tissue
from conftest import load_golden, scaled_difference
from gpu_util import oracle_state
from oracle import checks as CK
from oracle import tissue as T

pytestmark = pytest.mark.gpu
DT = [1e-3] * 6
HELD = [0, 0, 1, 1, 0, 1]
SLOTS = [0, -1, 1, -1, -1, 2]
COUNTS = [6, 6, 4]
ATOL, RTOL = np.full(3, 2e-11), 2e-3


def batch():
    rng = np.random.default_rng(31)
    ws = [worlds.grid_world(4, 4, worlds.world_rng(31, k), gate=(0.015, 0.2, 1.0)) for k in
          range(3)]
    b = worlds.pack(ws)
    c0 = T.Control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                   rng.uniform(0.6, 1, b.cells))
    m1 = c0.membrane.copy()
    m1[b.cell_offset[1] + 3] = 1.2  # world 1 refuses every step under control 1
    c1 = T.Control(m1, c0.junction * 0.9, c0.pump)
    return b, [c0, c1]


def oracle_window(b, controls):
    topo = T.topology(b)
    cur = T.initial_state(b)
    failed0, vals0 = CK.row_checks(cur, cur, b, topo, 0, ATOL, RTOL)
    pack = (failed0 << (np.arange(12) + 1)).sum(axis=1)
    ok = pack == 0
    first = np.where(ok, -1, 0)
    bits = pack.copy()
    maxima = np.where(ok[:, None], vals0, 0.0)
    stored = {}
    for j in range(1, len(DT) + 1):
        new, valid = T.ars222_step(cur, DT[j - 1], controls[HELD[j - 1]], b, topo)
        failed, vals = CK.row_checks(cur, new, b, topo, j, ATOL, RTOL)
        flags = np.where(valid, (failed << (np.arange(12) + 1)).sum(axis=1), 1)
        live = (j <= np.asarray(COUNTS)) & ok
        failing = live & (flags != 0)
        accept = live & (flags == 0)
        first = np.where(failing, j, first)
        bits = np.where(failing, flags, bits)
        cur = T._select(accept, new, cur, b, topo)
        maxima = np.where(accept[:, None], np.maximum(maxima, vals), maxima)
        if SLOTS[j - 1] >= 0:
            stored[SLOTS[j - 1]] = (accept.copy(), oracle_state(cur))
        ok = ok & ~failing
    return cur, first, bits, maxima, stored


def test_window_matches_the_oracle_window(cuda):
    torch = cuda
    b, controls = batch()
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    table = torch.from_numpy(np.stack([tissue.pack_control(c.membrane, c.junction, c.pump)
                                       for c in controls])).to(dev)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    win = windows.vector_window(tissue, state, DT, table, HELD, slots=SLOTS, counts=COUNTS,
                                material_atol=ATOL, energy_rtol=RTOL, rows=3)
    torch.cuda.synchronize(dev)
    cur, first, bits, maxima, stored = oracle_window(b, controls)
    assert np.array_equal(win.first.cpu().numpy(), first)
    assert np.array_equal(win.bits.cpu().numpy(), bits)
    assert first.tolist() == [-1, 3, -1] and windows.failure_names(bits[1]) == ("step_refused",)
    got = tissue.unpack_state(win.state.cpu().numpy())
    bad = {f: d for f, ref in oracle_state(cur).items()
           if (d := scaled_difference(got[f], ref)) > 1e-10}
    assert not bad, bad
    rows = win.rows.cpu().numpy()
    for slot, (accept, ref) in stored.items():
        got_row = tissue.unpack_state(rows[slot])
        cells = np.repeat(accept, np.diff(b.cell_offset))
        for f in ("amount_increment", "membrane_transferred", "pump_cycles"):
            g, r = np.asarray(got_row[f]), np.asarray(ref[f])
            assert scaled_difference(g[..., cells], r[..., cells]) <= 1e-10, (slot, f)
    m = win.maxima.cpu().numpy()
    for k in (6, 10):
        assert np.all(np.abs(m[:, k] - maxima[:, k]) <= 1e-8 * np.abs(maxima[:, k])), k


# Per-world rows: each world its own step sizes, held-control indices, observation slots and
# accepted-step count at the window start (the reference's [W, width] tables and [W] first_step).
DT_W = np.array([[1e-3] * 6, [5e-4] * 6, [1e-3, 2e-3, 1e-3, 2e-3, 1e-3, 2e-3]])
HELD_W = np.array([[0, 0, 1, 1, 0, 1], [1, 0, 0, 1, 1, 0], [0, 1, 0, 1, 0, 1]])
SLOTS_W = np.array([[0, -1, 1, -1, -1, 2], [-1, 0, -1, 1, 2, -1], [2, -1, -1, 0, 1, -1]])
FIRST_W = np.array([0, 7, 3])


def _control_of(controls, held_row, b, topo):
    """The oracle Control whose world w takes controls[held_row[w]]."""
    cw, ew = topo.cell_world, topo.edge_world
    cells = np.arange(b.cells)
    pick = held_row[cw]
    membrane = np.stack([c.membrane for c in controls])[pick, cells]
    pump = np.stack([c.pump for c in controls])[pick, cells]
    junction = np.stack([c.junction for c in controls])[held_row[ew], np.arange(b.edges)]
    channel = np.stack([np.asarray(c.channel) for c in controls])
    if channel.ndim == 3:  # [n, NCH, C]
        channel = channel[pick, :, cells].T
    else:  # no channel slots: the one (empty) control of every entry
        channel = np.asarray(controls[0].channel)
    return T.Control(membrane, junction, pump, channel)


def oracle_window_each(b, controls):
    topo = T.topology(b)
    cur = T.initial_state(b)

    def checks_each(prev, row, offset):
        failed = np.zeros((b.worlds, 12), dtype=bool)
        vals = np.zeros((b.worlds, 12))
        for steps in np.unique(FIRST_W + offset):
            f, v = CK.row_checks(prev, row, b, topo, int(steps), ATOL, RTOL)
            sel = FIRST_W + offset == steps
            failed[sel], vals[sel] = f[sel], v[sel]
        return failed, vals

    failed0, vals0 = checks_each(cur, cur, 0)
    pack = (failed0 << (np.arange(12) + 1)).sum(axis=1)
    ok = pack == 0
    first = np.where(ok, -1, 0)
    bits = pack.copy()
    maxima = np.where(ok[:, None], vals0, 0.0)
    stored = {}
    for j in range(1, DT_W.shape[1] + 1):
        control = _control_of(controls, HELD_W[:, j - 1], b, topo)
        new, valid = cur, np.zeros(b.worlds, dtype=bool)
        for size in np.unique(DT_W[:, j - 1]):
            trial, v = T.ars222_step(cur, float(size), control, b, topo)
            take = DT_W[:, j - 1] == size
            new = T._select(take, trial, new, b, topo)
            valid = np.where(take, v, valid)
        failed, vals = checks_each(cur, new, j)
        flags = np.where(valid, (failed << (np.arange(12) + 1)).sum(axis=1), 1)
        live = (j <= np.asarray(COUNTS)) & ok
        failing = live & (flags != 0)
        accept = live & (flags == 0)
        first = np.where(failing, j, first)
        bits = np.where(failing, flags, bits)
        cur = T._select(accept, new, cur, b, topo)
        maxima = np.where(accept[:, None], np.maximum(maxima, vals), maxima)
        for w in range(b.worlds):
            slot = SLOTS_W[w, j - 1]
            if slot >= 0 and accept[w]:
                stored[(slot, w)] = oracle_state(cur)
        ok = ok & ~failing
    return cur, first, bits, maxima, stored


def test_window_with_per_world_rows_matches_the_oracle(cuda):
    torch = cuda
    b, controls = batch()
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    table = torch.from_numpy(np.stack([tissue.pack_control(c.membrane, c.junction, c.pump)
                                       for c in controls])).to(dev)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    win = windows.vector_window(tissue, state, DT_W, table, HELD_W, slots=SLOTS_W,
                                counts=COUNTS, first_step=FIRST_W, material_atol=ATOL,
                                energy_rtol=RTOL, rows=3)
    torch.cuda.synchronize(dev)
    cur, first, bits, maxima, stored = oracle_window_each(b, controls)
    assert np.array_equal(win.first.cpu().numpy(), first)
    assert np.array_equal(win.bits.cpu().numpy(), bits)
    assert first[1] > 0 and windows.failure_names(bits[1]) == ("step_refused",)
    got = tissue.unpack_state(win.state.cpu().numpy())
    bad = {f: d for f, ref in oracle_state(cur).items()
           if (d := scaled_difference(got[f], ref)) > 1e-10}
    assert not bad, bad
    rows = win.rows.cpu().numpy()
    topo = T.topology(b)
    for (slot, w), ref in stored.items():
        got_row = tissue.unpack_state(rows[slot])
        cells = topo.cell_world == w
        for f in ("amount_increment", "membrane_transferred", "pump_cycles"):
            g, r = np.asarray(got_row[f]), np.asarray(ref[f])
            assert scaled_difference(g[..., cells], r[..., cells]) <= 1e-10, (slot, w, f)
    m = win.maxima.cpu().numpy()
    for k in (6, 10):
        assert np.all(np.abs(m[:, k] - maxima[:, k]) <= 1e-8 * np.abs(maxima[:, k])), k


def test_copy_worlds_is_a_masked_select(cuda):
    """cb_copy_worlds copies exactly the masked worlds' state elements (channel batch, uneven
    worlds), bit for bit, and leaves every other element as it was."""
    torch = cuda
    rng = np.random.default_rng(8)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(8, k)), rng)
          for k, n in enumerate((30, 257, 64, 700, 16))]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    n = tissue.state_size
    src = torch.from_numpy(rng.standard_normal(n)).to(dev)
    dst = torch.from_numpy(rng.standard_normal(n)).to(dev)
    mask = torch.tensor([1, 0, 1, 1, 0], dtype=torch.int32, device=dev)
    real = tissue.pack_state({f: np.ones_like(v, dtype=float)
                              for f, v in tissue.initial_state().items()}) == 1.0
    world = windows.world_of_elements(tissue)
    take = torch.from_numpy(real & mask.cpu().numpy().astype(bool)[world]).to(dev)
    want = torch.where(take, src, dst)
    tissue.copy_worlds(mask, src, dst)
    torch.cuda.synchronize(dev)
    assert torch.equal(dst, want)


def test_window_matches_the_reference_window(cuda):
    """The reference's own _vector_window (tests/golden/vector_window.npz: run by
    tests/golden/make_golden.py over @3's checked_step and device_checks, vmap a loop over worlds)
    on the per-world tables above: first failing rows and bits equal, the final states and the
    stored rows within 1e-10 scaled difference, the energy diagnostics' maxima to 1e-8."""
    torch = cuda
    z, b = load_golden("vector_window.npz")
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    table = torch.from_numpy(np.stack([
        tissue.pack_control(z[f"control{k}_membrane"], z[f"control{k}_junction"],
                            z[f"control{k}_pump"]) for k in range(2)])).to(dev)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    rows = int(z["rows"])
    win = windows.vector_window(tissue, state, z["dt"], table, z["held"], slots=z["slots"],
                                counts=z["counts"], first_step=z["first_step"],
                                material_atol=z["material_atol"],
                                energy_rtol=float(z["energy_rtol"]), rows=rows)
    torch.cuda.synchronize(dev)
    assert np.array_equal(win.first.cpu().numpy(), z["first"])
    assert np.array_equal(win.bits.cpu().numpy(), z["bits"])
    got = tissue.unpack_state(win.state.cpu().numpy())
    topo = T.topology(b)
    stored = win.rows.cpu().numpy()
    for w in range(b.worlds):
        cells, edges = topo.cell_world == w, topo.edge_world == w

        def part(f, v):
            v = np.asarray(v)
            if f in T.CELL_FIELDS:
                return v[..., cells]
            if f in T.EDGE_FIELDS:
                return v[..., edges]
            return v[..., w]

        for f in T.State._fields:
            if f"final{w}_{f}" not in z.files:
                continue
            ref = z[f"final{w}_{f}"]
            if f in T.WORLD_FIELDS:  # the reference's one outside node: slot 0
                ref = ref[..., 0]
            assert scaled_difference(part(f, got[f]), ref) <= 1e-10, (w, f)
        for r in range(rows):
            row = tissue.unpack_state(stored[r])
            for f in ("amount_increment", "membrane_transferred", "pump_cycles",
                      "junction_transferred", "junction_gate"):
                assert scaled_difference(part(f, row[f]), z[f"stored{w}_{r}_{f}"]) <= 1e-10, \
                    (w, r, f)
    m, ref = win.maxima.cpu().numpy(), z["maxima"]
    for k in (6, 10):
        assert np.all(np.abs(m[:, k] - ref[:, k]) <= 1e-8 * np.abs(ref[:, k])), k
