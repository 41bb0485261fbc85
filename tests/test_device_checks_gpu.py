"""The device accepted-row checks (cb_device_checks) against the reference's own device checks
(tests/golden/device_checks.npz, made by @3's device_checks) and against the checks oracle
(oracle/checks.py) on uneven worlds with planted faults.

Tolerances: every failed bit equal; the energy residual and its ratio to the flows to 1e-8
relative (the other diagnostics are rounding residuals whose low bits depend on the summation
order, and are checked through the bits against their step-scaled bounds); a planted material
error of 1e-8 fmol read back to 1e-6 relative.
"""

import numpy as np
import pytest

from cells_b200 import worlds
from cells_b200.tissue import CHECKS, Tissue
from conftest import load_golden
from gpu_util import oracle_state, run_device
from oracle import checks as CK
from oracle import tissue as T
from test_oracle_checks import case_states

pytestmark = pytest.mark.gpu
ENERGY_RTOL = 1e-8


def device_checks(torch, tissue, prev, row, steps, material_atol, energy_rtol):
    dev = torch.device("cuda", tissue.device)
    p = torch.from_numpy(tissue.pack_state(prev)).to(dev)
    r = torch.from_numpy(tissue.pack_state(row)).to(dev)
    n = tissue.batch.worlds
    failed = torch.full((n,), -1, dtype=torch.int32, device=dev)
    values = torch.full((n * 12,), float("nan"), dtype=torch.float64, device=dev)
    tissue.device_checks(p, r, steps, material_atol, energy_rtol, failed, values)
    torch.cuda.synchronize(dev)
    bits = failed.cpu().numpy().astype(np.uint32)
    return ((bits[:, None] >> np.arange(12)) & 1) == 1, values.cpu().numpy().reshape(n, 12)


def close(a, b, rtol):
    return abs(a - b) <= rtol * abs(b)


def test_device_checks_match_the_reference(cuda):
    z, b = load_golden("device_checks.npz")
    assert tuple(z["checks"]) == CHECKS
    tissue = Tissue(b)
    seen = []
    for i in range(int(z["cases"])):
        prev, row = case_states(z, b, i)
        failed, values = device_checks(cuda, tissue, oracle_state(prev), oracle_state(row),
                                       int(z[f"case{i}_steps"]), z["material_atol"],
                                       float(z["energy_rtol"]))
        ref_failed, ref_values = z[f"case{i}_failed"], z[f"case{i}_values"]
        assert np.array_equal(failed[0], ref_failed), (i, failed[0], ref_failed)
        for k in (6, 10):
            assert close(values[0, k], ref_values[k], ENERGY_RTOL), (i, k, values[0, k])
        label = str(z[f"case{i}_label"])
        if label == "material":
            assert close(values[0, 0], ref_values[0], 1e-6)
        seen.append((label, bool(failed[0].any())))
    assert ("material", True) in seen and ("dissipation", True) in seen
    assert all(not bad for label, bad in seen if label == "accepted")


def uneven_batch(seed=51):
    rng = np.random.default_rng(seed)
    ws = []
    for k, (n, gate) in enumerate(((30, (0.015, 0.2, 1.0)), (257, None), (64, (0.01, 0.3, 0.9)),
                                   (700, None), (16, (0.02, 0.1, 0.8)), (90, None))):
        w = worlds.delaunay_world(n, worlds.world_rng(seed, k), gate=gate)
        ws.append(worlds.with_channels(w, rng, na=("nav", 4e-10, 0.5), k=("hh", 5e-10, 0.5),
                                       sigma=0.3))
    return worlds.pack(ws)


def test_device_checks_match_the_oracle_with_planted_faults(cuda):
    b = uneven_batch()
    topo = T.topology(b)
    control = T.full_control(b)
    steps = 25
    prev = T.initial_state(b)
    for _ in range(steps - 1):
        prev, ok = T.ars222_step(prev, 1e-3, control, b, topo)
        assert ok.all()
    row, ok = T.ars222_step(prev, 1e-3, control, b, topo)
    assert ok.all()
    co, eo = b.cell_offset, b.edge_offset
    plant = {f: np.array(getattr(row, f), copy=True) for f in row._fields}
    plant["amount_increment"][1, co[1] + 5] += 1e-8                      # world 1: material
    plant["junction_dissipated"][eo[2] + 3] = prev.junction_dissipated[eo[2] + 3] - 1e-9  # 2
    plant["channel_gate"][0, 1, co[3] + 7] = 1.0 + 1e-9                   # world 3: domain
    plant["reservoir_work"][4] += 1e-6                                    # world 4: work
    plant["metabolic_work"][co[5] + 2] += 1e-9                            # world 5: metabolic
    bad_row = T.State(**plant)
    atol, rtol = np.full(3, 2e-11), 2e-3
    tissue = Tissue(b)
    for r, expect_any in ((row, False), (bad_row, True)):
        want, want_v = CK.row_checks(prev, r, b, topo, steps, atol, rtol)
        got, got_v = device_checks(cuda, tissue, oracle_state(prev), oracle_state(r), steps,
                                   atol, rtol)
        assert np.array_equal(got, want), (np.argwhere(got != want), got, want)
        for w in range(b.worlds):
            for k in (6, 10):
                assert close(got_v[w, k], want_v[w, k], ENERGY_RTOL), (w, k)
        assert bool(got[1:].any()) == expect_any
    names = {w: {CHECKS[k] for k in np.flatnonzero(got[w])} for w in range(b.worlds)}
    assert not names[0]
    assert {"local", "total"} <= names[1]
    assert names[2] == {"dissipation"}
    assert "domain" in names[3]
    assert "reservoir_work" in names[4]
    assert "metabolic_work" in names[5]
    assert close(got_v[1, 0], 1e-8, 1e-6)


def test_device_checks_pass_on_device_trajectories(cuda):
    """Rows of the device step on the batched 16x16 tissues (and gated worlds with channels)
    pass every check, at 1 and at 200 accepted steps."""
    rng = np.random.default_rng(5)
    ws = worlds.grid_tissues(16, side=16, seed=3)
    ws += [worlds.delaunay_world(120, worlds.world_rng(9, k), gate=(0.015, 0.2, 1.0))
           for k in range(4)]
    b = worlds.pack([worlds.with_channels(w, rng, sigma=0.3) for w in ws])
    tissue = Tissue(b)
    control = tissue.pack_control()
    prev = tissue.initial_state()
    done = 0
    for target in (1, 199, 200):
        row, status, _ = run_device(cuda, tissue, prev, control, 1e-3, target - done)
        assert np.all(status == 0)
        failed, values = device_checks(cuda, tissue, prev, row, target, np.full(3, 2e-11), 2e-3)
        assert not failed.any(), np.argwhere(failed)
        assert np.all(values[:, 10] < 2e-3) and np.all(values[:, 11] <= 1.0)
        prev, done = row, target


def test_per_world_step_counts_match_one_count_each(cuda):
    """cb_device_checks_each at counts [1, 25, 7, 200, 0, 3] gives each world cb_device_checks'
    bits and diagnostics at that world's count, bit for bit."""
    torch = cuda
    b = uneven_batch(52)
    topo = T.topology(b)
    prev = T.initial_state(b)
    row, ok = T.ars222_step(prev, 1e-3, T.full_control(b), b, topo)
    assert ok.all()
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    p = torch.from_numpy(tissue.pack_state(oracle_state(prev))).to(dev)
    r = torch.from_numpy(tissue.pack_state(oracle_state(row))).to(dev)
    counts = [1, 25, 7, 200, 0, 3]
    steps = torch.tensor(counts, dtype=torch.int64, device=dev)
    failed = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
    values = torch.zeros(b.worlds * 12, dtype=torch.float64, device=dev)
    tissue.device_checks(p, r, steps, np.full(3, 2e-11), 2e-3, failed, values)
    each_f, each_v = failed.clone(), values.clone()
    for w, n in enumerate(counts):
        tissue.device_checks(p, r, n, np.full(3, 2e-11), 2e-3, failed, values)
        assert int(each_f[w]) == int(failed[w])
        assert torch.equal(each_v[12 * w:12 * w + 12], values[12 * w:12 * w + 12])
