"""The device N2 step (cb_step with CB_METHOD_N2: implicit slope conductances, a sparse Cholesky
per world per step) against the reference's own N2 trajectories and the N2 oracle.

Tolerances as the plain step's (tests/test_step_gpu.py): every field within 1e-10 scaled
difference of the reference over the whole run; ledgers conserved to 1e-12; a fused launch
bit-identical to one-step launches.
"""

import dataclasses

import numpy as np
import pytest

from cells_b200 import _lib, worlds
from cells_b200.tissue import Tissue, decode_status
from conftest import load_golden, scaled_difference
from gpu_util import oracle_state
from oracle import n2 as N2
from oracle import tissue as T

pytestmark = pytest.mark.gpu
TOL = 1e-10


def run_n2(torch, tissue, state, control, dt, chunks, method=_lib.METHOD_N2):
    dev = torch.device("cuda", tissue.device)
    src = torch.from_numpy(tissue.pack_state(state)).to(dev)
    dst = torch.empty_like(src)
    ctl = torch.from_numpy(np.asarray(control, dtype=np.float64)).to(dev)
    status = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    taken = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    for k in chunks:
        tissue.step(src, dst, ctl, dt, k, status, taken, method=method)
        src, dst = dst, src
    torch.cuda.synchronize(dev)
    return tissue.unpack_state(src.cpu().numpy()), status.cpu().numpy(), taken.cpu().numpy()


@pytest.mark.parametrize("name", ["n2_grid4x4.npz", "n2_channels_delaunay.npz"])
def test_n2_matches_the_reference_trajectory(cuda, name):
    z, b = load_golden(name)
    tissue = Tissue(b)
    control = tissue.pack_control(**{f: z["control_" + f] for f in
                                     ("membrane", "junction", "pump", "channel")
                                     if "control_" + f in z.files})
    state, done, worst = tissue.initial_state(), 0, {}
    for idx, target in enumerate(z["steps"]):
        if target > done:
            state, status, taken = run_n2(cuda, tissue, state, control, float(z["dt"]),
                                          [int(target - done)])
            assert np.all(status == 0), decode_status(status[0])
            assert np.all(taken == target - done)
            done = int(target)
        for f in T.State._fields:
            if "ref_" + f in z.files:
                worst[f] = max(worst.get(f, 0.0), scaled_difference(state[f], z["ref_" + f][idx]))
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, bad


def uneven_batch(seed=41):
    rng = np.random.default_rng(seed)
    ws = []
    for k, (n, gate) in enumerate(((30, (0.015, 0.2, 1.0)), (257, None), (64, (0.01, 0.3, 0.9)),
                                   (700, None), (16, None))):
        w = worlds.delaunay_world(n, worlds.world_rng(seed, k), gate=gate)
        ws.append(worlds.with_channels(w, rng, na=("nav", 6e-10, 0.5), k=("hh", 5e-10, 0.5),
                                       sigma=0.3))
    return worlds.pack(ws), rng


def test_n2_matches_the_oracle_on_uneven_worlds(cuda):
    b, rng = uneven_batch()
    tissue = Tissue(b)
    ctl = T.Control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                    rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells)))
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(40):
        st, ok = N2.n2_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
    got, status, taken = run_n2(cuda, tissue, tissue.initial_state(),
                                tissue.pack_control(ctl.membrane, ctl.junction, ctl.pump,
                                                    ctl.channel), 1e-3, [15, 25])
    assert np.all(status == 0), [decode_status(s) for s in status]
    bad = {f: d for f, ref in oracle_state(st).items()
           if (d := scaled_difference(got[f], ref)) > TOL}
    assert not bad, bad


def test_n2_fused_launch_equals_one_step_launches_and_keeps_ledgers(cuda):
    torch = cuda
    b, _ = uneven_batch(43)
    tissue = Tissue(b)
    control = tissue.pack_control()
    fused, s1, _ = run_n2(torch, tissue, tissue.initial_state(), control, 1e-3, [30])
    single, s2, _ = run_n2(torch, tissue, tissue.initial_state(), control, 1e-3, [1] * 30)
    assert np.all(s1 == 0) and np.all(s2 == 0)
    for f in fused:
        assert np.array_equal(fused[f], single[f]), f
    dev = torch.device("cuda", tissue.device)
    st = torch.from_numpy(tissue.pack_state(fused)).to(dev)
    out = torch.zeros(b.worlds * 8, dtype=torch.float64, device=dev)
    tissue.balances(st, out)
    torch.cuda.synchronize(dev)
    res = out.cpu().numpy().reshape(b.worlds, 8)
    # The plain step's ledger bounds (tests/test_step_gpu.py): material against the reference
    # amounts, electrode and global charge against the electrode charge, 1e-12 relative.
    assert np.max(res[:, :3]) <= 1e-12 * np.max(np.abs(b.amount_reference))
    ec = np.max(np.abs(fused["electrode_charge"]))
    assert np.max(res[:, 3:5]) <= 1e-12 * ec
    for k, f in ((5, "reservoir_work"), (7, "metabolic_work")):
        assert np.max(res[:, k]) <= 1e-12 * np.max(np.abs(fused[f])), f


def test_n2_refuses_a_world_and_keeps_its_state(cuda):
    ws = [worlds.grid_world(4, 4, worlds.world_rng(12, k)) for k in range(3)]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    membrane = np.ones(b.cells)
    membrane[16:32] = 1.2  # world 1: availability above 1
    start = tissue.initial_state()
    got, status, taken = run_n2(cuda, tissue, start, tissue.pack_control(membrane=membrane),
                                1e-3, [5])
    assert status[0] == 0 and status[2] == 0 and status[1] & 8
    assert taken[1] == 0 and taken[0] == 5
    assert np.array_equal(got["amount_increment"][:, 16:32], start["amount_increment"][:, 16:32])


def test_n2_steps_where_the_explicit_step_is_refused_as_stiff(cuda):
    """Leak permeabilities x100 (charge relaxation in about 2 ms) at dt = 5 ms: the explicit
    ARS(2,2,2) refuses (CB_WORLD_STIFF); N2, with the slopes in the operator, steps, and agrees
    with the N2 oracle."""
    base = worlds.grid_world(6, 6, worlds.world_rng(13, 0))
    world = dataclasses.replace(base, permeability=base.permeability * 100.0)
    b = worlds.pack([world])
    tissue = Tissue(b)
    control = tissue.pack_control()
    _, status, _ = run_n2(cuda, tissue, tissue.initial_state(), control, 5e-3, [1],
                          method=_lib.METHOD_ARS222)
    assert status[0] & 64
    got, status, taken = run_n2(cuda, tissue, tissue.initial_state(), control, 5e-3, [20])
    assert status[0] == 0 and taken[0] == 20
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(20):
        st, ok = N2.n2_step(st, 5e-3, T.full_control(b), b, topo)
        assert ok.all()
    for f, ref in oracle_state(st).items():
        assert scaled_difference(got[f], ref) <= TOL, f


@pytest.mark.parametrize("name", ["n2_grid4x4.npz", "n2_channels_delaunay.npz"])
def test_mixed_n2_matches_the_reference_trajectory(cuda, name):
    """CB_METHOD_N2_MIXED (FP32 factor and substitutions, FP64 refinement of the stage charge
    residual): the reference's N2 trajectories within the FP64 tolerance."""
    z, b = load_golden(name)
    tissue = Tissue(b)
    control = tissue.pack_control(**{f: z["control_" + f] for f in
                                     ("membrane", "junction", "pump", "channel")
                                     if "control_" + f in z.files})
    state, done, worst = tissue.initial_state(), 0, {}
    for idx, target in enumerate(z["steps"]):
        if target > done:
            state, status, _ = run_n2(cuda, tissue, state, control, float(z["dt"]),
                                      [int(target - done)], method=_lib.METHOD_N2_MIXED)
            assert np.all(status == 0), decode_status(status[0])
            done = int(target)
        for f in T.State._fields:
            if "ref_" + f in z.files:
                worst[f] = max(worst.get(f, 0.0), scaled_difference(state[f], z["ref_" + f][idx]))
    bad = {k: v for k, v in worst.items() if v > TOL}
    assert not bad, bad


def test_mixed_n2_matches_fp64_n2_on_uneven_worlds(cuda):
    b, rng = uneven_batch(45)
    tissue = Tissue(b)
    control = tissue.pack_control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                                  rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells)))
    fp64, s1, _ = run_n2(cuda, tissue, tissue.initial_state(), control, 1e-3, [60])
    mixed, s2, _ = run_n2(cuda, tissue, tissue.initial_state(), control, 1e-3, [60],
                          method=_lib.METHOD_N2_MIXED)
    assert np.all(s1 == 0) and np.all(s2 == 0)
    bad = {f: d for f in fp64 if (d := scaled_difference(mixed[f], fp64[f])) > TOL}
    assert not bad, bad
