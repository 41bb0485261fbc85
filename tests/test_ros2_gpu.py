"""The device ROS2 step (cb_step with CB_METHOD_ROS2: Verwer's two-stage Rosenbrock method, one
sparse Cholesky of the cells' voltage operator per world per step) against the ROS2 oracle
(oracle/ros2.py, pinned by its order, ledger and stiffness tests against the oracle's RK4, which
reproduces the reference's rk4_checked_step).

Tolerances as the plain step's: every field within 1e-10 scaled difference of the oracle over the
whole run; ledgers conserved to 1e-12; a fused launch bit-identical to one-step launches.
"""

import dataclasses

import numpy as np
import pytest

from cells_b200 import _lib, worlds
from cells_b200.tissue import Tissue, decode_status
from conftest import scaled_difference
from gpu_util import oracle_state
from oracle import ros2 as RO
from oracle import tissue as T

pytestmark = pytest.mark.gpu
TOL = 1e-10


def run(torch, tissue, state, control, dt, chunks, method=_lib.METHOD_ROS2):
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


def uneven_batch(seed):
    rng = np.random.default_rng(seed)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(seed, k),
                                                     junction_sigma=0.3, gate=(0.02, 0.2, 0.9)),
                               rng, na=("nav", 1e-9, 0.5), k=("hh", 5e-10, 0.5), sigma=0.3)
          for k, n in enumerate((16, 140, 33, 700, 60))]
    return worlds.pack(ws), rng


def oracle_run(b, control, dt, steps):
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(steps):
        st, ok = RO.ros2_step(st, dt, control, b, topo)
        assert ok.all()
    return st


def test_ros2_matches_the_oracle_on_uneven_worlds(cuda):
    """Delaunay worlds of 16-700 cells with NaV1.2 + HH K populations, gated junctions and random
    partial controls, 60 steps of 1 ms in two launches."""
    b, rng = uneven_batch(61)
    tissue = Tissue(b)
    mem, jun = rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges)
    pmp, chn = rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells))
    got, status, taken = run(cuda, tissue, tissue.initial_state(),
                             tissue.pack_control(mem, jun, pmp, chn), 1e-3, [25, 35])
    assert np.all(status == 0), [decode_status(s) for s in status]
    assert np.all(taken == 35)
    ref = oracle_run(b, T.Control(mem, jun, pmp, chn), 1e-3, 60)
    bad = {f: d for f, r in oracle_state(ref).items()
           if (d := scaled_difference(got[f], r)) > TOL}
    assert not bad, bad


def test_ros2_4x4_world_for_10000_steps(cuda):
    """The single 4x4 CPU world (seed 0) by ROS2 at dt = 1 ms for 10,000 steps, against the oracle
    at steps 1, 100, 1000 and 10000 (1e-10); the FP32-factor form beside it, against the same
    FP64 oracle states at 1e-8 from step 100: its factor's rounding does not accumulate over the
    run. (After one step the junction transfers are a single step's flux between near-equal
    cells, the difference of nearly equal voltage rates; there the FP32 factor shows at 2.3e-8 of
    that field's own small scale.)"""
    b = worlds.pack([worlds.single_grid_tissue(0)])
    tissue = Tissue(b)
    control = tissue.pack_control()
    topo = T.topology(b)
    st = T.initial_state(b)
    state, done = tissue.initial_state(), 0
    mixed = tissue.initial_state()
    for target in (1, 100, 1000, 10000):
        state, status, taken = run(cuda, tissue, state, control, 1e-3, [target - done])
        assert status[0] == 0 and taken[0] == target - done
        mixed, status, taken = run(cuda, tissue, mixed, control, 1e-3, [target - done],
                                   method=_lib.METHOD_ROS2_MIXED)
        assert status[0] == 0 and taken[0] == target - done
        for _ in range(target - done):
            st, ok = RO.ros2_step(st, 1e-3, T.full_control(b), b, topo)
            assert ok.all()
        done = target
        bad = {f: d for f, r in oracle_state(st).items()
               if (d := scaled_difference(state[f], r)) > TOL}
        assert not bad, (target, bad)
        bad = {f: d for f, r in oracle_state(st).items()
               if (d := scaled_difference(mixed[f], r)) > (1e-8 if target >= 100 else 1e-7)}
        assert not bad, ("fp32 factor", target, bad)


def test_ros2_fused_equals_one_step_launches_and_conserves(cuda):
    b, rng = uneven_batch(62)
    tissue = Tissue(b)
    control = tissue.pack_control()
    fused, s1, _ = run(cuda, tissue, tissue.initial_state(), control, 1e-3, [40])
    single, s2, _ = run(cuda, tissue, tissue.initial_state(), control, 1e-3, [1] * 40)
    assert np.all(s1 == 0) and np.all(s2 == 0)
    for f in fused:
        assert np.array_equal(fused[f], single[f]), f
    dev = cuda.device("cuda", tissue.device)
    buf = cuda.from_numpy(tissue.pack_state(fused)).to(dev)
    out = cuda.zeros(b.worlds * 8, dtype=cuda.float64, device=dev)
    tissue.balances(buf, out)
    worst = out.view(-1, 8).max(dim=0).values.cpu().numpy()
    scale = float(np.max(np.abs(b.amount_reference)))
    assert worst[0] <= 1e-12 * scale and worst[2] <= 1e-12 * scale, worst


def test_ros2_steps_where_the_explicit_step_is_refused_as_stiff(cuda):
    """Leak permeabilities x100 at dt = 5 ms: the explicit ARS(2,2,2) refuses (CB_WORLD_STIFF);
    ROS2 steps and agrees with the oracle."""
    base = worlds.grid_world(6, 6, worlds.world_rng(13, 0))
    b = worlds.pack([dataclasses.replace(base, permeability=base.permeability * 100.0)])
    tissue = Tissue(b)
    control = tissue.pack_control()
    _, status, _ = run(cuda, tissue, tissue.initial_state(), control, 5e-3, [1],
                       method=_lib.METHOD_ARS222)
    assert status[0] & 64
    got, status, taken = run(cuda, tissue, tissue.initial_state(), control, 5e-3, [20])
    assert status[0] == 0 and taken[0] == 20
    ref = oracle_run(b, T.full_control(b), 5e-3, 20)
    for f, r in oracle_state(ref).items():
        assert scaled_difference(got[f], r) <= TOL, f


def test_ros2_refusal_keeps_the_state(cuda):
    b = worlds.pack([worlds.single_grid_tissue(0), worlds.single_grid_tissue(1),
                     worlds.single_grid_tissue(2)])
    tissue = Tissue(b)
    membrane = np.ones(b.cells)
    membrane[20] = 1.5  # world 1: an availability above 1
    start = tissue.initial_state()
    got, status, taken = run(cuda, tissue, start, tissue.pack_control(membrane=membrane), 1e-3,
                             [5])
    assert status[0] == 0 and status[2] == 0 and status[1] & 8
    assert taken[1] == 0 and taken[0] == 5
    assert np.array_equal(got["amount_increment"][:, 16:32], start["amount_increment"][:, 16:32])


def test_fp32_factor_ros2_within_1e8_of_fp64_and_conserves(cuda):
    """CB_METHOD_ROS2_MIXED (the voltage operator factored and substituted in FP32, no
    refinement): the uneven channel worlds with gated junctions and partial controls, 200 steps of
    1 ms, every state field within 1e-8 scaled difference of the FP64 oracle and of the device's
    FP64 ROS2 (each maximum printed), the ledgers balanced to 1e-12 of the material scale."""
    b, rng = uneven_batch(63)
    tissue = Tissue(b)
    mem, jun = rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges)
    pmp, chn = rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells))
    control = tissue.pack_control(mem, jun, pmp, chn)
    mixed, s1, _ = run(cuda, tissue, tissue.initial_state(), control, 1e-3, [100, 100],
                       method=_lib.METHOD_ROS2_MIXED)
    fp64, s2, _ = run(cuda, tissue, tissue.initial_state(), control, 1e-3, [100, 100])
    assert np.all(s1 == 0) and np.all(s2 == 0)
    ref = oracle_run(b, T.Control(mem, jun, pmp, chn), 1e-3, 200)
    vs_oracle = {f: scaled_difference(mixed[f], r) for f, r in oracle_state(ref).items()}
    vs_device = {f: scaled_difference(mixed[f], fp64[f]) for f in fp64}
    print("ROS2 FP32-factor vs FP64 oracle:", {k: f"{v:.1e}" for k, v in vs_oracle.items()})
    assert max(vs_oracle.values()) <= 1e-8, vs_oracle
    assert max(vs_device.values()) <= 1e-8, vs_device
    assert max(vs_device.values()) > 0.0  # the FP32 factor is in use
    dev = cuda.device("cuda", tissue.device)
    buf = cuda.from_numpy(tissue.pack_state(mixed)).to(dev)
    out = cuda.zeros(b.worlds * 8, dtype=cuda.float64, device=dev)
    tissue.balances(buf, out)
    worst = out.view(-1, 8).max(dim=0).values.cpu().numpy()
    scale = float(np.max(np.abs(b.amount_reference)))
    assert worst[0] <= 1e-12 * scale and worst[2] <= 1e-12 * scale, worst


def test_sparse_launch_setter_and_tuner(cuda):
    """cb_set_sparse_launch / cb_get_sparse_launch and autotune.tune_sparse: both CTA shapes step
    the same uneven worlds to within 1e-12 (the substitutions' narrow levels change form with
    the warp count, so the last bits may differ); 0 restores the plan's choice; other blocks are
    refused; the tuner times both and leaves the faster selected."""
    from cells_b200 import autotune

    b, rng = uneven_batch(64)
    tissue = Tissue(b)
    control = tissue.pack_control()
    default = tissue.get_sparse_launch()
    assert default in (128, 256)
    outs = {}
    for block in (128, 256):
        tissue.set_sparse_launch(block)
        assert tissue.get_sparse_launch() == block
        got, status, _ = run(cuda, tissue, tissue.initial_state(), control, 1e-3, [20])
        assert np.all(status == 0)
        outs[block] = got
    for f in outs[128]:
        assert scaled_difference(outs[128][f], outs[256][f]) <= 1e-12, f
    tissue.set_sparse_launch(0)
    assert tissue.get_sparse_launch() == default
    with pytest.raises(RuntimeError, match="128 or 256"):
        tissue.set_sparse_launch(64)
    dev = cuda.device("cuda", tissue.device)
    state = cuda.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    ctl = cuda.from_numpy(control).to(dev)
    best, timings = autotune.tune_sparse(tissue, state, ctl, 1e-3, steps=2, repeats=1, torch=cuda)
    assert best in (128, 256) and set(timings) == {128, 256}
    assert tissue.get_sparse_launch() == best
