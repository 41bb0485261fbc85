"""The open-channel block on the device (cb_set_channel_block; the packed kernel's blocked form)
against the reference's own @3 trajectories with blocked populations and against the oracle.

Tolerances as the unblocked step's: every state field within 1e-10 scaled difference of the
reference's trajectory and of the oracle. Bit-exact: a blocked batch whose populations all
declare no block (u = 1 exactly) steps as the unblocked packed kernel; the library's static
scratch entry point gives cb_step's bits on a blocked batch.
"""

import ctypes

import numpy as np
import pytest

from cells_b200 import _lib, worlds
from cells_b200.tissue import Tissue
from conftest import load_golden, scaled_difference
from gpu_util import oracle_state, run_device
from oracle import tissue as T
from test_step_gpu import TRAJECTORY_TOL, _golden_replay

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["ars222_v3_block.npz", "ars222_v3_block_delaunay.npz"])
def test_blocked_device_matches_reference_trajectory(cuda, name):
    worst = _golden_replay(cuda, name)
    bad = {k: v for k, v in worst.items() if v > TRAJECTORY_TOL}
    assert not bad, bad


def blocked_batch(seed=61):
    """Uneven Delaunay worlds with Na and K populations: blocks on slot 0, slot 1, both, none."""
    rng = np.random.default_rng(seed)
    ws = []
    for k, n in enumerate((40, 150, 333, 90)):
        w = worlds.with_channels(
            worlds.delaunay_world(n, worlds.world_rng(seed, k), junction_sigma=0.3,
                                  gate=(0.02, 0.2, 0.9)), rng,
            na=("nav", 3e-10, 0.5), k=("hh", 4e-10, 0.5), sigma=0.3)
        if k in (0, 2):
            worlds.with_block(w, rng, slot=0, fraction=0.7)
        if k in (1, 2):
            worlds.with_block(w, rng, slot=1, fraction=0.9, side="inside",
                              concentration_mM=(0.1, 1.0),
                              modes=((0.5, 0.05, 0.9), (0.25, 0.5, 0.5), (0.25, 5.0, 0.1)))
        ws.append(w)
    return worlds.pack(ws)


def test_blocked_device_matches_oracle_uneven(cuda):
    b = blocked_batch()
    tissue = Tissue(b)
    assert tissue.get_launch()[0] == _lib.KERNEL_PACKED
    topo = T.topology(b)
    ctl = T.full_control(b, channel=0.8)
    st = T.initial_state(b)
    for _ in range(120):
        st, ok = T.ars222_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
    got, status, taken = run_device(cuda, tissue, tissue.initial_state(),
                                    tissue.pack_control(channel=0.8), 1e-3, 120,
                                    chunks=[20, 100])
    assert np.all(status == 0) and np.all(taken == 100)
    for f, ref in oracle_state(st).items():
        assert scaled_difference(got[f], ref) <= TRAJECTORY_TOL, f


def test_undeclared_block_steps_as_the_unblocked_packed_kernel(cuda):
    b = blocked_batch(62)
    b.channel_block = worlds.unblocked(b.channel_slots, b.cells, 2)
    blocked = Tissue(b)
    b.channel_block = None
    plain = Tissue(b)
    plain.set_launch(_lib.KERNEL_PACKED, 1024)
    assert blocked.get_launch() == plain.get_launch()
    start, control = plain.initial_state(), plain.pack_control(channel=0.7)
    x, sx, _ = run_device(cuda, blocked, start, control, 1e-3, 50)
    y, sy, _ = run_device(cuda, plain, start, control, 1e-3, 50)
    assert np.array_equal(sx, sy)
    for f in x:
        assert np.array_equal(x[f], y[f]), f


def test_blocked_static_scratch_entry_matches_cb_step(cuda):
    torch = cuda
    b = blocked_batch(63)
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    start = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
    a, c = start.clone(), start.clone()  # the layout's padding is never written
    tissue.step(start, a, control, 1e-3, 30, status)
    _lib.check(tissue.lib.cb_step_packed_static(
        tissue.handle, ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(c.data_ptr()), 1e-3,
        ctypes.c_void_p(control.data_ptr()), 30, ctypes.c_void_p(status.data_ptr()), None,
        None))
    torch.cuda.synchronize(dev)
    assert torch.equal(a, c)


def test_blocked_batch_refusals(cuda):
    torch = cuda
    b = blocked_batch(64)
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    status = torch.zeros(b.worlds, dtype=torch.int32, device=dev)
    with pytest.raises(RuntimeError, match="N2"):
        tissue.step(state, state, control, 1e-3, 1, status, method=_lib.METHOD_N2)
    with pytest.raises(RuntimeError, match="CB_METHOD_ARS222"):
        tissue.step(state, state, control, 1e-3, 1, status, method=_lib.METHOD_ARS222_MIXED)
    with pytest.raises(RuntimeError, match="packed kernel only"):
        tissue.set_launch(_lib.KERNEL_SHARED, 256, 3)
    bad = worlds.ChannelBlock(*(np.array(getattr(b.channel_block, f)) for f in (
        "declared", "weight", "k0_mM", "distance", "modes_declared", "valence", "side",
        "concentration_mM")))
    bad.weight[0, 0, 0] = 0.9  # this population's weights no longer sum to 1
    with pytest.raises(RuntimeError, match="sum to 1"):
        tissue.set_channel_block(bad)
    bad.weight[0, 0, 0] = b.channel_block.weight[0, 0, 0]
    bad.concentration_mM[1, 3] = 2e3
    with pytest.raises(RuntimeError, match="blocker concentration"):
        tissue.set_channel_block(bad)
    tissue.set_channel_block(None)  # removing the block lets the other methods run again
    tissue.step(state, state, control, 1e-3, 1, status, method=_lib.METHOD_N2)
    torch.cuda.synchronize(dev)
    assert torch.all(status == 0)
