"""The device adjoint of the ROS2 step (cb_step_vjp_method with CB_METHOD_ROS2, the autograd
Function with method=METHOD_ROS2): against the oracle's ROS2 adjoint on the same steps
(cotangents and permeability gradients), against central finite differences of the device's own
ROS2 forward (h = 1e-6 relative, the differences' round-off floor allowed as in
tests/test_oracle_ros2_adjoint.py), checkpoint-interval invariance, refusals and the
ledger-cotangent flag."""

import numpy as np
import pytest

from cells_b200 import _lib, worlds
from cells_b200.tissue import Tissue
from conftest import scaled_difference
from oracle import adjoint as A
from oracle import ros2 as R2
from oracle import ros2_adjoint as RA
from oracle import tissue as T

pytestmark = pytest.mark.gpu
VJP_TOL = 1e-9  # device vs oracle adjoint, scaled difference per field
H = 1e-6
ROS2 = _lib.METHOD_ROS2


def gated_batch():
    ws = [worlds.grid_world(4, 4, worlds.world_rng(31, 0), gate=(0.015, 0.2, 1.0)),
          worlds.delaunay_world(60, worlds.world_rng(31, 1), gate=(0.01, 0.3, 0.9)),
          worlds.delaunay_world(150, worlds.world_rng(31, 2))]
    return worlds.pack(ws)


def channel_batch():
    rng = np.random.default_rng(32)
    ws = []
    for k, (n, gate) in enumerate(((50, (0.015, 0.2, 1.0)), (200, None), (33, None))):
        w = worlds.delaunay_world(n, worlds.world_rng(32, k), gate=gate)
        ws.append(worlds.with_channels(w, rng, **worlds.UNEVEN_CHANNELS))
    return worlds.pack(ws)


def device_vjp(torch, tissue, control, dt, n_steps, cot_fields):
    dev = torch.device("cuda", tissue.device)
    b = tissue.batch
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    ctl = torch.from_numpy(control).to(dev)
    cot = {f: np.zeros_like(v) for f, v in tissue.initial_state().items()}
    cot.update(cot_fields)
    cot_out = torch.from_numpy(tissue.pack_state(cot)).to(dev)
    cot_in = torch.empty_like(cot_out)
    gm = torch.zeros(3 * b.cells, dtype=torch.float64, device=dev)
    gj = torch.zeros(3 * b.edges, dtype=torch.float64, device=dev)
    gch = torch.zeros(max(b.channel_slots * b.cells, 1), dtype=torch.float64, device=dev)
    ws = torch.empty(tissue.vjp_workspace_bytes(n_steps, ROS2), dtype=torch.uint8, device=dev)
    status = torch.full((b.worlds,), 7, dtype=torch.int32, device=dev)
    tissue.step_vjp(state, ctl, dt, n_steps, cot_out, cot_in, gm, gj,
                    gch if b.channel_slots else None, ws, status, method=ROS2)
    torch.cuda.synchronize(dev)
    return (tissue.unpack_state(cot_in.cpu().numpy()), gm.cpu().numpy().reshape(3, b.cells),
            gj.cpu().numpy().reshape(3, b.edges),
            gch.cpu().numpy()[:b.channel_slots * b.cells].reshape(b.channel_slots, b.cells),
            status.cpu().numpy())


def oracle_vjp(b, control, dt, n_steps, cot):
    topo = T.topology(b)
    states = [T.initial_state(b)]
    for _ in range(n_steps):
        states.append(R2.ros2_step(states[-1], dt, control, b, topo)[0])
    total = A.zero_grads(b)
    for t in range(n_steps - 1, -1, -1):
        cot, g, _, _ = RA.step_vjp(states[t], dt, control, b, topo, *cot)
        total = A.Grads(*(x + y for x, y in zip(total, g, strict=True)))
    return cot, total


@pytest.mark.parametrize("which", ["gated", "channels"])
def test_ros2_vjp_matches_oracle_adjoint(cuda, which):
    b = gated_batch() if which == "gated" else channel_batch()
    tissue = Tissue(b)
    rng = np.random.default_rng(6)
    ctl = T.Control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                    rng.uniform(0.6, 1, b.cells), rng.uniform(0.5, 1, (b.channel_slots, b.cells)))
    control = tissue.pack_control(ctl.membrane, ctl.junction, ctl.pump, ctl.channel)
    cot = (rng.normal(size=(3, b.cells)), rng.normal(size=b.edges),
           rng.normal(size=(2, b.channel_slots, b.cells)))
    dt, n = 1e-3, 15
    got, gm, gj, gch, status = device_vjp(cuda, tissue, control, dt, n, {
        "amount_increment": cot[0], "junction_gate": cot[1], "channel_gate": cot[2]})
    assert np.all(status == 0)
    (lam_n, lam_g, lam_c), ref = oracle_vjp(b, ctl, dt, n, cot)
    bad = {}
    for name, a, r in (("amount", got["amount_increment"], lam_n),
                       ("junction_gate", got["junction_gate"], lam_g),
                       ("channel_gate", got["channel_gate"], lam_c),
                       ("grad_membrane", gm, ref.membrane), ("grad_junction", gj, ref.junction),
                       ("grad_channel", gch, ref.channel)):
        d = scaled_difference(a, r)
        if d > VJP_TOL:
            bad[name] = d
    assert not bad, bad


def test_ros2_gradient_matches_device_finite_differences(cuda):
    """64 random permeabilities of a 64-cell Delaunay tissue with NaV1.2 and HH K channels,
    200 ROS2 steps: the autograd gradient against central differences of the device's ROS2
    forward, every perturbed copy a world of one batch."""
    torch = cuda
    from cells_b200 import adjoint

    rng = worlds.world_rng(33, 0)
    world = worlds.with_channels(worlds.delaunay_world(64, rng), rng, **worlds.UNEVEN_CHANNELS)
    b1 = worlds.pack([world])
    target = worlds.voltage_target(b1)
    dt, steps = 1e-3, 200
    tissue = Tissue(b1)
    dev = torch.device("cuda", tissue.device)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    pm, pj, pc = (t.requires_grad_() for t in adjoint.permeabilities(tissue))
    final, refused = adjoint.trajectory(tissue, state, control, dt, steps, pm, pj, pc, every=50,
                                        method=ROS2)
    loss = adjoint.voltage_loss(tissue, final, torch.tensor(target, device=dev))
    loss.sum().backward()
    assert int(refused.abs().max()) == 0
    grads = {"permeability": pm.grad.cpu().numpy(), "junction_permeability": pj.grad.cpu().numpy(),
             "channel_permeability": pc.grad.cpu().numpy()}
    pick = np.random.default_rng(3)
    params = []
    for _ in range(64):
        kind = ("permeability", "junction_permeability", "channel_permeability")[pick.integers(3)]
        rows = 2 if kind == "channel_permeability" else 3
        n = b1.edges if kind == "junction_permeability" else b1.cells
        params.append((kind, int(pick.integers(rows)), int(pick.integers(n))))
    copies = worlds.pack([world] * (2 * len(params)))
    for j, (name, s, i) in enumerate(params):
        arr = getattr(copies, name)
        off = copies.edge_offset if name == "junction_permeability" else copies.cell_offset
        arr[s, off[2 * j] + i] *= 1 + H
        arr[s, off[2 * j + 1] + i] *= 1 - H
    many = Tissue(copies)
    st = torch.from_numpy(many.pack_state(many.initial_state())).to(dev)
    out = torch.empty_like(st)
    status = torch.zeros(copies.worlds, dtype=torch.int32, device=dev)
    many.step(st, out, torch.from_numpy(many.pack_control()).to(dev), dt, steps, status,
              method=ROS2)
    losses = adjoint.voltage_loss(many, out, torch.tensor(np.tile(target, 2 * len(params)),
                                                          device=dev)).cpu().numpy()
    assert int(status.abs().max()) == 0
    L = float(loss.detach().cpu().numpy()[0])
    worst, strong = 0.0, 0
    for j, (name, s, i) in enumerate(params):
        p = getattr(b1, name)[s, i]
        fd = (losses[2 * j] - losses[2 * j + 1]) / (2 * H * p)
        ad = grads[name][s, i]
        err = abs(p * (ad - fd))
        assert err <= 1e-6 * abs(p * fd) + 2e-9 * L, (name, s, i, p * ad, p * fd)
        if abs(p * fd) > 1e-3 * L:
            strong += 1
            worst = max(worst, err / abs(p * fd))
    assert strong >= 16 and worst <= 1e-6


def test_ros2_checkpoint_interval_does_not_change_the_gradient(cuda):
    """Checkpoints every 40, 7 or 1 steps give the same gradient (to 1e-12: checkpoint states
    come from fused launches, the recompute from one-step launches)."""
    torch = cuda
    from cells_b200 import adjoint

    b = channel_batch()
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    target = torch.tensor(worlds.voltage_target(b), device=dev)
    results = []
    for every in (40, 7, 1):
        params = [t.requires_grad_() for t in adjoint.permeabilities(tissue)]
        final, _ = adjoint.trajectory(tissue, state, control, 1e-3, 40, *params, every=every,
                                      method=ROS2)
        adjoint.voltage_loss(tissue, final, target).sum().backward()
        results.append([p.grad.cpu().numpy() for p in params])
    for other in results[1:]:
        for a, r in zip(other, results[0], strict=True):
            assert scaled_difference(a, r) <= 1e-12


def test_ros2_refused_world_and_ledger_cotangent(cuda):
    """World 0 refused at every step (a membrane availability above 1): its cotangent passes
    through and it gets no gradient. World 1 gets a ledger cotangent: flagged."""
    ws = [worlds.grid_world(3, 3, worlds.world_rng(9, k)) for k in range(3)]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    membrane = np.ones(b.cells)
    membrane[:9] = 1.5
    control = tissue.pack_control(membrane=membrane)
    rng = np.random.default_rng(4)
    cot_n = rng.normal(size=(3, b.cells))
    pump = np.zeros(b.cells)
    pump[9:18] = 1.0  # world 1's pump-cycle ledger
    got, gm, _, _, status = device_vjp(cuda, tissue, control, 1e-3, 5,
                                       {"amount_increment": cot_n, "pump_cycles": pump})
    assert status[0] != 0 and not status[0] & 256
    assert status[1] & 256 and status[2] == 0
    assert np.array_equal(got["amount_increment"][:, :9], cot_n[:, :9])
    assert not gm[:, :9].any() and gm[:, 9:].any()
    assert np.array_equal(got["pump_cycles"], pump)  # ledger cotangents pass through


def test_ros2_vjp_arguments(cuda):
    """The reverse refuses an undersized workspace and a method it does not cover (the
    FP32-factor form), with an error and no launch; zero steps pass the cotangent through and add
    nothing to the gradients."""
    torch = cuda
    b = worlds.pack([worlds.grid_world(3, 3, worlds.world_rng(9, 0))])
    tissue = Tissue(b)
    dev = torch.device("cuda", tissue.device)
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    control = torch.from_numpy(tissue.pack_control()).to(dev)
    rng = np.random.default_rng(3)
    cot = {f: np.zeros_like(v) for f, v in tissue.initial_state().items()}
    cot["amount_increment"] = rng.normal(size=(3, b.cells))
    cot_out = torch.from_numpy(tissue.pack_state(cot)).to(dev)
    cot_in = torch.zeros_like(cot_out)
    gm = torch.zeros(3 * b.cells, dtype=torch.float64, device=dev)
    gj = torch.zeros(3 * b.edges, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    need = tissue.vjp_workspace_bytes(4, ROS2)
    small = torch.empty(need - 256, dtype=torch.uint8, device=dev)
    with pytest.raises(RuntimeError, match="workspace too small"):
        tissue.step_vjp(state, control, 1e-3, 4, cot_out, cot_in, gm, gj, None, small, status,
                        method=ROS2)
    ws = torch.empty(need, dtype=torch.uint8, device=dev)
    with pytest.raises(RuntimeError, match="the reverse covers"):
        tissue.step_vjp(state, control, 1e-3, 4, cot_out, cot_in, gm, gj, None, ws, status,
                        method=_lib.METHOD_ROS2_MIXED)
    tissue.step_vjp(state, control, 1e-3, 0, cot_out, cot_in, gm, gj, None, ws, status,
                    method=ROS2)
    torch.cuda.synchronize(dev)
    assert torch.equal(cot_in, cot_out)
    assert not gm.any() and not gj.any() and int(status.item()) == 0


def test_ros2_vjp_on_a_benchmark_world(cuda):
    """One world of the adjoint benchmark (a 1024-cell Delaunay tissue with NaV1.2 and HH K
    populations, from the benchmark's generator): its factor plan does not fit shared memory, so
    the forward runs the four-CTAs-per-SM shape from global memory. 10 ROS2 steps: the device's
    reverse against the oracle's at 1e-9 on the cotangents and gradients."""
    b = worlds.pack([worlds.uneven_world(0, 1024, 4, worlds.UNEVEN_CHANNELS)])
    tissue = Tissue(b)
    rng = np.random.default_rng(8)
    cot = (rng.normal(size=(3, b.cells)), rng.normal(size=b.edges),
           rng.normal(size=(2, b.channel_slots, b.cells)))
    dt, n = 1e-3, 10
    got, gm, gj, gch, status = device_vjp(cuda, tissue, tissue.pack_control(), dt, n, {
        "amount_increment": cot[0], "junction_gate": cot[1], "channel_gate": cot[2]})
    assert np.all(status == 0)
    (lam_n, lam_g, lam_c), ref = oracle_vjp(b, T.full_control(b), dt, n, cot)
    bad = {name: d for name, a, r in (("amount", got["amount_increment"], lam_n),
                                       ("junction_gate", got["junction_gate"], lam_g),
                                       ("channel_gate", got["channel_gate"], lam_c),
                                       ("grad_membrane", gm, ref.membrane),
                                       ("grad_junction", gj, ref.junction),
                                       ("grad_channel", gch, ref.channel))
           if (d := scaled_difference(a, r)) > VJP_TOL}
    assert not bad, bad
