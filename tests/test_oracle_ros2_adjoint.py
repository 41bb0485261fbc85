"""The ROS2 step's discrete adjoint (oracle/ros2_adjoint.py) against central finite differences
of the oracle's own ROS2 step, and its second derivatives (the Bernoulli function's curvature,
the channel laws' target'' and tau'') against differences of the slopes they differentiate.

Finite differences use h = 1e-6 relative, central, as tests/test_oracle_adjoint.py: 1e-6
relative agreement plus the differences' round-off floor of 2e-9 L, and the strongly coupled
parameters (|p dL/dp| above 1e-3 L) at 1e-6 outright.
"""

import numpy as np
import pytest

from cells_b200 import worlds
from oracle import adjoint as A
from oracle import ros2_adjoint as RA
from oracle import tissue as T

H = 1e-6
REL = 1e-6


def fd_gradients(world, params, steps, dt, target):
    copies = 2 * len(params)
    b = worlds.pack([world] * copies)
    for j, (name, s, i) in enumerate(params):
        arr = getattr(b, name)
        off = b.edge_offset if name == "junction_permeability" else b.cell_offset
        arr[s, off[2 * j] + i] *= 1 + H
        arr[s, off[2 * j + 1] + i] *= 1 - H
    loss = RA.trajectory_loss(T.initial_state(b), dt, T.full_control(b), b, steps,
                              np.tile(target, copies))
    base = worlds.pack([world])
    return np.array([(loss[2 * j] - loss[2 * j + 1]) / (2 * H * getattr(base, name)[s, i])
                     for j, (name, s, i) in enumerate(params)])


def pick(b, rng, n):
    out = []
    for _ in range(n):
        kind = rng.integers(0, 3 if b.channel_slots else 2)
        if kind == 0:
            out.append(("permeability", int(rng.integers(3)), int(rng.integers(b.cells))))
        elif kind == 1:
            out.append(("junction_permeability", int(rng.integers(3)), int(rng.integers(b.edges))))
        else:
            out.append(("channel_permeability", int(rng.integers(b.channel_slots)),
                        int(rng.integers(b.cells))))
    return out


def values(grads, params):
    table = {"permeability": grads.membrane, "junction_permeability": grads.junction,
             "channel_permeability": grads.channel}
    return np.array([table[name][s, i] for name, s, i in params])


@pytest.mark.parametrize("case", ["gated_channels", "grid"])
def test_ros2_adjoint_matches_central_differences(case):
    if case == "gated_channels":
        rng = worlds.world_rng(3, 0)
        world = worlds.delaunay_world(30, rng, gate=(0.015, 0.2, 1.0))
        world = worlds.with_channels(world, rng, **worlds.UNEVEN_CHANNELS)
    else:
        world = worlds.grid_world(4, 4, worlds.world_rng(0, 0))
    b = worlds.pack([world])
    target = worlds.voltage_target(b)
    steps, dt = 30, 1e-3
    loss, grads, refused = RA.trajectory_grad(T.initial_state(b), dt, T.full_control(b), b,
                                              steps, target)
    assert refused[0] == 0
    params = pick(b, np.random.default_rng(1), 16)
    fd = fd_gradients(world, params, steps, dt, target)
    ad = values(grads, params)
    p = np.array([getattr(b, name)[s, i] for name, s, i in params])
    err = np.abs(p * (ad - fd))
    bound = REL * np.abs(p * fd) + 2e-9 * loss[0]
    assert np.all(err <= bound), (err / bound).max()
    strong = np.abs(p * fd) > 1e-3 * loss[0]
    assert strong.sum() >= 3
    assert np.all(err[strong] <= REL * np.abs(p * fd)[strong])


def test_ros2_adjoint_differs_from_frozen_jacobian():
    """The W-matrix's own dependence on the state and the permeabilities matters at this bar:
    leaving out J^T(y) (the second-derivative terms) changes the gradients by more than ten
    times the 1e-6 bar."""
    world = worlds.grid_world(4, 4, worlds.world_rng(0, 0))
    b = worlds.pack([world])
    topo = T.topology(b)
    st = T.initial_state(b)
    for _ in range(5):
        st, _ = RA.R2.ros2_step(st, 1e-3, T.full_control(b), b, topo)
    rng = np.random.default_rng(4)
    cot = (rng.normal(size=(3, b.cells)), np.zeros(b.edges), np.zeros_like(st.channel_gate))
    _, full, _, _ = RA.step_vjp(st, 1e-3, T.full_control(b), b, topo, *cot)
    saved = RA.pieces_vjp
    try:
        RA.pieces_vjp = lambda pc, state, control, jb, b, topo: (
            np.zeros((3, b.cells)), np.zeros(b.edges), np.zeros_like(state.channel_gate),
            A.zero_grads(b))
        _, frozen, _, _ = RA.step_vjp(st, 1e-3, T.full_control(b), b, topo, *cot)
    finally:
        RA.pieces_vjp = saved
    rel = np.max(np.abs(full.membrane - frozen.membrane)) / np.max(np.abs(full.membrane))
    assert rel > 1e-5


def test_curvature_matches_differences():
    # Closed form (|x| >= 0.1) against central differences of B' (B' near -1 for large negative
    # arguments, so the differences carry ~1e-16 / h of absolute noise).
    x = np.concatenate([np.linspace(0.1, 40, 400), -np.linspace(0.1, 40, 400)])
    h = 1e-5 * np.abs(x)
    fd = (A.bernoulli_slope(x + h) - A.bernoulli_slope(x - h)) / (2 * h)
    scale = np.maximum(np.abs(fd), 1e-12)
    assert np.all(np.abs(RA.curvature(x) - fd) <= 1e-7 * scale + 2e-11)
    # Series below 0.1: against the closed form, which loses few digits above 1e-2.
    xs = np.geomspace(1e-2, 0.0999, 40)
    a = xs
    om = -np.expm1(-a)
    closed = (1.0 - om) * (a * (2.0 - om) - 2.0 * om) / om**3
    assert np.allclose(RA.curvature(xs), closed, rtol=1e-10, atol=0)
    assert np.allclose(RA.curvature(-xs), closed, rtol=1e-10, atol=0)
    # Continuous across the switch, even, and 1/6 at 0.
    e = np.array([0.1 * (1 - 1e-12), 0.1 * (1 + 1e-12)])
    assert abs(np.diff(RA.curvature(e))[0]) < 1e-13
    assert RA.curvature(0.0) == 1.0 / 6.0


@pytest.mark.parametrize("code", [T.KV1P5, T.NAV1P2, T.HH_K_N4])
def test_channel_curvature_matches_differences(code):
    v = np.linspace(-0.115, 0.055, 171)
    codes = np.full((1, v.size), code)
    h = 1e-7
    t, dt_, d2t, kap, dkap, d2kap = RA.channel_kinetics_curvature(v[None], codes)
    tp, kp = RA.channel_kinetics_curvature(v[None] + h, codes)[1::3][0], \
        RA.channel_kinetics_curvature(v[None] + h, codes)[4]
    tm, km = RA.channel_kinetics_curvature(v[None] - h, codes)[1::3][0], \
        RA.channel_kinetics_curvature(v[None] - h, codes)[4]
    targets, tau = T.channel_kinetics(v[None], codes)
    rows = T.gate_rows_active(codes)
    assert np.allclose(np.where(rows, t, 0), np.where(rows, targets, 0), rtol=1e-13, atol=0)
    assert np.allclose(np.where(rows, kap * tau, 1), 1.0, rtol=1e-13)
    ds, dtau = A.channel_kinetics_slope(v[None], codes)
    assert np.allclose(np.where(rows, dt_, 0), np.where(rows, ds, 0), rtol=1e-9, atol=1e-12)
    assert np.allclose(np.where(rows, dkap, 0), np.where(rows, -dtau / tau**2, 0), rtol=1e-9,
                       atol=1e-9)
    for got, fp, fm in ((d2t, tp, tm), (d2kap, kp, km)):
        fd = (fp - fm) / (2 * h)
        scale = np.max(np.abs(fd), axis=-1, keepdims=True) + 1e-30
        assert np.all(np.abs(np.where(rows, got - fd, 0)) <= 1e-6 * scale)


def test_refused_world_contributes_nothing():
    """A world refused at the step (a membrane availability above 1) keeps its state; its
    cotangent passes through unchanged and its gradients stay zero."""
    ws = [worlds.grid_world(3, 3, worlds.world_rng(9, k)) for k in range(2)]
    b = worlds.pack(ws)
    topo = T.topology(b)
    control = T.full_control(b)
    control.membrane[:9] = 1.5  # world 0 only
    st = T.initial_state(b)
    rng = np.random.default_rng(2)
    cot = (rng.normal(size=(3, b.cells)), rng.normal(size=b.edges),
           np.zeros_like(st.channel_gate))
    (lam_n, lam_g, _), grads, _, valid = RA.step_vjp(st, 1e-3, control, b, topo, *cot)
    assert not valid[0] and valid[1]
    assert np.array_equal(lam_n[:, :9], cot[0][:, :9])
    assert np.array_equal(lam_g[:b.edge_offset[1]], cot[1][:b.edge_offset[1]])
    assert not grads.membrane[:, :9].any() and grads.membrane[:, 9:].any()
