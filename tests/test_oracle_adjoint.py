"""The oracle's discrete adjoint (oracle/adjoint.py) against central finite differences of the
oracle's own step (itself pinned to the reference's step), and each hand-derived slope against
differences of the function it differentiates.

Finite differences use h = 1e-6 relative, central. Their own error is round-off: the loss is
known to about 1e-16 of its size, so a difference carries about 1e-16 L / h of noise; the test
asks for 1e-6 relative agreement plus that floor (2e-9 L in units of p dL/dp).
"""

import numpy as np
import pytest

from cells_b200 import worlds
from oracle import adjoint as A
from oracle import tissue as T

H = 1e-6
REL = 1e-6


def fd_gradients(world, params, steps, dt, target):
    """Central differences of the per-world loss for each (field, species/slot, index): one
    batch of 2 copies per parameter, all stepped together."""
    copies = 2 * len(params)
    b = worlds.pack([world] * copies)
    for j, (name, s, i) in enumerate(params):
        arr = getattr(b, name)
        off = b.edge_offset if name == "junction_permeability" else b.cell_offset
        arr[s, off[2 * j] + i] *= 1 + H
        arr[s, off[2 * j + 1] + i] *= 1 - H
    loss = A.trajectory_loss(T.initial_state(b), dt, T.full_control(b), b, steps,
                             np.tile(target, copies))
    base = worlds.pack([world])
    return np.array([(loss[2 * j] - loss[2 * j + 1]) / (2 * H * getattr(base, name)[s, i])
                     for j, (name, s, i) in enumerate(params)])


def pick(world, rng, n):
    b = worlds.pack([world])
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


def adjoint_values(grads, params):
    table = {"permeability": grads.membrane, "junction_permeability": grads.junction,
             "channel_permeability": grads.channel}
    return np.array([table[name][s, i] for name, s, i in params])


@pytest.mark.parametrize("case", ["gated_channels", "pinned_grid"])
def test_adjoint_matches_central_differences(case):
    if case == "gated_channels":
        rng = worlds.world_rng(3, 0)
        world = worlds.delaunay_world(30, rng, gate=(0.015, 0.2, 1.0))
        world = worlds.with_channels(world, rng, **worlds.UNEVEN_CHANNELS)
    else:
        world = worlds.grid_world(4, 4, worlds.world_rng(0, 0))
    b = worlds.pack([world])
    target = worlds.voltage_target(b)
    steps, dt = 50, 1e-3
    loss, grads, refused = A.trajectory_grad(T.initial_state(b), dt, T.full_control(b), b, steps,
                                             target)
    assert refused[0] == 0
    params = pick(world, np.random.default_rng(1), 20)
    fd = fd_gradients(world, params, steps, dt, target)
    ad = adjoint_values(grads, params)
    p = np.array([getattr(b, name)[s, i] for name, s, i in params])
    err = np.abs(p * (ad - fd))
    bound = REL * np.abs(p * fd) + 2e-9 * loss[0]
    assert np.all(err <= bound), (err / bound).max()
    # The strongly coupled ones (|p dL/dp| above 1e-3 L) meet 1e-6 relative outright.
    strong = np.abs(p * fd) > 1e-3 * loss[0]
    assert strong.sum() >= 3
    assert np.all(err[strong] <= REL * np.abs(p * fd)[strong])


def test_bernoulli_slope_matches_differences():
    x = np.concatenate([np.linspace(-40, 40, 801), np.geomspace(1e-8, 5e-2, 60),
                        -np.geomspace(1e-8, 5e-2, 60)])
    h = 1e-6 * np.maximum(np.abs(x), 1e-2)
    fd = (T.bernoulli(x + h) - T.bernoulli(x - h)) / (2 * h)
    assert np.allclose(A.bernoulli_slope(x), fd, rtol=1e-6, atol=1e-9)
    # Continuity across the series switch at |x| = 1e-2.
    e = np.array([1e-2 * (1 - 1e-12), 1e-2 * (1 + 1e-12)])
    for sgn in (1, -1):
        v = A.bernoulli_slope(sgn * e)
        assert abs(v[0] - v[1]) < 1e-14


@pytest.mark.parametrize("code", [T.KV1P5, T.NAV1P2, T.HH_K_N4])
def test_channel_slopes_match_differences(code):
    v = np.linspace(-0.115, 0.055, 171)
    codes = np.full((1, v.size), code)
    h = 1e-7
    tp, taup = T.channel_kinetics(v[None] + h, codes)
    tm, taum = T.channel_kinetics(v[None] - h, codes)
    dt, dtau = A.channel_kinetics_slope(v[None], codes)
    for got, fp, fm in ((dt, tp, tm), (dtau, taup, taum)):
        fd = (fp - fm) / (2 * h)
        scale = np.max(np.abs(fd), axis=-1, keepdims=True) + 1e-30
        assert np.all(np.abs(got - fd) <= 1e-6 * scale)


def test_gate_advance_partials_match_differences():
    rng = np.random.default_rng(5)
    n = 200
    g, ts, te = rng.uniform(0, 1, n), rng.uniform(0, 1, n), rng.uniform(0, 1, n)
    taus, taue = 10 ** rng.uniform(-4, 0, n), 10 ** rng.uniform(-4, 0, n)
    h = np.where(rng.random(n) < 0.5, 1e-3, 2.9e-4)
    args = [g, ts, taus, te, taue]
    parts = A.advance_partials(*args, h)
    for k in range(5):
        step = 1e-4 * args[k] if k in (2, 4) else np.full(n, 1e-5)  # time constants: relative
        up = [a.copy() for a in args]
        dn = [a.copy() for a in args]
        up[k] += step
        dn[k] -= step
        fd = (T.advance_gates(*up, h) - T.advance_gates(*dn, h)) / (2 * step)
        assert np.allclose(parts[k], fd, rtol=1e-5, atol=1e-9), k


def test_refused_world_contributes_nothing():
    """A world refused at every step (a membrane availability above 1) keeps its state; its
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
    (lam_n, lam_g, _), grads, _, valid = A.step_vjp(st, 1e-3, control, b, topo, *cot)
    assert not valid[0] and valid[1]
    assert np.array_equal(lam_n[:, :9], cot[0][:, :9])
    assert np.array_equal(lam_g[:b.edge_offset[1]], cot[1][:b.edge_offset[1]])
    assert not grads.membrane[:, :9].any() and grads.membrane[:, 9:].any()
