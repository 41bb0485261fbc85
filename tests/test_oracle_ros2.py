"""The ROS2 oracle (oracle/ros2.py: Verwer's two-stage Rosenbrock method on the reference's
held-bath right-hand side). The reference has no Rosenbrock method on this path, so the method is
pinned the way the reference pins its integrators (tests/unit/test_surface_pump_v3_imex.py:
136-142, observed order against an RK4 run at a small step; tests/unit/test_rosenbrock_dense.py:
40-66, order and stiff damping), plus the conservation ledgers every step.
"""

import dataclasses

import numpy as np
import pytest

from cells_b200 import worlds
from oracle import ros2 as RO
from oracle import tissue as T

SPAN = 0.01  # s


def _run(step, b, dt, n, control=None):
    topo = T.topology(b)
    control = T.full_control(b) if control is None else control
    st = T.initial_state(b)
    for _ in range(n):
        st, ok = step(st, dt, control, b, topo)
        assert np.all(ok)
    return st


def _channel_world():
    rng = np.random.default_rng(5)
    w = worlds.delaunay_world(40, worlds.world_rng(15, 0), junction_sigma=0.3,
                              gate=(0.02, 0.2, 0.9))
    return worlds.pack([worlds.with_channels(w, rng, na=("nav", 1e-9, 0.5),
                                             k=("hh", 5e-10, 0.5), sigma=0.3)])


@pytest.mark.parametrize("kind", ["grid", "channels"])
def test_ros2_is_second_order_against_rk4(kind):
    """From a state past the initial transient (30 ms of ARS(2,2,2) at 20 us: the channel world
    starts at 0 V with its gates set near -60 mV, and NaV1.2's m relaxes in 0.2 ms there), 10 ms
    at dt = 1, 0.5, 0.25 ms against RK4 at 5 us: the error in the amounts and gates, relative to
    their change over the span, falls by at least 2^1.8 per halving."""
    b = worlds.pack([worlds.single_grid_tissue(0)]) if kind == "grid" else _channel_world()
    topo = T.topology(b)
    control = T.full_control(b)
    start = T.initial_state(b)
    for _ in range(1500):
        start, ok = T.ars222_step(start, 2e-5, control, b, topo)
        assert np.all(ok)

    def run(step, dt, n):
        st = start
        for _ in range(n):
            st, ok = step(st, dt, control, b, topo)
            assert np.all(ok)
        return st

    ref = run(T.rk4_step, 5e-6, int(round(SPAN / 5e-6)))
    fields = ["amount_increment"] + (["channel_gate"] if kind == "channels" else [])
    errors = []
    for dt in (1e-3, 5e-4, 2.5e-4):
        st = run(RO.ros2_step, dt, int(round(SPAN / dt)))
        errors.append(max(float(np.max(np.abs(getattr(st, f) - getattr(ref, f))))
                          / float(np.max(np.abs(getattr(ref, f) - getattr(start, f))))
                          for f in fields))
    orders = [np.log2(errors[i] / errors[i + 1]) for i in range(2)]
    assert all(p >= 1.8 for p in orders), (errors, orders)
    assert errors[-1] <= 1e-4, errors


def test_ros2_conserves_the_ledgers_every_step():
    """Uneven worlds with channels, gated junctions and partial controls, 100 steps of 1 ms: every
    ledger of oracle.tissue.balances within 1e-12 of its scale, every step."""
    rng = np.random.default_rng(9)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(16, k),
                                                     junction_sigma=0.3, gate=(0.02, 0.2, 0.9)),
                               rng, na=("nav", 1e-9, 0.5), k=("hh", 5e-10, 0.5), sigma=0.3)
          for k, n in enumerate((30, 75, 12))]
    b = worlds.pack(ws)
    topo = T.topology(b)
    control = T.Control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                        rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells)))
    st = T.initial_state(b)
    material = np.abs(b.amount_reference).sum()
    for _ in range(100):
        st, ok = RO.ros2_step(st, 1e-3, control, b, topo)
        assert np.all(ok)
        bal = T.balances(st, b, topo)
        for name in ("local", "outside", "total"):
            assert np.max(np.abs(bal[name])) <= 1e-12 * material, name
        # global charge against the charge the amounts carry (the cells start electroneutral)
        assert np.max(np.abs(bal["global_charge"])) <= 1e-12 * T.CHARGE_PER_FMOL * material


def test_ros2_steps_where_the_explicit_step_is_refused_as_stiff():
    """Leak permeabilities x100 (charge relaxation in about 2 ms) at dt = 5 ms: the explicit
    ARS(2,2,2) refuses; ROS2 (the slopes in W) steps, damps the fast charge mode (L-stable), and
    lands within 2% of an RK4 run at 10 us after 100 ms."""
    base = worlds.grid_world(4, 4, worlds.world_rng(13, 0))
    b = worlds.pack([dataclasses.replace(base, permeability=base.permeability * 100.0)])
    topo = T.topology(b)
    _, ok = T.ars222_step(T.initial_state(b), 5e-3, T.full_control(b), b, topo)
    assert not ok[0]
    st = _run(RO.ros2_step, b, 5e-3, 20)
    ref = _run(T.rk4_step, b, 1e-5, 10000)
    v, vr = T.membrane_voltage(st, b, topo), T.membrane_voltage(ref, b, topo)
    assert np.max(np.abs(v - vr)) <= 0.02 * np.max(np.abs(vr))


def test_ros2_refusal_keeps_the_state():
    b = worlds.pack([worlds.single_grid_tissue(0), worlds.single_grid_tissue(1)])
    topo = T.topology(b)
    control = T.full_control(b)
    membrane = control.membrane.copy()
    membrane[20] = 1.5  # world 1: an availability above 1
    start = T.initial_state(b)
    st, ok = RO.ros2_step(start, 1e-3, control._replace(membrane=membrane), b, topo)
    assert ok[0] and not ok[1]
    assert np.array_equal(st.amount_increment[:, 16:], start.amount_increment[:, 16:])
    assert not np.array_equal(st.amount_increment[:, :16], start.amount_increment[:, :16])


def test_fp32_factor_form_stays_within_1e8_of_fp64_and_conserves():
    """CB_METHOD_ROS2_MIXED's restatement (ros2_step(factor32=True): the voltage operator's factor
    and substitutions in FP32, no refinement): after 300 steps of 1 ms on uneven channel worlds
    with gated junctions and partial controls, every state field within 1e-8 scaled difference of
    the FP64 ROS2 (measured about 4e-10), and every ledger balanced to 1e-12 every step: the
    W-method's bookkeeping does not depend on W being exact."""
    from conftest import scaled_difference

    rng = np.random.default_rng(9)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(26, k),
                                                     junction_sigma=0.3, gate=(0.02, 0.2, 0.9)),
                               rng, na=("nav", 1e-9, 0.5), k=("hh", 5e-10, 0.5), sigma=0.3)
          for k, n in enumerate((60, 25))]
    b = worlds.pack(ws)
    topo = T.topology(b)
    control = T.Control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                        rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells)))
    a = m = T.initial_state(b)
    material = np.abs(b.amount_reference).sum()
    for _ in range(300):
        a, ok = RO.ros2_step(a, 1e-3, control, b, topo)
        assert np.all(ok)
        m, ok = RO.ros2_step(m, 1e-3, control, b, topo, factor32=True)
        assert np.all(ok)
        bal = T.balances(m, b, topo)
        for name in ("local", "outside", "total"):
            assert np.max(np.abs(bal[name])) <= 1e-12 * material, name
        assert np.max(np.abs(bal["global_charge"])) <= 1e-12 * T.CHARGE_PER_FMOL * material
    diffs = {f: scaled_difference(getattr(m, f), getattr(a, f)) for f in T.State._fields}
    assert max(diffs.values()) <= 1e-8, diffs
    assert max(diffs.values()) > 0.0  # the FP32 factor is in use


def test_fp32_factor_form_is_second_order_against_rk4():
    """The FP32-factor form keeps ROS2's order (the grid world of the order test above)."""
    b = worlds.pack([worlds.single_grid_tissue(0)])
    topo = T.topology(b)
    control = T.full_control(b)
    start = T.initial_state(b)
    for _ in range(1500):
        start, ok = T.ars222_step(start, 2e-5, control, b, topo)
    ref = start
    for _ in range(int(round(SPAN / 5e-6))):
        ref, _ = T.rk4_step(ref, 5e-6, control, b, topo)
    errors = []
    for dt in (1e-3, 5e-4, 2.5e-4):
        st = start
        for _ in range(int(round(SPAN / dt))):
            st, ok = RO.ros2_step(st, dt, control, b, topo, factor32=True)
            assert np.all(ok)
        errors.append(float(np.max(np.abs(st.amount_increment - ref.amount_increment)))
                      / float(np.max(np.abs(ref.amount_increment - start.amount_increment))))
    orders = [np.log2(errors[i] / errors[i + 1]) for i in range(2)]
    assert all(p >= 1.8 for p in orders), (errors, orders)


def test_tf32_rounded_factor_misses_the_bar_but_conserves():
    """Why the FP32-factor form stops at FP32: the same run with the factor rounded to TF32's
    10-bit mantissa (the tensor cores' FP32-class input format) stays conservative (ledgers to
    1e-12) and within 1e-6 of the FP64 step, but not within the 1e-8 bar (measured 1.0e-7 on the
    junction heat, 2.3e-8 on the amounts after 300 steps)."""
    import scipy.linalg as sl

    from conftest import scaled_difference

    def tf32(a):
        a = np.asarray(a, dtype=np.float32).copy()
        bits = a.view(np.int32)
        bits[:] = (bits + np.int32(0x1000)) & np.int32(-8192)  # round to 10 mantissa bits
        return a

    def voltage_rate_tf32(self, rho, b):
        u = np.zeros(b.cells)
        for wi, (_, scale, factor, free, _) in enumerate(self.operator.worlds):
            c0, c1 = b.cell_offset[wi], b.cell_offset[wi + 1]
            rhs = np.where(free, np.r_[rho[c0:c1], 0.0] * scale, 0.0)
            lower = tf32(factor)
            y = sl.solve_triangular(lower, rhs.astype(np.float32), lower=True)
            x = sl.solve_triangular(lower.T, y, lower=False).astype(np.float64)
            u[c0:c1] = np.where(free, x * scale, 0.0)[:-1]
        return u

    rng = np.random.default_rng(9)
    ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(26, k),
                                                     junction_sigma=0.3, gate=(0.02, 0.2, 0.9)),
                               rng, na=("nav", 1e-9, 0.5), k=("hh", 5e-10, 0.5), sigma=0.3)
          for k, n in enumerate((60, 25))]
    b = worlds.pack(ws)
    topo = T.topology(b)
    control = T.Control(rng.uniform(0.6, 1, b.cells), rng.uniform(0.6, 1, b.edges),
                        rng.uniform(0.6, 1, b.cells), rng.uniform(0.4, 1, (2, b.cells)))
    a = m = T.initial_state(b)
    for _ in range(300):
        a, _ = RO.ros2_step(a, 1e-3, control, b, topo)
    saved = RO.Jacobian.voltage_rate
    RO.Jacobian.voltage_rate = voltage_rate_tf32
    try:
        for _ in range(300):
            m, ok = RO.ros2_step(m, 1e-3, control, b, topo)
            assert np.all(ok)
    finally:
        RO.Jacobian.voltage_rate = saved
    worst = max(scaled_difference(getattr(m, f), getattr(a, f)) for f in T.State._fields)
    assert 1e-8 < worst < 1e-6, worst
    bal = T.balances(m, b, topo)
    material = np.abs(b.amount_reference).sum()
    for name in ("local", "outside", "total"):
        assert np.max(np.abs(bal[name])) <= 1e-12 * material, name
