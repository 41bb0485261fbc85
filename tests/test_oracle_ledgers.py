"""Ledger conservation of the oracle's step on the benchmark tissues (surface_tissue.balances):
moles per ion, charge and work ledgers hold to 1e-12 relative every step."""

import numpy as np

from cells_b200 import worlds
from oracle import tissue as T


def _relative(b, st):
    res = T.balances(st, b)
    scale_amount = np.max(np.abs(b.amount_reference))
    out = {k: float(np.max(np.abs(v))) for k, v in res.items()}
    out["local"] /= scale_amount
    out["outside"] /= scale_amount
    out["total"] /= scale_amount
    moved = np.max(np.abs(st.electrode_charge), initial=1e-30)
    out["electrode"] /= moved
    out["global_charge"] /= max(moved, 1e-30)
    for k in ("reservoir_work", "electrode_work", "metabolic_work"):
        out[k] /= max(np.max(np.abs(getattr(st, k))), 1e-30)
    return out


def test_ledgers_hold_every_step_single_world():
    b = worlds.pack([worlds.single_grid_tissue(0)])
    topo = T.topology(b)
    st = T.initial_state(b)
    ctl = T.full_control(b)
    for _ in range(300):
        st, ok = T.ars222_step(st, 1e-3, ctl, b, topo)
        assert ok.all()
        rel = _relative(b, st)
        assert all(v <= 1e-12 for v in rel.values()), rel


def test_rk4_and_ars222_converge_to_the_same_trajectory():
    """Observed order of ARS(2,2,2) against an RK4 run at a small step (the reference's order
    study, tests/unit/test_surface_pump_v3_imex.py:138)."""
    b = worlds.pack([worlds.single_grid_tissue(0)])
    topo = T.topology(b)
    ctl = T.full_control(b)
    ref = T.initial_state(b)
    for _ in range(400):
        ref, _ = T.rk4_step(ref, 0.5e-4, ctl, b, topo)
    errs = []
    for dt, n in ((4e-3, 5), (2e-3, 10), (1e-3, 20)):
        st = T.initial_state(b)
        for _ in range(n):
            st, _ = T.ars222_step(st, dt, ctl, b, topo)
        errs.append(np.max(np.abs(st.amount_increment - ref.amount_increment)))
    order = np.log2(errs[0] / errs[1]), np.log2(errs[1] / errs[2])
    assert min(order) > 1.7, (errs, order)
