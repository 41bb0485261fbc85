"""The oracle's window (tests/test_windows_gpu.py: oracle_window_each, the reference's vector
window restated over oracle/tissue.py's step and oracle/checks.py's row checks) against the
reference's own _vector_window (execution/vector_windows.py:348-410, run by
tests/golden/make_golden.py over @3's checked_step and device_checks; vector_window.npz) on the
same three gated worlds and per-world row tables: first failing rows, bits and the final states
equal, the energy diagnostics' maxima to 1e-8 (they are small nets of rounded ledgers).
"""

import numpy as np

from conftest import load_golden, scaled_difference
from oracle import tissue as T
from test_windows_gpu import ATOL, RTOL, batch, oracle_window_each


def test_oracle_window_matches_the_reference_window():
    z, b = load_golden("vector_window.npz")
    assert np.array_equal(z["material_atol"], ATOL) and float(z["energy_rtol"]) == RTOL
    b2, controls = batch()
    assert np.array_equal(b2.amount_reference, b.amount_reference)
    cur, first, bits, maxima, stored = oracle_window_each(b2, controls)
    assert np.array_equal(first, z["first"]) and np.array_equal(bits, z["bits"])
    topo = T.topology(b2)
    for w in range(b2.worlds):
        cells, edges = topo.cell_world == w, topo.edge_world == w
        for f in ("amount_increment", "membrane_transferred", "pump_cycles", "metabolic_work"):
            assert scaled_difference(getattr(cur, f)[..., cells], z[f"final{w}_{f}"]) <= 1e-14
        for f in ("junction_transferred", "junction_gate"):
            assert scaled_difference(getattr(cur, f)[..., edges], z[f"final{w}_{f}"]) <= 1e-14
        for (slot, ww), ref in stored.items():
            if ww != w:
                continue
            got = z[f"stored{w}_{slot}_amount_increment"]
            assert scaled_difference(ref["amount_increment"][:, cells], got) <= 1e-14
    ref = z["maxima"]
    for k in (6, 10):
        assert np.all(np.abs(maxima[:, k] - ref[:, k]) <= 1e-8 * np.abs(ref[:, k])), k
