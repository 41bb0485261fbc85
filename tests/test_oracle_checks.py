"""The accepted-row checks oracle (oracle/checks.py) against the reference's own device checks
(@3's device_checks, run by tests/golden/make_golden.py on rows of its trajectory): every
failed bit equal, on accepted rows and on rows with planted faults (a material error, a heat
that decreases); the physical diagnostics (the energy residual and its ratio to the flows) to
1e-8 relative. The other diagnostics are rounding residuals (1e-30 C, 1e-20 fmol) whose bits
depend on summation order; they are checked against their bounds through the failed bits."""

import numpy as np

from conftest import load_golden
from oracle import checks as CK
from oracle import tissue as T


def case_states(z, b, i):
    init = T.initial_state(b)

    def state(tag):
        return T.State(**{f: z[f"case{i}_{tag}_{f}"] if f"case{i}_{tag}_{f}" in z.files
                          else getattr(init, f) for f in T.State._fields})

    return state("prev"), state("row")


def test_checks_match_the_reference():
    z, b = load_golden("device_checks.npz")
    assert tuple(z["checks"]) == CK.CHECKS
    topo = T.topology(b)
    labels = []
    for i in range(int(z["cases"])):
        prev, row = case_states(z, b, i)
        failed, values = CK.row_checks(prev, row, b, topo, int(z[f"case{i}_steps"]),
                                       z["material_atol"], float(z["energy_rtol"]))
        ref_failed, ref_values = z[f"case{i}_failed"], z[f"case{i}_values"]
        assert np.array_equal(failed[0], ref_failed), (i, failed[0], ref_failed)
        for k in (6, 10):  # energy residual, energy relative
            assert abs(values[0, k] - ref_values[k]) <= 1e-8 * abs(ref_values[k]), (i, k)
        labels.append((str(z[f"case{i}_label"]), bool(failed[0].any())))
    assert ("material", True) in labels and ("dissipation", True) in labels
    assert all(not bad for label, bad in labels if label == "accepted")
