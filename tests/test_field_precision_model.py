"""What a lower-precision factor of the 128x128 field's stage operator costs in solves.

The precision form the field step would take factors the stage operator (capacitor + gamma dt
L(W), Jacobi-scaled, numerics/surface_imex.py:207-225) in FP32 or TF32 and wins the accuracy back
by FP64 iterative refinement of the charge residual up to solve_operator's acceptance
(|r| <= 3e-25 + 2e-12 max(|q|, |M phi|), numerics/surface_imex.py:269-278). These tests measure,
on one benchmark world (1024 cells in a 128x128 grid with its held ring, face conductivity
log-normal sigma 0.5), how many solves that takes:

* the operator's condition number after Jacobi scaling is about 7e3;
* an FP32 factor's first solve misses the acceptance by about 1e5 and one refinement meets it:
  every stage solve becomes two solves and a residual;
* a factor of the operator rounded to TF32 (the tensor cores' FP32-input format, 10 mantissa
  bits) gains only about two digits per refinement: five or more refinement solves per stage
  solve to reach the FP64 solution to 1e-10.

The factors here are SuperLU's (no pivoting, symmetric mode) standing in for the device's
supernodal Cholesky: the rounding class is the same.
"""

import numpy as np
import pytest

sp = pytest.importorskip("scipy.sparse")
from scipy.sparse.linalg import eigsh, splu  # noqa: E402

from cells_b200 import field_worlds as FW  # noqa: E402
from oracle import field as OF  # noqa: E402
from oracle import tissue as T  # noqa: E402

ATOL, RTOL = 3e-25, 2e-12


@pytest.fixture(scope="module")
def operator():
    w = FW.field_tissues(1)[0]
    tp = OF.bind(w)
    st = OF.initial_state(w)
    co = (w.outside_amount + st.extracellular_increment) / w.outside_volume
    weight, _ = OF.face_weights(co, w)
    matrix = (tp.capacitor + T.GAMMA * 5e-4 * OF.face_laplacian(weight, w, tp)).tocsr()
    free = tp.free
    scale = 1.0 / np.sqrt(np.where(free, matrix.diagonal(), 1.0))
    keep = sp.diags(free.astype(float) * scale)
    reduced = (keep @ matrix @ keep + sp.diags((~free).astype(float))).tocsc()
    rng = np.random.default_rng(1)
    qc, qo = OF.node_charge(st, w)
    charge = np.concatenate((qc, qo)) + 1e-15 * rng.standard_normal(qc.size + qo.size)
    return matrix, reduced, free, scale, charge


def _lu(a):
    return splu(a, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0,
                options=dict(SymmetricMode=True))


def _tf32(values):
    bits = np.asarray(values, dtype=np.float32).view(np.uint32)
    return ((bits + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def _refine(factor, reduced, rhs, exact, accept, target):
    """Solves until accept(x) and the error is below target; returns the solves taken."""
    x = factor.solve(rhs.astype(np.float32)).astype(np.float64)
    for solves in range(1, 16):
        if accept(x) and np.max(np.abs(x - exact)) <= target * np.max(np.abs(exact)):
            return solves
        x = x + factor.solve((rhs - reduced @ x).astype(np.float32)).astype(np.float64)
    return 16


def test_condition_number(operator):
    _, reduced, *_ = operator
    top = eigsh(reduced, k=1, which="LA", return_eigenvectors=False)[0]
    bottom = eigsh(reduced, k=1, sigma=0, which="LM", return_eigenvectors=False)[0]
    assert 1e3 <= top / bottom <= 1e5


def test_fp32_factor_needs_one_refinement(operator):
    matrix, reduced, free, scale, charge = operator
    rhs = np.where(free, charge * scale, 0.0)
    exact = _lu(reduced).solve(rhs)

    def accept(x):
        phi = np.where(free, x * scale, 0.0)
        lphi = matrix @ phi
        r = np.where(free, lphi - charge, 0.0)
        return bool(np.all(np.abs(r) <= ATOL + RTOL * np.maximum(np.abs(charge), np.abs(lphi))))

    assert accept(exact)
    f32 = _lu(reduced.astype(np.float32))
    assert not accept(f32.solve(rhs.astype(np.float32)).astype(np.float64))
    assert _refine(f32, reduced, rhs, exact, accept, 1e-10) == 2


def test_tf32_operator_needs_many_refinements(operator):
    _, reduced, free, scale, charge = operator
    rhs = np.where(free, charge * scale, 0.0)
    exact = _lu(reduced).solve(rhs)
    rounded = reduced.astype(np.float32).tocsc()
    rounded.data = _tf32(rounded.data)
    assert _refine(_lu(rounded), reduced, rhs, exact, lambda x: True, 1e-10) >= 6
