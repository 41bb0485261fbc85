"""The mixed-precision ARS(2,2,2) step (CB_METHOD_ARS222_MIXED: FP32 rates on FP64 differences,
FP64 near-zero GHK series and FP64 accumulation) against the FP64 device step.

Per-output errors are printed (pytest -s shows them) and bounded: state amounts within 1e-8 of
the FP64 amounts (relative to the cells' physical amounts), every field's scaled difference
within 1e-5, and the conservation ledgers within 1e-12 relative, every launch, as the FP64 step.
"""

import numpy as np
import pytest

from cells_b200 import _lib, worlds
from cells_b200.tissue import Tissue
from conftest import scaled_difference

pytestmark = pytest.mark.gpu


def _run(torch, tissue, method, steps, chunks):
    dev = torch.device("cuda")
    state = torch.from_numpy(tissue.pack_state(tissue.initial_state())).to(dev)
    ctl = torch.from_numpy(tissue.pack_control()).to(dev)
    status = torch.zeros(tissue.batch.worlds, dtype=torch.int32, device=dev)
    out = torch.zeros(tissue.batch.worlds * 8, dtype=torch.float64, device=dev)
    worst = np.zeros(8)
    for _ in range(chunks):
        tissue.step(state, state, ctl, 1e-3, steps, status, method=method)
        tissue.balances(state, out)
        worst = np.maximum(worst, out.view(-1, 8).max(dim=0).values.cpu().numpy())
    torch.cuda.synchronize()
    assert int(status.abs().max()) == 0
    return tissue.unpack_state(state.cpu().numpy()), worst


@pytest.mark.parametrize("kind", ["grid", "channels", "packed"])
def test_mixed_step_error_against_fp64(cuda, kind):
    """grid and channels on the one-world-per-CTA kernel; packed: uneven Delaunay worlds of
    40-2500 cells with NaV1.2 + HH K on the packed kernel (both methods)."""
    rng = np.random.default_rng(3)
    if kind == "grid":
        ws = worlds.grid_tissues(64, side=16, seed=12)
    elif kind == "packed":
        ws = [worlds.with_channels(worlds.delaunay_world(n, worlds.world_rng(14, k),
                                                         junction_sigma=0.3,
                                                         gate=(0.02, 0.2, 0.9)), rng,
                                   na=("nav", 1e-9, 0.5), k=("hh", 5e-10, 0.5), sigma=0.3)
              for k, n in enumerate((2500, 1100, 700, 333, 150, 90, 40))]
    else:
        ws = [worlds.with_channels(worlds.delaunay_world(200, worlds.world_rng(13, k),
                                                         junction_sigma=0.3), rng,
                                   na=("nav", 3e-10, 0.5), k=("hh", 6e-10, 0.5), sigma=0.3)
              for k in range(16)]
    b = worlds.pack(ws)
    tissue = Tissue(b)
    if kind == "packed":
        assert tissue.get_launch()[0] == _lib.KERNEL_PACKED
    ref, _ = _run(cuda, tissue, _lib.METHOD_ARS222, 100, 5)
    got, ledgers = _run(cuda, tissue, _lib.METHOD_ARS222_MIXED, 100, 5)
    amounts = np.abs(b.amount_reference + ref["amount_increment"])
    amount_err = float(np.max(np.abs(got["amount_increment"] - ref["amount_increment"]) / amounts))
    errors = {f: scaled_difference(got[f], ref[f]) for f in ref if ref[f].size}
    print(f"\nmixed vs fp64 ({kind}, 500 steps): amounts {amount_err:.2e}; " +
          ", ".join(f"{f} {v:.1e}" for f, v in errors.items()))
    assert amount_err <= 1e-8
    assert max(errors.values()) <= 1e-5
    scale = float(np.max(np.abs(b.amount_reference)))
    assert ledgers[0] <= 1e-12 * scale  # local material balance per cell
