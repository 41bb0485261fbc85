"""The mixed-precision ARS(2,2,2) step (CB_METHOD_ARS222_MIXED: FP32 constant-field fluxes on
FP64 concentration differences; everything else, the near-zero GHK series and every accumulation
in FP64) against the FP64 device step.

Per-output errors are printed (pytest -s shows them) and bounded, in four classes:
* the amounts within 1e-8 of the cells' physical amounts (measured about 1e-11);
* conservation: the ledgers balance within 1e-12 relative, every launch, as the FP64 step;
* the gates within 1e-7 scaled (measured 5e-8 for channel gates, 0 for junction gates): their
  laws run in FP64, but they follow the membrane voltage, a small net charge over C, which
  carries the amount increments' FP32-flux rounding;
* the ledgers that integrate a flux (amount increments over the reference, membrane, junction
  and channel transfers and heats; the pump's ledgers, in FP64, only through the voltage) carry
  the FP32 flux's rounding: within 5e-7 scaled difference (measured about 1e-7).
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
    gates = {f: errors[f] for f in ("junction_gate", "channel_gate") if f in errors}
    assert all(v <= 1e-7 for v in gates.values()), gates
    assert max(errors.values()) <= 5e-7, errors
    scale = float(np.max(np.abs(b.amount_reference)))
    assert ledgers[0] <= 1e-12 * scale  # local material balance per cell
