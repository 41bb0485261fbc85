"""Shared fixtures. ``-m gpu`` tests need a CUDA device and the in-tree library; everything
else runs on the CPU. Golden fixtures come from tests/golden/make_golden.py (the reference's own
step, run where its source is present)."""

import os
import sys
from dataclasses import fields

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libcellsb200.so")


def load_golden(name):
    """(npz, Batch) of one golden fixture."""
    from cells_b200 import worlds

    z = np.load(os.path.join(GOLDEN, name))
    batch = worlds.Batch(**{f.name: z["batch_" + f.name] for f in fields(worlds.Batch)
                            if "batch_" + f.name in z.files})
    if "block_weight" in z.files:
        batch.channel_block = worlds.ChannelBlock(
            **{f.name: z["block_" + f.name] for f in fields(worlds.ChannelBlock)})
    return z, batch


def load_field_golden(name):
    """(npz, FieldWorld) of one field fixture (tests/golden/make_golden.py, field_*.npz)."""
    from cells_b200 import field_worlds

    z = np.load(os.path.join(GOLDEN, name))
    values = {}
    for f in fields(field_worlds.FieldWorld):
        v = z["fw_" + f.name]
        if f.name in ("side", "cells_side", "stride"):
            v = int(v)
        elif f.name in ("face_area", "face_length", "temperature"):
            v = float(v)
        elif f.name == "pump":
            v = tuple(float(x) for x in v)
        values[f.name] = v
    return z, field_worlds.FieldWorld(**values)


def scaled_difference(a, b):
    """max |a - b| / max(|a|, |b|) over a field: the reference's own trajectory comparison
    (tests/unit/test_surface_pump_v3_imex.py:45-48)."""
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = max(np.max(np.abs(a), initial=0), np.max(np.abs(b), initial=0))
    return 0.0 if scale == 0 else float(np.max(np.abs(a - b)) / scale)


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; skips only when no device exists (a missing library fails)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cells_b200 import _lib

    _lib.load()  # LibraryMissing fails the test: there is no fallback.
    return torch
