"""The C-ABI library: it builds, loads without a GPU, and exports every entry point that
include/cells_b200.h declares; the ctypes description matches the header's struct."""

import os
import re
import subprocess

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cells_b200.h")


def _declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(cb_\w+)\s*\(", text, re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    from cells_b200 import _lib

    lib = _lib.load()
    declared = _declared_functions()
    assert declared, "no cb_ functions found in the header"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIBRARY], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (cb_\w+)", out))
    assert set(declared) <= exported
    assert lib.cb_version().decode().startswith("cells_b200")


def test_descriptor_matches_header_struct():
    from cells_b200 import _lib

    text = open(HEADER).read()
    body = text[text.index("typedef struct cb_tissue_desc {"):text.index("} cb_tissue_desc;")]
    names = re.findall(r"\*?\s*(\w+);", body)
    assert names == [f for f, _ in _lib.TissueDesc._fields_]


def test_state_field_order_matches_header_enum():
    from cells_b200 import _lib

    text = open(HEADER).read()
    body = text[text.index("enum cb_state_field {"):text.index("CB_STATE_FIELDS\n")]
    names = [n.lower() for n in re.findall(r"CB_(\w+)\s*(?:=\s*0)?,", body)]
    assert names == list(_lib.STATE_FIELDS)


def test_library_refuses_bad_layouts_without_a_gpu():
    """Layout refusals happen on the host before any device call (cb_bind returns
    CB_ERR_LAYOUT), so they run here."""
    import ctypes

    import numpy as np

    from cells_b200 import _lib, worlds

    lib = _lib.load()
    b = worlds.pack([worlds.single_grid_tissue(0)])
    b.sender = b.sender.copy()
    b.sender[0] = 99  # out of its world
    from cells_b200.tissue import Tissue

    try:
        Tissue(b)
    except RuntimeError as error:
        assert "error 2" in str(error) and "endpoint" in str(error)
    else:
        raise AssertionError("bad junction endpoint was accepted")
    assert lib.cb_bind(None, 0, ctypes.byref(ctypes.c_void_p())) == 1
    assert np.isfinite(0.0)
