"""The reference's own pytrees rebuilt from a golden fixture (tests/golden/make_golden.py),
as NamedTuples with the reference's field names."""

from collections import namedtuple

import numpy as np

from conftest import GOLDEN


def load_pytrees(name="pytrees_gated_padded.npz"):
    z = np.load(f"{GOLDEN}/{name}")
    layout_fields = [k[len("layout_"):] for k in z.files if k.startswith("layout_")]
    Layout = namedtuple("ReferenceLayout", layout_fields)
    p = Layout(*(z["layout_" + f] for f in layout_fields))
    control_fields = [k[len("control_ref_"):] for k in z.files if k.startswith("control_ref_")]
    Control = namedtuple("ReferenceControl", control_fields)
    control = Control(*(z["control_ref_" + f] for f in control_fields))
    state_fields = [str(f) for f in z["state_fields"]]
    State = namedtuple("ReferenceState", state_fields)
    states = [State(*(z["refstate_" + f][k] for f in state_fields)) for k in range(len(z["steps"]))]
    return z, p, control, states
