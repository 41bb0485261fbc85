"""ctypes binding of libcellsb200.so (the C ABI declared in include/cells_b200.h).

The library is built in-tree by ``cells_b200.build`` (nvcc, sm_100a) and loaded from this
package directory only. There is no fallback: a missing or unloadable library raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libcellsb200.so")

# include/cells_b200.h
CB_OK = 0
STATE_FIELDS = (
    "amount_increment",
    "membrane_transferred",
    "membrane_dissipated",
    "pump_cycles",
    "pump_dissipated",
    "metabolic_work",
    "junction_transferred",
    "junction_dissipated",
    "junction_gate",
    "reservoir_supplied",
    "electrode_charge",
    "reservoir_work",
    "electrode_work",
    "channel_gate",
    "channel_transferred",
    "channel_dissipated",
)
CONTROL_FIELDS = ("membrane", "junction", "pump", "channel")
METHOD_ARS222 = 0
METHOD_ARS222_MIXED = 1
METHOD_N2 = 2
METHOD_N2_MIXED = 3
METHOD_ROS2 = 4
METHOD_RK4 = 5
METHOD_ROS2_MIXED = 6
KERNEL_SHARED, KERNEL_PACKED = 0, 1
WORLD_BITS = {
    1: "transport",
    2: "pump_domain",
    4: "gate_domain",
    8: "control",
    16: "residual",
    32: "domain",
    64: "stiff",
    128: "channel_domain",
    256: "ledger_cotangent",
    512: "operator",
    1024: "field",
}
# Field worlds (cb_field_*): state fields in CB_FIELD_* order.
FIELD_STATE_FIELDS = (
    "amount_increment", "extracellular_increment", "membrane_transferred",
    "junction_transferred", "face_transferred", "reservoir_supplied", "membrane_dissipated",
    "junction_dissipated", "face_dissipated", "electrode_charge", "reservoir_work",
    "electrode_work", "junction_gate", "pump_cycles", "pump_dissipated", "metabolic_work",
)
EXPORTS = (
    "cb_bind",
    "cb_free",
    "cb_state_layout",
    "cb_control_layout",
    "cb_step",
    "cb_step_host",
    "cb_step_packed_static",
    "cb_set_launch",
    "cb_get_launch",
    "cb_balances",
    "cb_step_vjp",
    "cb_vjp_workspace",
    "cb_step_vjp_method",
    "cb_vjp_workspace_method",
    "cb_set_sparse_launch",
    "cb_get_sparse_launch",
    "cb_set_permeability",
    "cb_set_channel_block",
    "cb_device_checks",
    "cb_device_checks_each",
    "cb_copy_worlds",
    "cb_window_row",
    "cb_store_worlds",
    "cb_field_bind",
    "cb_field_free",
    "cb_field_state_layout",
    "cb_field_control_length",
    "cb_field_info",
    "cb_field_launches",
    "cb_field_levels",
    "cb_field_counts",
    "cb_field_flops",
    "cb_field_step",
    "cb_field_step_host",
    "cb_probe_fp64",
    "cb_last_error",
    "cb_version",
)

_p = ctypes.c_void_p
_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_i32 = ctypes.POINTER(ctypes.c_int32)


class TissueDesc(ctypes.Structure):
    """cb_tissue_desc (include/cells_b200.h)."""

    _fields_ = [
        ("n_worlds", ctypes.c_int32),
        ("n_cells", ctypes.c_int64),
        ("n_edges", ctypes.c_int64),
        ("cell_offset", _i64),
        ("edge_offset", _i64),
        ("temperature", _d),
        ("bath_amount", _d),
        ("bath_volume", _d),
        ("bath_potential", _d),
        ("pump", _d),
        ("volume", _d),
        ("area", _d),
        ("capacitance", _d),
        ("permeability", _d),
        ("pump_capacity", _d),
        ("amount_reference", _d),
        ("initial_charge", _d),
        ("sender", _i32),
        ("receiver", _i32),
        ("junction_area", _d),
        ("junction_permeability", _d),
        ("gate_threshold", _d),
        ("gate_minimum", _d),
        ("channel_slots", ctypes.c_int32),
        ("channel_code", _i32),
        ("channel_species", _i32),
        ("channel_permeability", _d),
        ("channel_abundance", _d),
    ]


class FieldDesc(ctypes.Structure):
    """cb_field_desc (include/cells_b200.h)."""

    _fields_ = [
        ("worlds", ctypes.c_int32),
        ("cells", ctypes.c_int32),
        ("nodes", ctypes.c_int32),
        ("junctions", ctypes.c_int32),
        ("faces", ctypes.c_int32),
        ("cell_node", _i64),
        ("junction_sender", _i64),
        ("junction_receiver", _i64),
        ("face_sender", _i64),
        ("face_receiver", _i64),
        ("reservoir", ctypes.POINTER(ctypes.c_uint8)),
        ("temperature", _d),
        ("pump", _d),
        ("volume", _d),
        ("area", _d),
        ("capacitance", _d),
        ("permeability", _d),
        ("pump_capacity", _d),
        ("amount", _d),
        ("initial_charge", _d),
        ("junction_area", _d),
        ("junction_permeability", _d),
        ("gate_threshold", _d),
        ("gate_minimum", _d),
        ("outside_volume", _d),
        ("outside_amount", _d),
        ("outside_charge", _d),
        ("boundary_V", _d),
        ("face_factor", _d),
    ]


class LibraryMissing(RuntimeError):
    """The CUDA library is not built or cannot be loaded; nothing runs without it."""


_lib = None


def load(path=LIBRARY):
    """Load (once) and type the library. Raises LibraryMissing if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise LibraryMissing(
            f"{path} is not built; run `python -m cells_b200.build` (nvcc, sm_100a)"
        )
    try:
        lib = ctypes.CDLL(path)
    except OSError as error:
        raise LibraryMissing(f"cannot load {path}: {error}") from error
    lib.cb_bind.argtypes = [ctypes.POINTER(TissueDesc), ctypes.c_int, ctypes.POINTER(_p)]
    lib.cb_bind.restype = ctypes.c_int
    lib.cb_free.argtypes = [_p]
    lib.cb_free.restype = None
    lib.cb_state_layout.argtypes = [_p, _i64, _i64]
    lib.cb_state_layout.restype = ctypes.c_int
    lib.cb_control_layout.argtypes = [_p, _i64, _i64]
    lib.cb_control_layout.restype = ctypes.c_int
    lib.cb_step.argtypes = [_p, ctypes.c_int, _p, _p, ctypes.c_double, _p, ctypes.c_int, _p, _p,
                            _p]
    lib.cb_step.restype = ctypes.c_int
    lib.cb_step_host.argtypes = [_p, ctypes.c_int, _p, _p, ctypes.c_double, _p, ctypes.c_int,
                                 _p, _p]
    lib.cb_step_host.restype = ctypes.c_int
    lib.cb_step_packed_static.argtypes = [_p, _p, _p, ctypes.c_double, _p, ctypes.c_int, _p,
                                          _p, _p]
    lib.cb_step_packed_static.restype = ctypes.c_int
    lib.cb_set_launch.argtypes = [_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.cb_set_launch.restype = ctypes.c_int
    _ip = ctypes.POINTER(ctypes.c_int)
    lib.cb_get_launch.argtypes = [_p, _ip, _ip, _ip]
    lib.cb_get_launch.restype = ctypes.c_int
    lib.cb_balances.argtypes = [_p, _p, _p, _p]
    lib.cb_balances.restype = ctypes.c_int
    lib.cb_step_vjp.argtypes = [_p, _p, ctypes.c_double, _p, ctypes.c_int, _p, _p, _p, _p, _p,
                                _p, ctypes.c_size_t, _p, _p]
    lib.cb_step_vjp.restype = ctypes.c_int
    lib.cb_vjp_workspace.argtypes = [_p, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
    lib.cb_vjp_workspace.restype = ctypes.c_int
    lib.cb_step_vjp_method.argtypes = [_p, ctypes.c_int, _p, ctypes.c_double, _p, ctypes.c_int,
                                       _p, _p, _p, _p, _p, _p, ctypes.c_size_t, _p, _p]
    lib.cb_step_vjp_method.restype = ctypes.c_int
    lib.cb_vjp_workspace_method.argtypes = [_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_size_t)]
    lib.cb_vjp_workspace_method.restype = ctypes.c_int
    lib.cb_set_sparse_launch.argtypes = [_p, ctypes.c_int]
    lib.cb_set_sparse_launch.restype = ctypes.c_int
    lib.cb_get_sparse_launch.argtypes = [_p, ctypes.POINTER(ctypes.c_int)]
    lib.cb_get_sparse_launch.restype = ctypes.c_int
    lib.cb_set_permeability.argtypes = [_p, _p, _p, _p, _p]
    lib.cb_set_permeability.restype = ctypes.c_int
    lib.cb_set_channel_block.argtypes = [_p, ctypes.c_int32, _d, _d, _d, _d]
    lib.cb_set_channel_block.restype = ctypes.c_int
    lib.cb_device_checks.argtypes = [_p, _p, _p, ctypes.c_int64, _d, ctypes.c_double, _p, _p, _p]
    lib.cb_device_checks.restype = ctypes.c_int
    lib.cb_device_checks_each.argtypes = [_p, _p, _p, _p, _d, ctypes.c_double, _p, _p, _p]
    lib.cb_device_checks_each.restype = ctypes.c_int
    lib.cb_copy_worlds.argtypes = [_p, _p, _p, _p, _p]
    lib.cb_copy_worlds.restype = ctypes.c_int
    lib.cb_window_row.argtypes = [_p, _p, _p, ctypes.c_int32, _p, ctypes.c_int64, _d,
                                  ctypes.c_double, _p, _p, _p, _p, _p, _p, _p, _p]
    lib.cb_window_row.restype = ctypes.c_int
    lib.cb_store_worlds.argtypes = [_p, _p, _p, _p, _p, ctypes.c_int32, _p]
    lib.cb_store_worlds.restype = ctypes.c_int
    lib.cb_field_bind.argtypes = [ctypes.POINTER(FieldDesc), ctypes.c_int, ctypes.POINTER(_p)]
    lib.cb_field_bind.restype = ctypes.c_int
    lib.cb_field_free.argtypes = [_p]
    lib.cb_field_free.restype = None
    lib.cb_field_state_layout.argtypes = [_p, _i64, _i64]
    lib.cb_field_state_layout.restype = ctypes.c_int
    lib.cb_field_launches.argtypes = [_p]
    lib.cb_field_launches.restype = ctypes.c_int64
    lib.cb_field_counts.argtypes = [_p, _i64]
    lib.cb_field_counts.restype = ctypes.c_int
    lib.cb_field_flops.argtypes = [_p, _d]
    lib.cb_field_flops.restype = ctypes.c_int
    lib.cb_field_levels.argtypes = [_p, _i32, ctypes.c_int32]
    lib.cb_field_levels.restype = ctypes.c_int32
    lib.cb_field_info.argtypes = [_p, _i64]
    lib.cb_field_info.restype = ctypes.c_int
    lib.cb_field_control_length.argtypes = [_p]
    lib.cb_field_control_length.restype = ctypes.c_int64
    lib.cb_field_step.argtypes = [_p, _p, _p, ctypes.c_double, _p, ctypes.c_int, _p, _p, _p]
    lib.cb_field_step.restype = ctypes.c_int
    lib.cb_field_step_host.argtypes = [_p, _d, _d, ctypes.c_double, _d, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_uint32), _i32]
    lib.cb_field_step_host.restype = ctypes.c_int
    lib.cb_probe_fp64.argtypes = [ctypes.c_int, ctypes.c_int64, _d, _d]
    lib.cb_probe_fp64.restype = ctypes.c_int
    lib.cb_last_error.argtypes = []
    lib.cb_last_error.restype = ctypes.c_char_p
    lib.cb_version.argtypes = []
    lib.cb_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(code):
    if code != CB_OK:
        message = _lib.cb_last_error().decode() if _lib is not None else "library not loaded"
        raise RuntimeError(f"cells_b200 error {code}: {message}")
