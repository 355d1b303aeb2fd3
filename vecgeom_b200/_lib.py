"""ctypes binding of libvgb.so, the C-ABI library declared in include/vgb.h.

The library is built in-tree (vecgeom_b200/lib/libvgb.so) by
``make -C vecgeom_b200/csrc``.  Loading fails loudly when it is missing: there
is no CPU fallback for any operation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libvgb.so")

# vgb_status (include/vgb.h)
OK, EINVAL, ENOMEM, ECUDA, ELOOPCAP, ETIMEDOUT, ENOTSUP, ENOSPC = range(8)
STATUS_NAMES = {0: "VGB_OK", 1: "VGB_EINVAL", 2: "VGB_ENOMEM", 3: "VGB_ECUDA",
                4: "VGB_ELOOPCAP", 5: "VGB_ETIMEDOUT", 6: "VGB_ENOTSUP", 7: "VGB_ENOSPC"}

# vgb_op
OP_CONTAINS = 0
OP_INSIDE = 1
OP_DISTANCE_TO_IN = 2
OP_DISTANCE_TO_OUT = 3
OP_SAFETY_TO_IN = 4
OP_SAFETY_TO_OUT = 5
OP_DISTANCE_TO_IN_MINIMIZE = 6
OP_SAFETY_TO_IN_MINIMIZE = 7
OP_SAFETY_TO_OUT_MINIMIZE = 8
OP_DISTANCE_TO_OUT_NODE = 9
OP_PLACED_DISTANCE_TO_OUT = 10

PREC_FP64 = 0
PREC_FP32_REFINE = 1

FUSED_DTO_INSIDE_ONLY = 1
FUSED_LOCAL_INSIDE_ONLY = 2


class VgbError(RuntimeError):
    """A vgb_status other than VGB_OK, with vgb_last_error()'s message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

# (name, restype, argtypes)
_i32, _i64, _u32, _dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32, ctypes.c_double
_vp, _cp = ctypes.c_void_p, ctypes.c_char_p
_pi32, _pi64 = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64)

SIGNATURES = {
    "vgb_last_error": (_cp, []),
    "vgb_version": (_cp, []),
    "vgb_launch_count": (_i64, []),
    "vgb_launch_count_reset": (None, []),
    "vgb_measure_fma_peak": (ctypes.c_int, [_i32, _i32, _vp, ctypes.POINTER(_dbl),
                                            ctypes.POINTER(ctypes.c_float)]),
    "vgb_refine_counts": (ctypes.c_int, [_pi64, _pi64, _i32]),
    "vgb_geometry_create": (ctypes.c_int, [ctypes.POINTER(_vp)]),
    "vgb_geometry_destroy": (ctypes.c_int, [_vp]),
    "vgb_unplaced_box": (ctypes.c_int, [_vp, _dbl, _dbl, _dbl, _pi32]),
    "vgb_unplaced_tube": (ctypes.c_int, [_vp, _dbl, _dbl, _dbl, _dbl, _dbl, _pi32]),
    "vgb_unplaced_cone": (ctypes.c_int, [_vp] + [_dbl] * 7 + [_pi32]),
    "vgb_unplaced_sphere": (ctypes.c_int, [_vp] + [_dbl] * 6 + [_pi32]),
    "vgb_unplaced_torus": (ctypes.c_int, [_vp] + [_dbl] * 5 + [_pi32]),
    "vgb_unplaced_polycone": (ctypes.c_int, [_vp, _dbl, _dbl, _i32, _vp, _vp, _vp, _pi32]),
    "vgb_unplaced_polyhedron": (ctypes.c_int, [_vp, _dbl, _dbl, _i32, _i32, _vp, _vp, _vp, _pi32]),
    "vgb_unplaced_trd": (ctypes.c_int, [_vp] + [_dbl] * 5 + [_pi32]),
    "vgb_unplaced_orb": (ctypes.c_int, [_vp, _dbl, _pi32]),
    "vgb_unplaced_parallelepiped": (ctypes.c_int, [_vp] + [_dbl] * 6 + [_pi32]),
    "vgb_unplaced_paraboloid": (ctypes.c_int, [_vp] + [_dbl] * 3 + [_pi32]),
    "vgb_unplaced_trapezoid": (ctypes.c_int, [_vp] + [_dbl] * 11 + [_pi32]),
    "vgb_unplaced_trapezoid_corners": (ctypes.c_int, [_vp, _vp, _pi32]),
    "vgb_unplaced_boolean": (ctypes.c_int, [_vp, _i32, _i32, _i32, _pi32]),
    "vgb_transformation": (ctypes.c_int, [_vp] + [_dbl] * 6 + [_pi32]),
    "vgb_transformation_matrix": (ctypes.c_int, [_vp, _dbl, _dbl, _dbl, _vp, _pi32]),
    "vgb_logical_volume": (ctypes.c_int, [_vp, _cp, _i32, _pi32]),
    "vgb_place": (ctypes.c_int, [_vp, _i32, _i32, _pi32]),
    "vgb_place_daughter": (ctypes.c_int, [_vp, _i32, _i32, _i32, _pi32]),
    "vgb_set_world": (ctypes.c_int, [_vp, _i32]),
    "vgb_geometry_close": (ctypes.c_int, [_vp]),
    "vgb_geometry_max_depth": (ctypes.c_int, [_vp, _pi32]),
    "vgb_geometry_device_bytes": (ctypes.c_int, [_vp, _pi64]),
    "vgb_geometry_serialize": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t,
                                              ctypes.POINTER(ctypes.c_size_t)]),
    "vgb_geometry_deserialize": (ctypes.c_int, [_vp, ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "vgb_geometry_save": (ctypes.c_int, [_vp, _cp]),
    "vgb_geometry_load": (ctypes.c_int, [_cp, ctypes.POINTER(_vp)]),
    "vgb_geometry_export_cpp": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t,
                                               ctypes.POINTER(ctypes.c_size_t)]),
    "vgb_batch": (ctypes.c_int, [_vp, _i32, _i32, _i64] + [_vp] * 9 + [_i32, _i32, _vp]),
    "vgb_batch_fused": (ctypes.c_int, [_vp, _i32, _u32, _i64] + [_vp] * 8 + [_u32, _i32, _vp]),
    "vgb_Contains": (ctypes.c_int, [_vp, _i32, _i64, _vp, _vp, _vp, _vp, _vp]),
    "vgb_Inside": (ctypes.c_int, [_vp, _i32, _i64, _vp, _vp, _vp, _vp, _vp]),
    "vgb_DistanceToIn": (ctypes.c_int, [_vp, _i32, _i64] + [_vp] * 9),
    "vgb_DistanceToOut": (ctypes.c_int, [_vp, _i32, _i64] + [_vp] * 9),
    "vgb_SafetyToIn": (ctypes.c_int, [_vp, _i32, _i64, _vp, _vp, _vp, _vp, _vp]),
    "vgb_SafetyToOut": (ctypes.c_int, [_vp, _i32, _i64, _vp, _vp, _vp, _vp, _vp]),
    "vgb_basket_plan_create": (ctypes.c_int, [_vp, _vp, _i32, _u32, _i32, _i32,
                                              ctypes.POINTER(_vp)]),
    "vgb_basket_plan_destroy": (ctypes.c_int, [_vp]),
    "vgb_basket_plan_info": (ctypes.c_int, [_vp, _pi64, _pi64, _pi32, _pi32]),
    "vgb_basket_run": (ctypes.c_int, [_vp] + [_vp] * 8 + [_u32, _vp]),
    "vgb_basket_tune": (ctypes.c_int, [_vp] + [_vp] * 8 + [_u32, _i32, _vp, _pi32, _pi32,
                                                          ctypes.POINTER(ctypes.c_float)]),
    "vgb_basket_graph_capture": (ctypes.c_int, [_vp] + [_vp] * 8 + [_u32]),
    "vgb_basket_graph_launch": (ctypes.c_int, [_vp, _vp]),
    "vgb_basket_run_noalloc": (ctypes.c_int, [_vp, _vp, _i32, _u32] + [_vp] * 8 + [_u32, _vp]),
    "vgb_server_create": (ctypes.c_int, [_vp, _i64, _i32, _i32, _dbl, _i32,
                                         ctypes.POINTER(_vp)]),
    "vgb_server_destroy": (ctypes.c_int, [_vp]),
    "vgb_server_info": (ctypes.c_int, [_vp, _pi64, _pi64]),
    "vgb_server_submit": (ctypes.c_int, [_vp, _i64] + [_vp] * 6 + [_pi64]),
    "vgb_server_step": (ctypes.c_int, [_vp, _pi64, _i32, _pi32, _pi64, _pi64]),
    "vgb_server_result": (ctypes.c_int, [_vp, _i64] + [_vp] * 5),
    "vgb_navpool_create": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(_vp)]),
    "vgb_navpool_destroy": (ctypes.c_int, [_vp]),
    "vgb_navpool_info": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), _pi64, _pi64]),
    "vgb_navpool_upload": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "vgb_navpool_download": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "vgb_nav_locate": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "vgb_nav_find_next_boundary_and_step": (ctypes.c_int, [_vp, _i64] + [_vp] * 11 + [_i32, _vp]),
    "vgb_nav_trace": (ctypes.c_int, [_vp, _i64] + [_vp] * 6 + [_dbl, _i32] + [_vp] * 4
                      + [_i32, _vp]),
    "vgb_nav_find_next_boundary_and_step_basket": (ctypes.c_int, [_vp, _i64] + [_vp] * 13),
    "vgb_abbox_nav_find_next_boundary_and_step": (ctypes.c_int, [_vp, _i64] + [_vp] * 12),
    "vgb_abbox_nav_trace": (ctypes.c_int, [_vp, _i64] + [_vp] * 6 + [_dbl, _i32] + [_vp] * 5),
    "vgb_abbox_compute": (ctypes.c_int, [_vp, _i32, _vp]),
    "vgb_nav_error_flags": (ctypes.c_int, [_vp, ctypes.POINTER(_u32)]),
}

NAV_ERR_DEPTH = 1
NOALLOC_MAX_BASKETS = 8192


def lib():
    """Load libvgb.so once; raise if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libvgb.so not found at {LIB_PATH}: build it with "
            "`make -C vecgeom_b200/csrc` (or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != OK:
        raise VgbError(status, lib().vgb_last_error().decode(errors="replace"))
