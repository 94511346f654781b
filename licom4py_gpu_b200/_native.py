"""ctypes binding of ``libbt.so`` (include/licom_bt.h).

The package has no CPU fallback: if the library is missing, or no CUDA device
is visible, the first call raises instead of computing anything elsewhere.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbt.so")

BT_OK, BT_EINVAL, BT_ENOMEM, BT_ECUDA, BT_EDEVICE, BT_ENOTSUP = 0, -1, -2, -3, -4, -5
BT_F64, BT_F32 = 0, 1
BT_MODE_STREAM, BT_MODE_GRAPH, BT_MODE_PERSISTENT, BT_MODE_RESIDENT = 0, 1, 2, 3
BT_OPT_MAX_CTAS, BT_OPT_SPIN_LIMIT, BT_OPT_KERNEL_TIMING, BT_OPT_FULL_TILES = 1, 2, 3, 4
BT_INFO_LAST_GRID, BT_INFO_SCRATCH_BYTES, BT_INFO_FULL_TILES = 1, 2, 3
BT_KERNEL_ROUND, BT_KERNEL_PHASE_H, BT_KERNEL_PHASE_UV = 0, 1, 2

_vp = ctypes.c_void_p


class GridDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("dtype", ctypes.c_int)] + [
        (name, _vp) for name in (
            "dzph_x", "dzph_y", "rdx", "rdy", "a_f", "k2e_coef", "loc_i_local", "loc_j_local",
            "a_c2l", "a_l2c", "inner", "outer", "a_gct", "a_sina", "rda", "c_dy", "d_dx")]


class StateIn(ctypes.Structure):
    _fields_ = [(k, _vp) for k in ("h0", "h0p", "ub", "vb", "ubp", "vbp")]


class StateOut(ctypes.Structure):
    _fields_ = [("h0", _vp), ("ub", _vp), ("vb", _vp), ("diag", _vp * 10)]


class Member(ctypes.Structure):
    _fields_ = [("plan", _vp), ("inp", StateIn), ("out", StateOut), ("scratch", _vp), ("nbb", ctypes.c_int),
                ("dtb", ctypes.c_double)]


class BtError(RuntimeError):
    """A CUDA or device-side failure reported by libbt."""


_lib = None

# every symbol declared in include/licom_bt.h
EXPORTS = ("bt_plan_create", "bt_plan_destroy", "bt_plan_set_tile", "bt_plan_set_mode",
           "bt_plan_set_option", "bt_plan_get_info", "bt_plan_kernel_time", "bt_round",
           "bt_stage", "bt_fill_halo", "bt_edge_average", "bt_check_device_error", "bt_halo_table_host", "bt_interior_stats", "bt_conservation",
           "bt_round_noalloc",
           "bt_member_scratch_bytes", "bt_batch_create", "bt_batch_destroy", "bt_batch_set_mode",
           "bt_batch_set_tile", "bt_batch_set_option", "bt_batch_get_info", "bt_batch_round",
           "bt_batch_check_device_error",
           "bt_last_error", "bt_version")


def lib():
    """Load libbt.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA extension with `python -m licom4py_gpu_b200.build`"
            " (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.bt_plan_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(_vp)]
    L.bt_plan_destroy.argtypes = [_vp]
    L.bt_plan_set_tile.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.bt_plan_set_mode.argtypes = [_vp, ctypes.c_int]
    L.bt_plan_set_option.argtypes = [_vp, ctypes.c_int, ctypes.c_longlong]
    L.bt_plan_get_info.argtypes = [_vp, ctypes.c_int]
    L.bt_plan_kernel_time.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int)]
    L.bt_round.argtypes = [_vp, ctypes.POINTER(StateIn), ctypes.POINTER(StateOut), ctypes.c_int,
                           ctypes.c_double, ctypes.c_int, _vp]
    L.bt_stage.argtypes = [_vp, ctypes.POINTER(StateIn), ctypes.POINTER(StateOut), ctypes.c_double,
                           ctypes.c_double, ctypes.c_int, _vp]
    L.bt_fill_halo.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.bt_edge_average.argtypes = [_vp, _vp, _vp, _vp]
    L.bt_check_device_error.argtypes = [_vp]
    L.bt_halo_table_host.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp]
    L.bt_interior_stats.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp]
    L.bt_conservation.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, ctypes.c_double, _vp, _vp]
    L.bt_round_noalloc.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(StateIn), ctypes.POINTER(StateOut),
                                   ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp]
    L.bt_member_scratch_bytes.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]
    L.bt_batch_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]
    L.bt_batch_destroy.argtypes = [_vp]
    L.bt_batch_set_mode.argtypes = [_vp, ctypes.c_int]
    L.bt_batch_set_tile.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.bt_batch_set_option.argtypes = [_vp, ctypes.c_int, ctypes.c_longlong]
    L.bt_batch_get_info.argtypes = [_vp, ctypes.c_int]
    L.bt_batch_round.argtypes = [_vp, ctypes.POINTER(Member), ctypes.c_int, ctypes.c_int, _vp]
    L.bt_batch_check_device_error.argtypes = [_vp]
    L.bt_last_error.argtypes = []
    L.bt_last_error.restype = ctypes.c_char_p
    L.bt_version.argtypes = []
    for name in EXPORTS:
        if name != "bt_last_error":
            getattr(L, name).restype = ctypes.c_int
    L.bt_plan_get_info.restype = ctypes.c_longlong
    L.bt_batch_get_info.restype = ctypes.c_longlong
    _lib = L
    return L


def check(rc: int) -> None:
    """Map a libbt return code to the reference's exception types."""
    if rc == BT_OK:
        return
    msg = lib().bt_last_error().decode(errors="replace")
    if rc == BT_EINVAL:
        raise ValueError(msg)
    if rc == BT_ENOMEM:
        raise MemoryError(msg)
    if rc == BT_ENOTSUP:
        raise NotImplementedError(msg)
    raise BtError(f"libbt error {rc}: {msg}")
