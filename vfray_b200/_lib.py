"""ctypes binding of the vfray_b200 C ABI (include/vfray.h).

The shared library is built in-tree (``make -C vfray_b200`` or
``__graft_entry__.build()``) as vfray_b200/libvfray_b200.so.  There is no
fallback: if the library is missing, or a call fails, this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvfray_b200.so")

VFR_OK = 0
VFR_ERR_INVALID = -1
VFR_ERR_CUDA = -2
VFR_ERR_MESH = -3
VFR_ERR_NOMEM = -4
VFR_ERR_DEVICE = -5
VFR_ERR_STATE = -6
VFR_ERR_IO = -7
VFR_ERR_BUDGET = -8
VFR_ERR_TIMEOUT = -9

VFR_DEV_STEP_CAP = 2
VFR_DEV_RANGE = 4
VFR_DEV_QUEUE = 8
VFR_DEV_OVERFLOW = 16
VFR_DEV_CYCLE = 32

OPT_STEP_CAP = 1
OPT_BLOCKS_PER_SM = 3
OPT_PROFILE = 4
OPT_TRAVERSE_VARIANT = 5
OPT_REFILL = 6
OPT_RASTER_WARPS = 7
OPT_TILE_WIDTH = 8

MODE_REF = 0
MODE_COMPOSITED = 1


class VfrError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class RenderStats(C.Structure):
    _fields_ = [("num_ext", C.c_uint32), ("num_vis", C.c_uint32), ("num_rays", C.c_uint32),
                ("num_entries", C.c_uint32), ("num_steps", C.c_uint64),
                ("device_status", C.c_uint32), ("ms_visible", C.c_float),
                ("ms_project", C.c_float), ("ms_traverse", C.c_float), ("ms_total", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Job(C.Structure):
    """vfr_job of include/vfray.h."""
    _fields_ = [("mesh_id", C.c_int), ("W", C.c_uint32), ("H", C.c_uint32), ("use_mv", C.c_int),
                ("mv", C.c_float * 16), ("rgb8_dev", C.c_void_p), ("rgba_dev", C.c_void_p),
                ("steps_dev", C.c_void_p)]


class Tuning(C.Structure):
    """vfr_tuning of include/vfray.h."""
    _fields_ = [("variant", C.c_uint32), ("refill", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("tile_w", C.c_uint32), ("raster_warps_per_sm", C.c_uint32), ("ms", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Request(C.Structure):
    """vfr_request of include/vfray.h."""
    _fields_ = [("mesh_id", C.c_int), ("W", C.c_uint32), ("H", C.c_uint32), ("use_mv", C.c_int),
                ("mv", C.c_float * 16), ("mode", C.c_int), ("rgb8_host", C.c_void_p)]


class RequestInfo(C.Structure):
    """vfr_request_info of include/vfray.h."""
    _fields_ = [("status", C.c_int), ("t_submit_ms", C.c_double), ("t_start_ms", C.c_double),
                ("t_done_ms", C.c_double), ("batch_id", C.c_uint32), ("batch_jobs", C.c_uint32),
                ("num_rays", C.c_uint32), ("num_steps", C.c_uint64),
                ("device_status", C.c_uint32), ("t_ready_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    """vfr_server_stats of include/vfray.h."""
    _fields_ = [("batches", C.c_uint32), ("pending", C.c_uint32), ("completed", C.c_uint64),
                ("rejected", C.c_uint64), ("budget_used", C.c_uint64), ("rays", C.c_uint64),
                ("steps", C.c_uint64), ("launches", C.c_uint32), ("epochs", C.c_uint32),
                ("queue_timeouts", C.c_uint32), ("mesh_bytes", C.c_uint64),
                ("arena_bytes", C.c_uint64), ("prep_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = C.c_void_p
_u32 = C.c_uint32
_i = C.c_int
_f = C.c_float

# name -> (restype, argtypes); mirrors include/vfray.h
SIGNATURES = {
    "vfr_create": (_i, [C.POINTER(_vp), _i]),
    "vfr_destroy": (None, [_vp]),
    "vfr_last_error": (C.c_char_p, [_vp]),
    "vfr_status_string": (C.c_char_p, [_i]),
    "vfr_set_stream": (_i, [_vp, _vp]),
    "vfr_synchronize": (_i, [_vp]),
    "vfr_set_option": (_i, [_vp, _i, C.c_int64]),
    "vfr_profile_read": (_i, [_vp, _vp, _i, C.POINTER(_i)]),
    "vfr_tables_upload": (_i, [_vp, _vp, _vp]),
    "vfr_mesh_upload": (_i, [_vp, _vp, _u32, _vp, _vp, _u32, _vp, _u32, _f, _f, _f,
                             C.POINTER(_i)]),
    "vfr_mesh_release": (_i, [_vp, _i]),
    "vfr_mesh_bytes": (_i, [_vp, _i, C.POINTER(C.c_uint64)]),
    "vfr_find_visible": (_i, [_vp, _i, C.POINTER(_u32), _vp, _vp]),
    "vfr_project": (_i, [_vp, _i, _u32, _u32, _vp, _vp]),
    "vfr_traverse": (_i, [_vp, _i, _vp, _vp, _vp, C.POINTER(RenderStats)]),
    "vfr_render": (_i, [_vp, _i, _vp, _u32, _u32, _i, _vp, _vp, _vp, C.POINTER(RenderStats)]),
    "vfr_render_device": (_i, [_vp, _i, _vp, _u32, _u32, _i, _vp, _vp, _vp, _vp]),
    "vfr_device_status": (_i, [_vp, C.POINTER(_u32)]),
    "vfr_batch_create": (_i, [_vp, C.POINTER(_vp)]),
    "vfr_batch_destroy": (None, [_vp]),
    "vfr_batch_set_jobs": (_i, [_vp, C.POINTER(Job), _u32, _i]),
    "vfr_batch_capture": (_i, [_vp]),
    "vfr_batch_run": (_i, [_vp]),
    "vfr_batch_stats": (_i, [_vp, C.POINTER(RenderStats), _u32]),
    "vfr_batch_output": (_i, [_vp, _u32, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
    "vfr_batch_read": (_i, [_vp, _vp, _vp, _vp]),
    "vfr_batch_read_async": (_i, [_vp, _vp, _vp, _vp]),
    "vfr_batch_synchronize": (_i, [_vp]),
    "vfr_batch_set_stream": (_i, [_vp, _vp]),
    "vfr_batch_set_cameras": (_i, [_vp, _vp, _u32]),
    "vfr_batch_autotune": (_i, [_vp, _i, C.POINTER(Tuning)]),
    "vfr_batch_scratch_bytes": (_i, [_vp, C.POINTER(C.c_uint64)]),
    "vfr_server_create": (_i, [_vp, C.c_uint64, _u32, C.POINTER(_vp)]),
    "vfr_server_submit": (_i, [_vp, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "vfr_server_wait": (_i, [_vp, C.c_uint64, _i, C.POINTER(RequestInfo)]),
    "vfr_server_stats": (_i, [_vp, C.POINTER(ServerStats)]),
    "vfr_server_set_idle": (_i, [_vp, _u32, _u32]),
    "vfr_server_destroy": (None, [_vp]),
    "vfr_find_visible_static": (_i, [_vp, _u32, _vp, _u32, _vp, _u32, _vp, _vp, _vp]),
    "vfr_psi_table": (_i, [_vp]),
    "vfr_psi_table_reference": (_i, [_vp]),
    "vfr_normalize": (_i, [_vp, _u32]),
    "vfr_rotate": (_i, [_vp, _u32, _vp]),
    "vfr_build_con": (_i, [_vp, _u32, _u32, _vp, C.POINTER(_u32), _i]),
    "vfr_build_extf": (_i, [_vp, _u32, _vp, _u32, C.POINTER(_u32)]),
    "vfr_build_lmt": (_i, [_vp, _u32, _vp, _u32, _vp]),
    "vfr_default_tf": (_i, [_vp]),
    "vfr_read_off": (_i, [C.c_char_p, _vp, C.POINTER(_u32), _vp, C.POINTER(_u32)]),
    "vfr_read_con": (_i, [C.c_char_p, _vp, C.POINTER(_u32), C.POINTER(_u32)]),
    "vfr_read_extf": (_i, [C.c_char_p, _vp, C.POINTER(_u32)]),
    "vfr_read_lmt": (_i, [C.c_char_p, _vp]),
    "vfr_read_tf": (_i, [C.c_char_p, _vp]),
    "vfr_write_off": (_i, [C.c_char_p, _vp, _u32, _vp, _u32]),
    "vfr_write_con": (_i, [C.c_char_p, _vp, _u32, _u32]),
    "vfr_write_extf": (_i, [C.c_char_p, _vp, _u32]),
    "vfr_write_lmt": (_i, [C.c_char_p, _vp]),
    "vfr_write_tf": (_i, [C.c_char_p, _vp]),
    "vfr_write_ppm": (_i, [C.c_char_p, _vp, _u32, _u32]),
    "vfr_read_psi_source": (_i, [C.c_char_p, _vp]),
    "vfr_clean_tf": (_i, [C.c_char_p, C.c_char_p]),
    "vfr_write_mesh_cache": (_i, [C.c_char_p, _vp, _u32, _vp, _vp, _u32, _vp, _u32, _vp]),
    "vfr_read_mesh_cache": (_i, [C.c_char_p, _vp, C.POINTER(_u32), _vp, _vp, C.POINTER(_u32), _vp,
                                 C.POINTER(_u32), _vp]),
}

_LIB = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library (once).  Raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C vfray_b200` "
                          "or __graft_entry__.build()")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def ptr(a) -> C.c_void_p | None:
    """Pointer of a C-contiguous numpy array or a torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return C.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return C.c_void_p(a.data_ptr())
    raise TypeError(f"cannot take a pointer of {type(a)}")


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc == VFR_OK:
        return
    lib = load()
    msg = lib.vfr_status_string(rc).decode()
    if ctx is not None:
        detail = lib.vfr_last_error(ctx).decode()
        if detail:
            msg += f": {detail}"
    raise VfrError(rc, f"{what}: {msg}" if what else msg)
