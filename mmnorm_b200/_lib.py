"""ctypes binding of the C ABI in include/mmnorm_b200.h (libmmnorm_b200.so, in-tree).

There is no CPU fallback: if the library is missing it is built with nvcc on first
use, and if that is impossible importing the product API raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

MMN_OK = 0
MMN_ERR_INVALID_ARGUMENT = 1
MMN_ERR_NULL_POINTER = 2
MMN_ERR_UNSUPPORTED = 3
MMN_ERR_WORKSPACE = 4
MMN_ERR_CUDA = 5
MMN_ERR_TIMEOUT = 6
MMN_ERR_TOO_LARGE = 7

MODE_MIXED = 0
MODE_PLAIN = 1
MODE_INTERP = 2
MODE_INTERP_FAST = 3
MODES = {"mixed": MODE_MIXED, "plain": MODE_PLAIN, "interp": MODE_INTERP,
         "interp_fast": MODE_INTERP_FAST}

_ERR_NAMES = {
    MMN_ERR_INVALID_ARGUMENT: "invalid argument",
    MMN_ERR_NULL_POINTER: "null pointer",
    MMN_ERR_UNSUPPORTED: "unsupported device or feature",
    MMN_ERR_WORKSPACE: "workspace missing, misaligned or too small",
    MMN_ERR_CUDA: "CUDA runtime error",
    MMN_ERR_TIMEOUT: "bounded in-kernel wait timed out",
    MMN_ERR_TOO_LARGE: "size exceeds a documented maximum",
}


class MmnError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__("%s failed: %s (code %d)" % (where, _ERR_NAMES.get(code, "?"), code))


class MmnProblem(ctypes.Structure):
    """Mirror of ``mmn_problem`` (include/mmnorm_b200.h)."""

    _fields_ = [
        ("num_x", ctypes.c_int32), ("num_y", ctypes.c_int32), ("num_z", ctypes.c_int32),
        ("x_locs", ctypes.c_void_p), ("y_locs", ctypes.c_void_p), ("z_locs", ctypes.c_void_p),
        ("num_antennas", ctypes.c_int32), ("num_rx", ctypes.c_int32),
        ("antenna_locs", ctypes.c_void_p), ("rx_offsets", ctypes.c_void_p),
        ("pos_offsets", ctypes.c_void_p),
        ("num_samples", ctypes.c_int32),
        ("meas", ctypes.c_void_p),
        ("wavelength", ctypes.c_double), ("slope", ctypes.c_double),
        ("fft_spacing", ctypes.c_double),
        ("is_ti_radar", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


class MmnIsoScene(ctypes.Structure):
    """Mirror of ``mmn_iso_scene`` (include/mmnorm_b200.h)."""

    _fields_ = [
        ("grids", ctypes.c_void_p), ("num_comp", ctypes.c_int32),
        ("res_x", ctypes.c_int32), ("res_y", ctypes.c_int32), ("res_z", ctypes.c_int32),
        ("bbox", ctypes.c_float * 6), ("voxel_size", ctypes.c_float),
        ("lower", ctypes.c_float * 3), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
        ("width_fov", ctypes.c_float), ("height_fov", ctypes.c_float),
        ("range_offset", ctypes.c_double), ("f0_over_c", ctypes.c_double),
        ("df_over_c", ctypes.c_double), ("num_wl", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]


# (name, restype, argtypes) of every entry point in include/mmnorm_b200.h
_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I = ctypes.c_int
_SZ = ctypes.c_size_t
_F = ctypes.c_float
_PROB = ctypes.POINTER(MmnProblem)
_I32P = ctypes.POINTER(ctypes.c_int32)
SIGNATURES = [
    ("mmn_version", ctypes.c_char_p, []),
    ("mmn_check_device", _I, [_I]),
    ("mmn_workspace_bytes", _SZ, [_PROB, _I32, _I32]),
    ("mmn_num_variants", _I, [_I32]),
    ("mmn_variant_info", _I, [_I32, _I32, _I32P, _I32P]),
    ("mmn_set_variant", _I, [_I32, _I32]),
    ("mmn_get_variant", _I, [_I32]),
    ("mmn_variant_name", ctypes.c_char_p, [_I32, _I32]),
    ("mmn_plan_info", _I, [_PROB, _I32, _I32P, _I32P, _I32P, _I32P, _I32P]),
    ("mmn_plan_launches", _I, [_PROB, _I32, _I32P]),
    ("mmn_backproject", _I, [_PROB, _I32, _P, _P, _P, _SZ, _P]),
    ("mmn_backproject_noalloc", _I, [_PROB, _I32, _P, _P, _P]),
    ("mmn_noalloc_read_status", _I, [_I32P, _P]),
    ("mmn_backward_workspace_bytes", _SZ, [_PROB]),
    ("mmn_backproject_nufft_workspace_bytes", _SZ, [_PROB]),
    ("mmn_backproject_nufft", _I, [_PROB, _P, _P, _P, _SZ, _P]),
    ("mmn_set_position_pass", _I, [_I32]),
    ("mmn_set_measurement_pass", _I, [_I32]),
    ("mmn_set_interp_fast_form", _I, [_I32]),
    ("mmn_num_position_variants", _I, []),
    ("mmn_position_variant_name", ctypes.c_char_p, [_I32]),
    ("mmn_set_position_variant", _I, [_I32]),
    ("mmn_get_position_variant", _I, []),
    ("mmn_backproject_backward", _I, [_PROB, _P, _P, _P, _P, _P, _SZ, _P]),
    ("mmn_normals_workspace_bytes", _SZ, [ctypes.c_int64]),
    ("mmn_normals", _I, [ctypes.c_int64, _P, _P, _F, _P, _P, _P, _P, _SZ, _P]),
    ("mmn_image_max_abs", _I, [ctypes.c_int64, _P, _P, _P]),
    ("mmn_iso_channels_workspace_bytes", _SZ, [ctypes.POINTER(MmnIsoScene), _I32, _I32]),
    ("mmn_iso_channels", _I, [ctypes.POINTER(MmnIsoScene), _P, _I32, _P, _P, _I32, _P, _P, _SZ,
                              _P]),
    ("mmn_iso_march", _I, [ctypes.POINTER(MmnIsoScene), _I32, _F, _P, _P, _P, _P, _P, _P]),
    ("mmn_adc_unpack", _I, [_P, ctypes.c_int64, _P, _P]),
    ("mmn_correlate_poses", _I, [_P, _P, ctypes.c_int64, _I32, _P, _P, _I32, _I32,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                 ctypes.c_int64, _I32, _P, _P, _P, _P]),
    ("mmn_components_workspace_bytes", _SZ, [ctypes.c_int64]),
    ("mmn_components", _I, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P,
                            _SZ, _P]),
    ("mmn_rsdf_workspace_bytes", _SZ, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    ("mmn_rsdf_component", _I, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P,
                                ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _P, _P, _P,
                                _SZ, _P]),
    ("mmn_normals_from_max", _I, [ctypes.c_int64, _P, _P, _P, _F, _P, _P, _P, _P]),
    ("mmn_cuda_image_workspace_bytes", _SZ, [_I, _I, _I]),
    ("mmn_cuda_image_workspace_bytes_for", _SZ, [_I, _I, _I, _I, _I, _I, _I, _I]),
    ("mmn_cuda_image", _I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _F, _F, _F, _I, _I, _I, _I,
                            _I, _I, _I, _I, _I, _I, _P, _SZ, _P]),
    ("mmn_cuda_sn_est_workspace_bytes", _SZ, [_I, _I]),
    ("mmn_cuda_sn_est", _I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _F,
                             _F, _F, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _SZ, _P]),
    ("mmn_cuda_sn_est_fast", _I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                  _F, _F, _F, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _SZ,
                                  _P]),
    ("mmn_fp32_peak_probe", _I, [_I, _I, _P, _P]),
    ("mmn_wait_timeout_probe", _I, [ctypes.c_uint32, _I, _P, _P]),
    ("mmn_batch_create", _I, [_PROB, _I32, _I32, _P, _P, _I32, ctypes.POINTER(_P),
                              ctypes.POINTER(_SZ)]),
    ("mmn_batch_upload", _I, [_P, _P, _SZ, _P]),
    ("mmn_batch_run", _I, [_P, _P, _P]),
    ("mmn_batch_info", _I, [_P, _I32P, _I32P, _I32P, _I32P]),
    ("mmn_batch_destroy", None, [_P]),
    ("mmn_read_status", _I, [_P, _I32P, _P]),
]

_lock = threading.Lock()
_handle = None


def library_path() -> str:
    return _build.LIB


def load():
    """Load (building first if absent) the CUDA library; raises if impossible."""
    global _handle
    with _lock:
        if _handle is not None:
            return _handle
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        if not os.path.exists(path):
            raise ImportError("mmnorm_b200: CUDA library %s is missing" % path)
        h = ctypes.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _handle = h
        return h


def check(code: int, where: str) -> None:
    if code != MMN_OK:
        raise MmnError(code, where)
