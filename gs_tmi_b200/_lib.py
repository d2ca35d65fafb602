"""ctypes binding of ``lib/libgsv_b200.so`` (the C ABI of ``include/gsv.h``).

There is deliberately no fallback: if the sm_100a library is missing the
import of this module raises, and every voxelizer entry point with it.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgsv_b200.so")

GSV_OK = 0
GSV_ERR_INVALID_ARGUMENT = 1
GSV_ERR_CAPACITY = 2
GSV_ERR_CUDA = 3
GSV_ERR_EMPTY_BOX = 4
GSV_ERR_TOO_MANY_PAIRS = 5

GSV_FLAG_CAPACITY_OVERFLOW = 0x1
GSV_FLAG_EMPTY_BOX = 0x2
GSV_FLAG_TOO_MANY_PAIRS = 0x4
GSV_FLAG_SCAN_STALLED = 0x8

GSV_BACKWARD_DETERMINISTIC = 0x1
GSV_TUNE_NO_CULL = 0x1

GSV_BIN_AUTO, GSV_BIN_RADIX, GSV_BIN_COUNTING = 0, 1, 2


class GsvShape(ctypes.Structure):
    _fields_ = [("d", ctypes.c_int32), ("h", ctypes.c_int32), ("w", ctypes.c_int32),
                ("tile_size", ctypes.c_int32)]


class GsvParams(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("scales", ctypes.c_void_p),
                ("rotations", ctypes.c_void_p), ("density_r", ctypes.c_void_p),
                ("density_i", ctypes.c_void_p), ("n", ctypes.c_int64)]


class GsvGrads(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("scales", ctypes.c_void_p),
                ("rotations", ctypes.c_void_p), ("density_r", ctypes.c_void_p),
                ("density_i", ctypes.c_void_p)]


class GsvBatchItem(ctypes.Structure):
    _fields_ = [("shape", GsvShape), ("params", GsvParams), ("ws_gauss", ctypes.c_void_p),
                ("ws_pairs", ctypes.c_void_p), ("capacity", ctypes.c_int64), ("volume", ctypes.c_void_p),
                ("grad_volume", ctypes.c_void_p), ("grads", GsvGrads), ("chunk", ctypes.c_int32)]


GSV_DENSITY_SPLIT = 0x1
GSV_DENSITY_CLONE = 0x2
GSV_DENSITY_PRUNE = 0x4
GSV_DENSITY_ROW_OVERFLOW = 0x8


class GsvDensityRows(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("log_scales", ctypes.c_void_p), ("rotations", ctypes.c_void_p),
                ("density_r", ctypes.c_void_p), ("density_i", ctypes.c_void_p),
                ("exp_avg", ctypes.c_void_p * 5), ("exp_avg_sq", ctypes.c_void_p * 5), ("capacity", ctypes.c_int64)]


class GsvDensityConfig(ctypes.Structure):
    _fields_ = [("grad_threshold", ctypes.c_float), ("scale_threshold", ctypes.c_float),
                ("opacity_threshold", ctypes.c_float), ("max_scale", ctypes.c_float),
                ("long_axis_offset_factor", ctypes.c_float), ("long_axis_split", ctypes.c_int32),
                ("use_cloning", ctypes.c_int32), ("min_keep", ctypes.c_int32), ("max_points", ctypes.c_int64)]


class GsvTuning(ctypes.Structure):
    _fields_ = [("rows_per_lane", ctypes.c_int32), ("chunk", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("split", ctypes.c_int32)]


# name -> (restype, argtypes); the complete exported C ABI.
_vp, _i32, _i64, _sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_size_t
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_S, _P, _G = GsvShape, ctypes.POINTER(GsvParams), ctypes.POINTER(GsvGrads)
SIGNATURES = {
    "gsv_abi_version": (ctypes.c_int, []),
    "gsv_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "gsv_last_error": (ctypes.c_char_p, []),
    "gsv_num_tiles": (_i64, [_S]),
    "gsv_gauss_workspace_bytes": (_sz, [_i64, _S]),
    "gsv_pair_workspace_bytes": (_sz, [_i64, _S, ctypes.c_int]),
    "gsv_prepare": (ctypes.c_int, [_P, _S, _vp, _sz, _i64p, _vp]),
    "gsv_prepare_live": (ctypes.c_int, [_P, _vp, _S, _vp, _sz, _i64p, _vp]),
    "gsv_bin": (ctypes.c_int, [_S, _i64, _vp, _vp, _sz, _i64, _vp]),
    "gsv_bin_ex": (ctypes.c_int, [_S, _i64, _vp, _vp, _sz, _i64, ctypes.c_int, _vp]),
    "gsv_bin_views": (ctypes.c_int, [_S, _i64, _vp, _vp, _i64, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "gsv_status_views": (ctypes.c_int, [_S, _i64, _vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "gsv_read_status": (ctypes.c_int, [_S, _i64, _vp, _i64p, _i32p, _vp]),
    "gsv_forward": (ctypes.c_int, [_S, _i64, _vp, _vp, _i64, _vp, _vp]),
    "gsv_forward_ex": (ctypes.c_int, [_S, _i64, _vp, _vp, _i64, _vp, ctypes.c_void_p, _vp]),
    "gsv_backward_ex": (ctypes.c_int, [_P, _S, _vp, _vp, _i64, _vp, _G, ctypes.c_int, ctypes.c_void_p, _vp]),
    "gsv_backward": (ctypes.c_int, [_P, _S, _vp, _vp, _i64, _vp, _G, ctypes.c_int, _vp]),
    "gsv_batch_workspace_bytes": (_sz, [ctypes.c_int]),
    "gsv_batch_setup": (ctypes.c_int, [ctypes.POINTER(GsvBatchItem), ctypes.c_int, ctypes.c_int, _vp, _sz, _vp]),
    "gsv_forward_batched": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "gsv_backward_batched": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    "gsv_count_work": (ctypes.c_int, [_S, _i64, _vp, _vp, _i64, ctypes.c_void_p, _vp, _vp]),
    "gsv_build_tile_pairs_count": (ctypes.c_int, [_vp, _vp, _i64, _S, _vp, _sz, _i64p, _vp]),
    "gsv_build_tile_pairs_fill": (ctypes.c_int, [_S, _i64, _vp, _vp, _sz, _i64, _vp, _vp, _vp]),
    "gsv_build_tile_pairs_noalloc": (ctypes.c_int, [_vp, _vp, _i64, _S, _vp, _vp, _i64, _i64p, _vp]),
    "gsv_mlp_gemm": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_longlong, _vp, ctypes.c_longlong,
                                    ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                    _vp, _vp, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int, _vp, _vp, _vp]),
    "gsv_mlp_gemm_test_timeout": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                 ctypes.c_longlong, _vp, _vp]),
    "gsv_sense_workspace_bytes": (_sz, []),
    "gsv_sense_expand": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp]),
    "gsv_sense_residual": (ctypes.c_int, [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _sz, _vp]),
    "gsv_sense_adjoint": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, _i32, _vp, _vp]),
    "gsv_tv_magnitude": (ctypes.c_int, [_vp, _i32, _i32, _i32, _vp, _vp, _vp, _sz, _vp]),
    "gsv_density_workspace_bytes": (_sz, [_i64]),
    "gsv_density_control": (ctypes.c_int, [ctypes.POINTER(GsvDensityRows), _vp, _vp,
                                           ctypes.POINTER(GsvDensityConfig), _vp, _vp, _vp, _sz, _vp]),
    "gsv_normal_fill": (ctypes.c_int, [_vp, _i64, ctypes.c_uint64, _vp, _vp]),
    "gsv_poisson_workspace_bytes": (_sz, [_i32, _i32, _i32]),
    "gsv_poisson_masks": (ctypes.c_int, [_vp, _vp, _i32, _i32, _i32, _i64, _i32, _vp, _vp, _vp, _sz, _vp]),
    "gsv_knn3_mean_distance": (ctypes.c_int, [_vp, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _vp]),
    "gsv_tile_forward": (ctypes.c_int, [_vp] * 7 + [_i64, _i64, _i32, _i32, _i32, _i32, _vp, _vp, _vp]),
    "gsv_tile_backward": (ctypes.c_int, [_vp] * 9 + [_i64, _i64, _i32, _i32, _i32, _i32] + [_vp] * 5),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the sm_100a voxelizer library with "
            "`python gs_tmi_b200/build.py` (this package has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class GsvError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib.gsv_status_string(status).decode()
        if status == GSV_ERR_CUDA:
            msg += ": " + lib.gsv_last_error().decode()
        super().__init__(f"{where}: {msg}")
        self.status = status


def check(status: int, where: str) -> None:
    if status != GSV_OK:
        raise GsvError(status, where)
