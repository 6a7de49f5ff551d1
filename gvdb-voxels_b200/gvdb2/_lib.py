"""ctypes binding of libgvdb2.so (the C-ABI in include/gvdb2.h).

The library is built in-tree (gvdb-voxels_b200/lib/libgvdb2.so).  There is
no fallback: if it cannot be loaded, every call raises.
"""
import ctypes
import os
import re

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libgvdb2.so")
HEADER = os.path.join(os.path.dirname(_PKG), "include", "gvdb2.h")

OK = 0
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_DEPTH", 3: "ERR_STATE", 4: "ERR_UNSUPPORTED", 5: "ERR_NOMEM",
                6: "ERR_CUDA", 7: "ERR_CAPACITY", 8: "ERR_NOT_AVAILABLE"}
T_FLOAT = 3
KERNEL_TENT1 = 1
KERNEL_CUBIC2 = 2
OPT_DETERMINISTIC = 1
OPT_AUTOTUNE = 2
NV_FLOAT = 1
NV_VEC3F = 3


class PointsView(ctypes.Structure):
    _fields_ = [("base", ctypes.c_void_p), ("count", ctypes.c_int64),
                ("stride_bytes", ctypes.c_int32), ("offset_bytes", ctypes.c_int32)]


class Info(ctypes.Structure):
    _fields_ = [("depth", ctypes.c_int32), ("top_level", ctypes.c_int32), ("num_levels", ctypes.c_int32),
                ("apron", ctypes.c_int32), ("pool_count", ctypes.c_int64 * 10), ("used_leaves", ctypes.c_int64),
                ("atlas_slots", ctypes.c_int64), ("atlas_capacity", ctypes.c_int64),
                ("atlas_subdim", ctypes.c_int32 * 3), ("res", ctypes.c_int32 * 10), ("range", ctypes.c_int64 * 10),
                ("posmin", ctypes.c_float * 3), ("posmax", ctypes.c_float * 3), ("root_pos", ctypes.c_int32 * 3),
                ("tile_res", ctypes.c_int32), ("splat_cells", ctypes.c_int64),
                ("vol_min", ctypes.c_float * 3), ("vol_max", ctypes.c_float * 3), ("vox_res", ctypes.c_float * 3),
                ("vox_res_max", ctypes.c_float * 3)]


class Tuning(ctypes.Structure):
    _fields_ = [("dense", ctypes.c_int32), ("slice", ctypes.c_int32), ("light", ctypes.c_int32)]


class GvdbError(RuntimeError):
    def __init__(self, status, what, msg=""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)} {msg}".strip())


_lib = None

_vp, _i32, _i64, _f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_SIGS = {
    "gvdb2_create": [ctypes.POINTER(_vp), _i32],
    "gvdb2_destroy": [_vp],
    "gvdb2_set_stream": [_vp, _vp],
    "gvdb2_synchronize": [_vp],
    "gvdb2_set_option": [_vp, _i32, _i32],
    "gvdb2_configure": [_vp, _i32, _i32, _i32, _i32, _i32],
    "gvdb2_set_channel_default": [_vp, _i32, _i32, _i32],
    "gvdb2_add_channel": [_vp, _i32, _i32, _i32],
    "gvdb2_set_points": [_vp, PointsView, PointsView, PointsView],
    "gvdb2_request_full_rebuild": [_vp, _i32],
    "gvdb2_batch_points": [_vp, ctypes.POINTER(PointsView), _i32, _i32, ctypes.POINTER(ctypes.c_int64)],
    "gvdb2_batch_origin": [_vp, _i32, ctypes.POINTER(ctypes.c_int32)],
    "gvdb2_rebuild_topology": [_vp, _i32, _f32, _fp],
    "gvdb2_accumulate_topology": [_vp, _i32, _f32, _fp, _i32],
    "gvdb2_finish_topology": [_vp, _i32, _i32],
    "gvdb2_update_atlas": [_vp],
    "gvdb2_activate_space": [_vp, _fp, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)],
    "gvdb2_compact_pools": [_vp],
    "gvdb2_clear_channel": [_vp, _i32],
    "gvdb2_update_neighbors": [_vp],
    "gvdb2_insert_points": [_vp, _i32, _fp, _i32],
    "gvdb2_insert_points_subcell": [_vp, _i32, _i32, _f32, _fp, _ip],
    "gvdb2_insert_points_subcell_fp16": [_vp, _i32, _i32, _f32, _fp, _ip],
    "gvdb2_get_min_max_vel": [_vp, _i32],
    "gvdb2_set_transform": [_vp, _fp, _fp, _fp, _fp],
    "gvdb2_get_transform": [_vp, _fp, _fp, _fp, _fp],
    "gvdb2_save_vbx": [_vp, ctypes.c_char_p],
    "gvdb2_load_vbx": [_vp, ctypes.c_char_p],
    "gvdb2_nanovdb_size": [_vp, _i32, ctypes.POINTER(ctypes.c_size_t)],
    "gvdb2_export_nanovdb": [_vp, _i32, _ip, _fp, ctypes.c_char_p, _i32, _vp, ctypes.c_size_t],
    "gvdb2_gather_level_set_fp16": [_vp, _i32, _i32, _f32, _fp, _ip, _i32, _i32],
    "gvdb2_scatter_density": [_vp, _i32, _f32, _f32, _fp, _i32, _i32],
    "gvdb2_gather_density": [_vp, _i32, _i32, _f32, _fp, _ip, _i32, _i32, _i32],
    "gvdb2_gather_level_set": [_vp, _i32, _i32, _f32, _fp, _ip, _i32, _i32, _i32],
    "gvdb2_scatter_reduce_level_set": [_vp, _i32, _i32, _f32, _fp, _ip, _i32, _i32, _i32],
    "gvdb2_update_apron": [_vp, _i32, _f32],
    "gvdb2_update_apron_faces": [_vp, _i32],
    "gvdb2_scatter_kernel": [_vp, _i32, _i32, _fp, PointsView, _f32, _vp, _ip, _i32],
    "gvdb2_gather_kernel": [_vp, _i32, _i32, _fp, _ip, _i32, _vp, _i64],
    "gvdb2_gather_kernel_noalloc": [_vp, _i32, _i32, _fp, _ip, _i32, _vp, _i64],
    "gvdb2_scatter_kernel_backward": [_vp, _i32, _i32, _fp, PointsView, _f32, _vp, _i32, _ip, _vp, _vp, _vp],
    "gvdb2_gather_kernel_backward": [_vp, _i32, _i32, _fp, _ip, _i32, _vp, _ip, _vp],
    "gvdb2_set_tuning": [_vp, ctypes.POINTER(Tuning)],
    "gvdb2_get_tuning": [_vp, ctypes.POINTER(Tuning)],
    "gvdb2_set_tune_cache": [_vp, ctypes.c_char_p],
    "gvdb2_autotune_scatter": [_vp, _i32, _i32, _fp, PointsView, _f32, _vp, _ip, _i32, ctypes.POINTER(Tuning)],
    "gvdb2_autotune_gather": [_vp, _i32, _i32, _fp, _ip, _i32, _vp, _i64, ctypes.POINTER(Tuning)],
    "gvdb2_tune_cache_get": [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_float)],
    "gvdb2_tune_cache_put": [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(Tuning), ctypes.c_float],
    "gvdb2_get_info": [_vp, ctypes.POINTER(Info)],
    "gvdb2_copy_nodes": [_vp, _i32, _vp, _i64],
    "gvdb2_copy_childlists": [_vp, _i32, _vp, _i64],
    "gvdb2_copy_atlas": [_vp, _i32, _vp, _i64],
    "gvdb2_copy_atlas_map": [_vp, _vp, _i64],
    "gvdb2_copy_neighbors": [_vp, _vp, _i64],
    "gvdb2_copy_point_nodes": [_vp, _vp, _vp, _i64, _vp, _i64],
    "gvdb2_copy_subcells": [_vp, _vp, _vp, _vp, _i64],
    "gvdb2_copy_subcell_points_fp16": [_vp, _vp, _vp, _i64],
    "gvdb2_atlas_device_ptr": [_vp, _i32, ctypes.POINTER(_vp)],
}


def declared_symbols(header=HEADER):
    """Names of every function the public header declares."""
    txt = open(header).read()
    return sorted(set(re.findall(r"GVDB2_API\s+[\w\s\*]*?\b(gvdb2_\w+)\s*\(", txt)))


def lib():
    """Load libgvdb2.so (raises if it is missing or fails to load)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libgvdb2.so not built ({LIB_PATH}); run gvdb-voxels_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGS.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L.gvdb2_last_error.argtypes = [_vp]
    L.gvdb2_last_error.restype = ctypes.c_char_p
    _lib = L
    return L
