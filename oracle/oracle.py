"""ctypes binding of the CPU oracle (oracle/lib/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product path (gvdb-voxels_b200/) never
imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")

KERNEL_TENT1 = 1
KERNEL_CUBIC2 = 2

NODE_DTYPE = np.dtype([
    ("mLev", np.uint8), ("mFlags", np.uint8), ("mPriority", np.uint8), ("pad", np.uint8),
    ("mPos", np.int32, 3), ("mValue", np.int32, 3), ("mVRange", np.float32, 3),
    ("mParent", np.uint64), ("mChildList", np.uint64), ("mMask", np.uint64),
])
assert NODE_DTYPE.itemsize == 64
AMAP_DTYPE = np.dtype([("mPos", np.int32, 3), ("mLeafID", np.int32)])


class _View(ctypes.Structure):
    _fields_ = [("base", ctypes.c_void_p), ("count", ctypes.c_int64),
                ("stride", ctypes.c_int32), ("offset", ctypes.c_int32)]


def build():
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float
        fp = ctypes.POINTER(ctypes.c_float)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        sig = {
            "orc_create": (vp, []),
            "orc_destroy": (None, [vp]),
            "orc_configure": (i32, [vp, i32, i32, i32, i32, i32]),
            "orc_set_channel_default": (i32, [vp, i32, i32, i32]),
            "orc_add_channel": (i32, [vp, i32, i32]),
            "orc_request_full_rebuild": (None, [vp, i32]),
            "orc_rebuild_topology": (i32, [vp, _View, i32, f32, fp]),
            "orc_accumulate_topology": (i32, [vp, _View, i32, f32, fp, i32]),
            "orc_update_atlas": (i32, [vp]),
            "orc_activate_space": (ctypes.c_uint64, [vp, f32, f32, f32]),
            "orc_activate_points": (i64, [vp, _View, i64, f32, fp]),
            "orc_compute_bounds": (i32, [vp, fp, fp]),
            "orc_root": (ctypes.c_uint64, [vp]),
            "orc_compact_pools": (i32, [vp]),
            "orc_clear_channel": (i32, [vp, i32]),
            "orc_insert_points": (i32, [vp, _View, i32, fp, ip, ip, ip]),
            "orc_scatter_density": (i32, [vp, _View, i32, f32, f32, fp, i32, ip]),
            "orc_update_apron": (i32, [vp, i32, f32]),
            "orc_update_neighbors": (i32, [vp]),
            "orc_update_apron_faces": (i32, [vp, i32]),
            "orc_insert_points_subcell": (i32, [vp, i32, _View, i32, f32, fp, ip]),
            "orc_gather_density": (i32, [vp, i32, f32, i32, i32]),
            "orc_gather_level_set": (i32, [vp, i32, f32, i32, i32]),
            "orc_insert_points_subcell_fp16": (i32, [vp, i32, _View, _View, i32, f32, fp, ip]),
            "orc_gather_level_set_fp16": (i32, [vp, i32, f32, i32]),
            "orc_get_min_max_vel": (i32, [vp, _View, i32]),
            "orc_scatter_kernel": (i32, [vp, i32, _View, i32, fp, _View, f32, vp, ip, i32]),
            "orc_gather_kernel": (i32, [vp, i32, _View, i32, fp, ip, i32, dp]),
            "orc_scatter_kernel_backward": (i32, [vp, i32, _View, i32, fp, _View, f32, vp, ip, i32, ip, dp, dp, dp]),
            "orc_gather_kernel_backward": (i32, [vp, i32, _View, i32, fp, ip, i32, dp, ip, dp]),
            "orc_depth": (i32, [vp]),
            "orc_top_level": (i32, [vp]),
            "orc_pool_count": (i64, [vp, i32]),
            "orc_used_leaves": (i64, [vp]),
            "orc_nodes": (vp, [vp, i32]),
            "orc_childlists": (vp, [vp, i32]),
            "orc_childlist_len": (i64, [vp, i32]),
            "orc_res": (i32, [vp, i32]),
            "orc_range": (i32, [vp, i32]),
            "orc_bbox": (None, [vp, fp, fp]),
            "orc_apron": (i32, [vp]),
            "orc_tile_res": (i32, [vp]),
            "orc_atlas_slots": (i64, [vp]),
            "orc_atlas_capacity": (i64, [vp]),
            "orc_atlas_subdim": (None, [vp, ip]),
            "orc_atlas": (vp, [vp, i32]),
            "orc_atlas_map": (vp, [vp]),
            "orc_neighbors": (vp, [vp]),
            "orc_subcell_count": (i64, [vp]),
            "orc_subcell_cnt": (vp, [vp]),
            "orc_subcell_nid": (vp, [vp]),
            "orc_subcell_pos": (vp, [vp]),
            "orc_subcell_off": (vp, [vp]),
            "orc_subcell_len": (i64, [vp]),
            "orc_subcell_points": (vp, [vp]),
            "orc_subcell_points_fp16": (vp, [vp]),
            "orc_subcell_vel_fp16": (vp, [vp]),
            "orc_leaf_of_point": (i64, [vp, f32, f32, f32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _f3(t):
    a = (ctypes.c_float * 3)(*[float(x) for x in t])
    return a


def view(arr, comp=0, ncomp=None):
    """AoS view of a C-contiguous float32 array: element i at row i, column comp."""
    if arr is None:
        return _View(None, 0, 0, 0)
    assert arr.dtype == np.float32 and arr.flags["C_CONTIGUOUS"]
    stride = arr.strides[0] if arr.ndim > 1 else 4
    return _View(arr.ctypes.data, arr.shape[0], stride, 4 * comp)


class OracleError(RuntimeError):
    pass


def _check(st, what):
    if st != 0:
        raise OracleError(f"{what} failed with status {st}")


class Oracle:
    """CPU restatement of VolumeGVDB's point path (see gvdb_oracle.h)."""

    def __init__(self):
        self.L = lib()
        self.h = self.L.orc_create()
        self._keep = []

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- set-up -------------------------------------------------------
    def configure(self, q4, q3, q2, q1, q0):
        _check(self.L.orc_configure(self.h, q4, q3, q2, q1, q0), "configure")

    def set_channel_default(self, cx, cy, cz):
        _check(self.L.orc_set_channel_default(self.h, cx, cy, cz), "set_channel_default")

    def add_channel(self, chan, apron=1):
        _check(self.L.orc_add_channel(self.h, chan, apron), "add_channel")

    def request_full_rebuild(self, flag=True):
        self.L.orc_request_full_rebuild(self.h, 1 if flag else 0)

    # --- topology -----------------------------------------------------
    def rebuild_topology(self, pos, radius, orig=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        return self.L.orc_rebuild_topology(self.h, view(pos), pos.shape[0], float(radius), _f3(orig))

    def accumulate_topology(self, pos, radius, orig=(0, 0, 0), min_depth=0):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        return self.L.orc_accumulate_topology(self.h, view(pos), pos.shape[0], float(radius), _f3(orig), min_depth)

    def activate_space(self, x, y, z):
        """ActivateSpace(Vector3DF): the leaf's pool reference when it existed,
        ID_UNDEFL (0xFFFFFFFF) when it was created or nothing was activated."""
        return int(self.L.orc_activate_space(self.h, float(x), float(y), float(z)))

    def activate_points(self, pos, radius, orig=(0, 0, 0)):
        """The reference's host topology path: ActivateSpace at every leaf
        brick of each point's activation box, in point order.  Returns the
        number of ActivateSpace calls."""
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        calls = int(self.L.orc_activate_points(self.h, view(pos), pos.shape[0], float(radius), _f3(orig)))
        if calls < 0:
            raise OracleError("activate_points: a tree walk failed")
        return calls

    def compute_bounds(self):
        """ComputeBounds: (mVoxMin, mVoxMax) as float32 arrays."""
        lo = np.zeros(3, np.float32)
        hi = np.zeros(3, np.float32)
        fpp = ctypes.POINTER(ctypes.c_float)
        if self.L.orc_compute_bounds(self.h, lo.ctypes.data_as(fpp), hi.ctypes.data_as(fpp)) != 0:
            raise OracleError("compute_bounds: no leaf")
        return lo, hi

    def root(self):
        return int(self.L.orc_root(self.h))

    def compact_pools(self):
        _check(self.L.orc_compact_pools(self.h), "compact_pools")

    def update_atlas(self):
        _check(self.L.orc_update_atlas(self.h), "update_atlas")

    def clear_channel(self, chan):
        _check(self.L.orc_clear_channel(self.h, chan), "clear_channel")

    # --- points -------------------------------------------------------
    def insert_points(self, pos, trans=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        n = pos.shape[0]
        pnode = np.empty(n, np.int32)
        poff = np.zeros(n, np.int32)
        gcnt = np.zeros(max(1, self.pool_count(0)), np.int32)
        ip = ctypes.POINTER(ctypes.c_int32)
        _check(self.L.orc_insert_points(self.h, view(pos), n, _f3(trans), pnode.ctypes.data_as(ip),
                                        poff.ctypes.data_as(ip), gcnt.ctypes.data_as(ip)), "insert_points")
        return pnode, poff, gcnt[:self.pool_count(0)]

    def scatter_density(self, pos, radius, amp, trans, expand, pnode):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        pnode = np.ascontiguousarray(pnode, dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int32)
        _check(self.L.orc_scatter_density(self.h, view(pos), pos.shape[0], float(radius), float(amp), _f3(trans),
                                          1 if expand else 0, pnode.ctypes.data_as(ip)), "scatter_density")

    def update_apron(self, chan, boundval=0.0):
        _check(self.L.orc_update_apron(self.h, chan, float(boundval)), "update_apron")

    def update_neighbors(self):
        _check(self.L.orc_update_neighbors(self.h), "update_neighbors")

    def update_apron_faces(self, chan):
        _check(self.L.orc_update_apron_faces(self.h, chan), "update_apron_faces")

    def insert_points_subcell(self, sc, pos, radius, trans=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        ln = ctypes.c_int32(0)
        _check(self.L.orc_insert_points_subcell(self.h, sc, view(pos), pos.shape[0], float(radius), _f3(trans),
                                                ctypes.byref(ln)), "insert_points_subcell")
        return ln.value

    def gather_density(self, sc, radius, chan, accum=False):
        _check(self.L.orc_gather_density(self.h, sc, float(radius), chan, 1 if accum else 0), "gather_density")

    def gather_level_set(self, sc, radius, chan, accum=False):
        _check(self.L.orc_gather_level_set(self.h, sc, float(radius), chan, 1 if accum else 0), "gather_level_set")

    def insert_points_subcell_fp16(self, sc, pos, radius, trans=(0, 0, 0), vel=None):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        vv = _View(None, 0, 0, 0)
        if vel is not None:
            vel = np.ascontiguousarray(vel, dtype=np.float32)
            vv = view(vel)
        ln = ctypes.c_int32(0)
        _check(self.L.orc_insert_points_subcell_fp16(self.h, sc, view(pos), vv, pos.shape[0], float(radius),
                                                     _f3(trans), ctypes.byref(ln)), "insert_points_subcell_fp16")
        return ln.value

    def gather_level_set_fp16(self, sc, radius, chan):
        _check(self.L.orc_gather_level_set_fp16(self.h, sc, float(radius), chan), "gather_level_set_fp16")

    def get_min_max_vel(self, vel):
        vel = np.ascontiguousarray(vel, dtype=np.float32)
        _check(self.L.orc_get_min_max_vel(self.h, view(vel), vel.shape[0]), "get_min_max_vel")

    def _attr_views(self, attrs, nch):
        arr = (_View * nch)()
        keep = []
        for c in range(nch):
            a = None if attrs is None else attrs[c]
            if a is None:
                arr[c] = _View(None, 0, 0, 0)
            else:
                a = np.ascontiguousarray(a, dtype=np.float32)
                keep.append(a)
                arr[c] = view(a)
        return arr, keep

    def scatter_kernel(self, kernel, pos, chans, weight=None, weight_const=1.0, attrs=None, trans=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        chans = np.ascontiguousarray(chans, dtype=np.int32)
        nch = len(chans)
        av, keep = self._attr_views(attrs, nch)
        w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float32)
        _check(self.L.orc_scatter_kernel(self.h, kernel, view(pos), pos.shape[0], _f3(trans), view(w),
                                         float(weight_const), ctypes.cast(av, ctypes.c_void_p),
                                         chans.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nch), "scatter_kernel")

    def gather_kernel(self, kernel, pos, chans, trans=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        chans = np.ascontiguousarray(chans, dtype=np.int32)
        out = np.zeros((pos.shape[0], len(chans)), np.float64)
        _check(self.L.orc_gather_kernel(self.h, kernel, view(pos), pos.shape[0], _f3(trans),
                                        chans.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(chans),
                                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "gather_kernel")
        return out

    def scatter_kernel_backward(self, kernel, pos, chans, grad_chans, weight=None, weight_const=1.0, attrs=None,
                                trans=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        n = pos.shape[0]
        chans = np.ascontiguousarray(chans, dtype=np.int32)
        gch = np.ascontiguousarray(grad_chans, dtype=np.int32)
        nch = len(chans)
        av, keep = self._attr_views(attrs, nch)
        w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float32)
        gpos = np.zeros((n, 3), np.float64)
        gw = np.zeros(n, np.float64)
        ga = np.zeros((n, nch), np.float64)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        _check(self.L.orc_scatter_kernel_backward(self.h, kernel, view(pos), n, _f3(trans), view(w), float(weight_const),
                                                  ctypes.cast(av, ctypes.c_void_p), chans.ctypes.data_as(ip), nch,
                                                  gch.ctypes.data_as(ip), gpos.ctypes.data_as(dp),
                                                  gw.ctypes.data_as(dp), ga.ctypes.data_as(dp)),
               "scatter_kernel_backward")
        return gpos, gw, ga

    def gather_kernel_backward(self, kernel, pos, chans, grad_out, grad_chans=None, trans=(0, 0, 0)):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        n = pos.shape[0]
        chans = np.ascontiguousarray(chans, dtype=np.int32)
        go = np.ascontiguousarray(grad_out, dtype=np.float64).reshape(n, len(chans))
        gpos = np.zeros((n, 3), np.float64)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        gch = None if grad_chans is None else np.ascontiguousarray(grad_chans, dtype=np.int32)
        _check(self.L.orc_gather_kernel_backward(self.h, kernel, view(pos), n, _f3(trans), chans.ctypes.data_as(ip),
                                                 len(chans), go.ctypes.data_as(dp),
                                                 None if gch is None else gch.ctypes.data_as(ip),
                                                 gpos.ctypes.data_as(dp)), "gather_kernel_backward")
        return gpos

    # --- inspection ---------------------------------------------------
    def depth(self):
        return self.L.orc_depth(self.h)

    def top_level(self):
        return self.L.orc_top_level(self.h)

    def pool_count(self, lev):
        return int(self.L.orc_pool_count(self.h, lev))

    def used_leaves(self):
        return int(self.L.orc_used_leaves(self.h))

    def nodes(self, lev):
        n = self.pool_count(lev)
        if n == 0:
            return np.zeros(0, NODE_DTYPE)
        ptr = self.L.orc_nodes(self.h, lev)
        buf = (ctypes.c_char * (n * 64)).from_address(ptr)
        return np.frombuffer(buf, NODE_DTYPE, n).copy()

    def childlists(self, lev):
        n = self.pool_count(lev)
        ln = int(self.L.orc_childlist_len(self.h, lev))
        if n == 0 or ln == 0:
            return np.zeros((0, ln), np.uint64)
        ptr = self.L.orc_childlists(self.h, lev)
        buf = (ctypes.c_char * (n * ln * 8)).from_address(ptr)
        return np.frombuffer(buf, np.uint64, n * ln).reshape(n, ln).copy()

    def res(self, lev):
        return self.L.orc_res(self.h, lev)

    def range(self, lev):
        return self.L.orc_range(self.h, lev)

    def bbox(self):
        a = (ctypes.c_float * 3)()
        b = (ctypes.c_float * 3)()
        self.L.orc_bbox(self.h, a, b)
        return np.array(a[:], np.float32), np.array(b[:], np.float32)

    def apron(self):
        return self.L.orc_apron(self.h)

    def tile_res(self):
        return self.L.orc_tile_res(self.h)

    def atlas_slots(self):
        return int(self.L.orc_atlas_slots(self.h))

    def atlas_subdim(self):
        a = (ctypes.c_int32 * 3)()
        self.L.orc_atlas_subdim(self.h, a)
        return tuple(a[:])

    def atlas(self, chan):
        """Channel data of the used slots, shape (slots, T, T, T) as (z,y,x), float64."""
        s = self.atlas_slots()
        t = self.tile_res()
        ptr = self.L.orc_atlas(self.h, chan)
        if s == 0 or not ptr:
            return np.zeros((0, t, t, t))
        buf = (ctypes.c_char * (s * t * t * t * 8)).from_address(ptr)
        return np.frombuffer(buf, np.float64, s * t ** 3).reshape(s, t, t, t).copy()

    def atlas_map(self):
        s = int(self.L.orc_atlas_capacity(self.h))
        ptr = self.L.orc_atlas_map(self.h)
        if not ptr:
            return np.zeros(0, AMAP_DTYPE)
        buf = (ctypes.c_char * (s * 16)).from_address(ptr)
        return np.frombuffer(buf, AMAP_DTYPE, s).copy()

    def neighbors(self):
        n = self.pool_count(0)
        ptr = self.L.orc_neighbors(self.h)
        buf = (ctypes.c_char * (n * 6 * 4)).from_address(ptr)
        return np.frombuffer(buf, np.int32, n * 6).reshape(n, 6).copy()

    def subcells(self):
        m = int(self.L.orc_subcell_count(self.h))

        def arr(ptr, cnt):
            buf = (ctypes.c_char * (cnt * 4)).from_address(ptr)
            return np.frombuffer(buf, np.int32, cnt).copy()
        return (arr(self.L.orc_subcell_cnt(self.h), m), arr(self.L.orc_subcell_nid(self.h), m),
                arr(self.L.orc_subcell_pos(self.h), 3 * m).reshape(m, 3))

    def subcell_lists(self):
        """Offsets per subcell and the list entries: float xyz, or quantized
        (uint16 xyz, uint16 velocity or None) after an FP16 insert."""
        m = int(self.L.orc_subcell_count(self.h))
        ln = int(self.L.orc_subcell_len(self.h))
        off = np.frombuffer((ctypes.c_char * (4 * m)).from_address(self.L.orc_subcell_off(self.h)), np.int32).copy()

        def arr(ptr, dtype, width):
            if not ptr or ln == 0:
                return None
            n = ln * 3
            return np.frombuffer((ctypes.c_char * (n * width)).from_address(ptr), dtype, n).copy().reshape(ln, 3)
        pts = arr(self.L.orc_subcell_points(self.h), np.float32, 4)
        if pts is not None:
            return off, pts
        return off, arr(self.L.orc_subcell_points_fp16(self.h), np.uint16, 2), \
            arr(self.L.orc_subcell_vel_fp16(self.h), np.uint16, 2)

    def leaf_of_point(self, x, y, z):
        return int(self.L.orc_leaf_of_point(self.h, x, y, z))
