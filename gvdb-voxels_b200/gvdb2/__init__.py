"""gvdb2 -- host-side mirror of nvdb::VolumeGVDB's point path over libgvdb2.

Method names, argument order and meaning follow VolumeGVDB
(source/gvdb_library/src/gvdb_volume_gvdb.h:325-562); errors raise
GvdbError instead of printing and returning.  Point data are CUDA tensors
(the SetDataGPU contract): float32 rows of 3 for positions, or any float32
column of a 2-D tensor for per-point attributes.  PyTorch only supplies
device memory and streams; all work runs in libgvdb2's CUDA kernels.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import (KERNEL_CUBIC2, KERNEL_TENT1, NV_FLOAT, NV_VEC3F, OPT_AUTOTUNE, OPT_DETERMINISTIC, T_FLOAT, GvdbError,
                   Info, PointsView, Tuning, declared_symbols)

NODE_DTYPE = np.dtype([
    ("mLev", np.uint8), ("mFlags", np.uint8), ("mPriority", np.uint8), ("pad", np.uint8),
    ("mPos", np.int32, 3), ("mValue", np.int32, 3), ("mVRange", np.float32, 3),
    ("mParent", np.uint64), ("mChildList", np.uint64), ("mMask", np.uint64),
])
AMAP_DTYPE = np.dtype([("mPos", np.int32, 3), ("mLeafID", np.int32)])
ID_UNDEFL = 0xFFFFFFFF  # gvdb_types.h:55: no node

__all__ = ["VolumeGVDB", "GvdbError", "KERNEL_TENT1", "KERNEL_CUBIC2", "T_FLOAT", "NODE_DTYPE", "AMAP_DTYPE", "ID_UNDEFL",
           "view_of", "declared_symbols"]


def _f3(t):
    return (ctypes.c_float * 3)(*[float(x) for x in t])


def view_of(t, col=None):
    """PointsView of a CUDA float32 tensor: rows of a (N,3) tensor, or column
    `col` of a 2-D tensor, or a 1-D tensor."""
    if t is None:
        return PointsView(None, 0, 0, 0)
    if hasattr(t, "data_ptr"):
        assert t.is_cuda and str(t.dtype) == "torch.float32", "point data must be float32 CUDA tensors"
        es = t.element_size()
        if t.dim() == 1:
            return PointsView(t.data_ptr(), t.shape[0], t.stride(0) * es, 0)
        off = 0 if col is None else col * t.stride(1) * es
        return PointsView(t.data_ptr() + off, t.shape[0], t.stride(0) * es, 0)
    raise TypeError("expected a CUDA tensor")


class VolumeGVDB:
    """One sparse volume on one GPU (VolumeGVDB, gvdb_volume_gvdb.h:319-901)."""

    def __init__(self, device=0):
        self._L = _lib.lib()
        h = ctypes.c_void_p()
        self._check(self._L.gvdb2_create(ctypes.byref(h), int(device)), "SetCudaDevice", handle=False)
        self._h = h
        self._keep = {}
        self.device = device

    # -- plumbing -------------------------------------------------------
    def _check(self, st, what, handle=True):
        if st != _lib.OK:
            msg = self._L.gvdb2_last_error(self._h).decode() if handle and getattr(self, "_h", None) else ""
            raise GvdbError(st, what, msg)

    def close(self):
        if getattr(self, "_h", None):
            self._L.gvdb2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def SetStream(self, stream):
        ptr = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream or 0)
        self._check(self._L.gvdb2_set_stream(self._h, ctypes.c_void_p(ptr)), "SetStream")

    def Synchronize(self):
        self._check(self._L.gvdb2_synchronize(self._h), "Synchronize")

    def SetDeterministic(self, flag=True):
        self._check(self._L.gvdb2_set_option(self._h, OPT_DETERMINISTIC, 1 if flag else 0), "SetDeterministic")

    def SetAutotune(self, flag=True):
        """GVDB2_OPT_AUTOTUNE: kernel splats and gathers take their workload
        class's setting from the tuning cache when it has one."""
        self._check(self._L.gvdb2_set_option(self._h, OPT_AUTOTUNE, 1 if flag else 0), "SetAutotune")

    # -- configuration (V:2364-2453) -----------------------------------------
    def Initialize(self):
        return None

    def Configure(self, q4, q3, q2, q1, q0):
        self._check(self._L.gvdb2_configure(self._h, q4, q3, q2, q1, q0), "Configure")

    def SetChannelDefault(self, cx, cy, cz):
        self._check(self._L.gvdb2_set_channel_default(self._h, cx, cy, cz), "SetChannelDefault")

    def AddChannel(self, chan, dt=T_FLOAT, apron=1):
        self._check(self._L.gvdb2_add_channel(self._h, chan, dt, apron), "AddChannel")

    # -- points (V:4900-4908) ---------------------------------------------
    def SetPoints(self, pos, vel=None, clr=None):
        self._keep["points"] = (pos, vel, clr)
        self._check(self._L.gvdb2_set_points(self._h, view_of(pos), view_of(vel), view_of(clr)), "SetPoints")

    def BatchPoints(self, clouds, space_log2):
        """Packs several clouds (CUDA (N,3) float32 tensors, each in its own
        [0, 2**space_log2)^3 index space) into this volume's point set.
        Returns numpy int64 first-index offsets (len = clouds + 1); later
        per-point arrays are in that packed order."""
        import numpy as np
        n = len(clouds)
        views = (PointsView * n)(*[view_of(c) for c in clouds])
        first = np.zeros(n + 1, np.int64)
        self._keep["batch"] = (clouds, views)
        self._check(self._L.gvdb2_batch_points(self._h, views, n, int(space_log2),
                                               first.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))), "BatchPoints")
        return first

    def BatchOrigin(self, cloud):
        """Voxel offset of a cloud in the packed batch."""
        o = (ctypes.c_int32 * 3)()
        self._check(self._L.gvdb2_batch_origin(self._h, int(cloud), o), "BatchOrigin")
        return tuple(o[:])

    # -- topology ---------------------------------------------------------
    def RequestFullRebuild(self, flag=True):
        self._check(self._L.gvdb2_request_full_rebuild(self._h, 1 if flag else 0), "RequestFullRebuild")

    def RebuildTopology(self, num_pnts, radius, orig=(0, 0, 0)):
        self._check(self._L.gvdb2_rebuild_topology(self._h, int(num_pnts), float(radius), _f3(orig)),
                    "RebuildTopology")

    def AccumulateTopology(self, num_pnts, radius, orig=(0, 0, 0), iDepth=1):
        self._check(self._L.gvdb2_accumulate_topology(self._h, int(num_pnts), float(radius), _f3(orig), int(iDepth)),
                    "AccumulateTopology")

    def FinishTopology(self, commit=True, bounds=True):
        self._check(self._L.gvdb2_finish_topology(self._h, int(commit), int(bounds)), "FinishTopology")

    def getVolMin(self):
        """gvdb_volume_base.h:57: the bounds of the last FinishTopology(bounds=True)."""
        return tuple(self.info().vol_min)

    def getVolMax(self):
        return tuple(self.info().vol_max)

    def UpdateAtlas(self):
        self._check(self._L.gvdb2_update_atlas(self._h), "UpdateAtlas")

    def ActivateSpace(self, pos):
        """ActivateSpace(Vector3DF) (V:2766-2856) for one (x, y, z) or an (N, 3)
        host array of positions, in order: the leaf's pool reference where it
        existed, ID_UNDEFL where the call created it (or could not activate
        it).  Returns an int for one position, else a uint64 numpy array."""
        import numpy as np
        p = np.ascontiguousarray(pos, dtype=np.float32)
        one = p.ndim == 1
        p = p.reshape(-1, 3)
        out = np.empty(len(p), np.uint64)
        self._check(self._L.gvdb2_activate_space(self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), len(p),
                                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))), "ActivateSpace")
        return int(out[0]) if one else out

    def CompactPools(self):
        """Drop the nodes incremental rebuilds delinked and renumber the rest
        (no reference counterpart); call UpdateAtlas before the next splat."""
        self._check(self._L.gvdb2_compact_pools(self._h), "CompactPools")

    def ClearChannel(self, chan):
        self._check(self._L.gvdb2_clear_channel(self._h, chan), "ClearChannel")

    def UpdateNeighbors(self):
        self._check(self._L.gvdb2_update_neighbors(self._h), "UpdateNeighbors")

    # -- insertion ----------------------------------------------------------
    def InsertPoints(self, num_pnts, trans=(0, 0, 0), prefix=False):
        self._check(self._L.gvdb2_insert_points(self._h, int(num_pnts), _f3(trans), 1 if prefix else 0),
                    "InsertPoints")

    def InsertPointsSubcell(self, subcell_size, num_pnts, radius, trans=(0, 0, 0)):
        ln = ctypes.c_int(0)
        self._check(self._L.gvdb2_insert_points_subcell(self._h, subcell_size, int(num_pnts), float(radius),
                                                        _f3(trans), ctypes.byref(ln)), "InsertPointsSubcell")
        return ln.value

    # -- reference-mode splat / gathers / apron -------------------------------
    def ScatterDensity(self, num_pnts, radius, amp, trans=(0, 0, 0), expand=True, avgColor=False):
        self._check(self._L.gvdb2_scatter_density(self._h, int(num_pnts), float(radius), float(amp), _f3(trans),
                                                  1 if expand else 0, 1 if avgColor else 0), "ScatterDensity")

    def SetTransform(self, pretrans, scale, angs, trans):
        """Grid transform (SetTransform, V:5770); stored in VBX files."""
        self._check(self._L.gvdb2_set_transform(self._h, _f3(pretrans), _f3(scale), _f3(angs), _f3(trans)),
                    "SetTransform")

    def GetTransform(self):
        """(pretrans, scale, angs, trans) as tuples."""
        parts = [(ctypes.c_float * 3)() for _ in range(4)]
        self._check(self._L.gvdb2_get_transform(self._h, *parts), "GetTransform")
        return tuple(tuple(float(x) for x in p) for p in parts)

    def SaveVBX(self, fname):
        """Writes the volume as a VBX file (V:1626-1768)."""
        self._check(self._L.gvdb2_save_vbx(self._h, os.fsencode(fname)), "SaveVBX")

    def LoadVBX(self, fname):
        """Replaces the volume with a VBX file's (V:507-685)."""
        self._check(self._L.gvdb2_load_vbx(self._h, os.fsencode(fname)), "LoadVBX")

    def ExportToNanoVDB(self, chans, background=0.0, grid_name="", grid_class=0):
        """The volume as one NanoVDB-form device buffer (ExportToNanoVDB,
        gNanoVDB/gvdb_export_nanovdb.cpp:379-700): a uint8 torch tensor on
        the volume's device, laid out as gvdb2_nv_* in include/gvdb2.h.  One
        channel gives a float grid, three channels (x, y, z) a Vec3f grid."""
        import torch
        chans = [int(c) for c in chans]
        nv = {1: NV_FLOAT, 3: NV_VEC3F}.get(len(chans))
        if nv is None:
            raise GvdbError(1, "ExportToNanoVDB", "one or three channels")
        bg = [float(b) for b in np.broadcast_to(np.asarray(background, np.float32), (len(chans),))]
        size = ctypes.c_size_t()
        self._check(self._L.gvdb2_nanovdb_size(self._h, nv, ctypes.byref(size)), "ExportToNanoVDB")
        out = torch.empty(max(int(size.value), 1), dtype=torch.uint8, device=f"cuda:{self.device}")
        self._check(self._L.gvdb2_export_nanovdb(self._h, nv, (ctypes.c_int * len(chans))(*chans),
                                                 (ctypes.c_float * len(bg))(*bg), os.fsencode(grid_name),
                                                 int(grid_class), ctypes.c_void_p(out.data_ptr()), int(size.value)),
                    "ExportToNanoVDB")
        return out[:int(size.value)]

    def InsertPointsSubcell_FP16(self, subcell_size, num_pnts, radius, trans=(0, 0, 0)):
        """InsertPointsSubcell with 16-bit list entries (V:5094-5189); returns the list length."""
        ln = ctypes.c_int(0)
        self._check(self._L.gvdb2_insert_points_subcell_fp16(self._h, subcell_size, int(num_pnts), float(radius),
                                                             _f3(trans), ctypes.byref(ln)), "InsertPointsSubcell_FP16")
        return ln.value

    def GetMinMaxVel(self, num_pnts):
        """Velocity range used to quantize the 16-bit velocity lists (V:5469-5521)."""
        self._check(self._L.gvdb2_get_min_max_vel(self._h, int(num_pnts)), "GetMinMaxVel")

    def GatherLevelSet_FP16(self, subcell_size, num_pnts, radius, trans, sc_len, chanLevelset, chanClr=-1):
        ln = ctypes.c_int(int(sc_len))
        self._check(self._L.gvdb2_gather_level_set_fp16(self._h, subcell_size, int(num_pnts), float(radius),
                                                        _f3(trans), ctypes.byref(ln), chanLevelset, chanClr),
                    "GatherLevelSet_FP16")

    def _gather(self, fn, what, subcell_size, num_pnts, radius, trans, sc_len, chan, chan_clr, accum):
        ln = ctypes.c_int(int(sc_len))
        self._check(fn(self._h, subcell_size, int(num_pnts), float(radius), _f3(trans), ctypes.byref(ln), chan,
                       chan_clr, 1 if accum else 0), what)

    def GatherDensity(self, subcell_size, num_pnts, radius, trans, sc_len, chanDensity, chanClr=-1, bAccum=False):
        self._gather(self._L.gvdb2_gather_density, "GatherDensity", subcell_size, num_pnts, radius, trans, sc_len,
                     chanDensity, chanClr, bAccum)

    def GatherLevelSet(self, subcell_size, num_pnts, radius, trans, sc_len, chanLevelset, chanClr=-1, bAccum=False):
        self._gather(self._L.gvdb2_gather_level_set, "GatherLevelSet", subcell_size, num_pnts, radius, trans, sc_len,
                     chanLevelset, chanClr, bAccum)

    def ScatterReduceLevelSet(self, subcell_size, num_pnts, radius, trans, sc_len, chanLevelset, chanClr=-1,
                              bAccum=False):
        self._gather(self._L.gvdb2_scatter_reduce_level_set, "ScatterReduceLevelSet", subcell_size, num_pnts,
                     radius, trans, sc_len, chanLevelset, chanClr, bAccum)

    def UpdateApron(self, chan=-1, boundval=0.0):
        self._check(self._L.gvdb2_update_apron(self._h, int(chan), float(boundval)), "UpdateApron")

    def UpdateApronFaces(self, chan):
        self._check(self._L.gvdb2_update_apron_faces(self._h, int(chan)), "UpdateApronFaces")

    # -- kernel splats and adjoints ----------------------------------------
    @staticmethod
    def _attr_array(attrs, nch):
        arr = (PointsView * max(nch, 1))()
        for c in range(nch):
            a = None if attrs is None else attrs[c]
            if a is None:
                arr[c] = PointsView(None, 0, 0, 0)
            elif isinstance(a, tuple):
                arr[c] = view_of(a[0], a[1])
            else:
                arr[c] = view_of(a)
        return arr

    @staticmethod
    def _chans(chans):
        return (ctypes.c_int * len(chans))(*[int(c) for c in chans])

    def ScatterKernel(self, kernel, num_pnts, chans, weight=1.0, attrs=None, trans=(0, 0, 0)):
        """channel chans[c] := sum_p weight_p * attr_c(p) * W(v + 0.5 - x_p)."""
        wv = view_of(weight) if hasattr(weight, "data_ptr") else PointsView(None, 0, 0, 0)
        wc = 1.0 if hasattr(weight, "data_ptr") else float(weight)
        av = self._attr_array(attrs, len(chans))
        self._keep["scatter"] = (weight, attrs, av)
        self._check(self._L.gvdb2_scatter_kernel(self._h, kernel, int(num_pnts), _f3(trans), wv, wc,
                                                 ctypes.cast(av, ctypes.c_void_p), self._chans(chans), len(chans)),
                    "ScatterKernel")

    def GatherKernel(self, kernel, num_pnts, chans, out=None, trans=(0, 0, 0)):
        """out[p, c] := sum_v G_chans[c][v] * W(v + 0.5 - x_p); returns out."""
        import torch
        if out is None:
            out = torch.empty((int(num_pnts), len(chans)), dtype=torch.float32, device=f"cuda:{self.device}")
        self._check(self._L.gvdb2_gather_kernel(self._h, kernel, int(num_pnts), _f3(trans), self._chans(chans),
                                                len(chans), ctypes.c_void_p(out.data_ptr()), out.stride(0)),
                    "GatherKernel")
        return out

    def SetTuning(self, dense=512, slice=4096, light=32):
        """Launch settings of the kernel splats (gvdb2_tuning)."""
        t = Tuning(int(dense), int(slice), int(light))
        self._check(self._L.gvdb2_set_tuning(self._h, ctypes.byref(t)), "SetTuning")

    def GetTuning(self):
        t = Tuning()
        self._check(self._L.gvdb2_get_tuning(self._h, ctypes.byref(t)), "GetTuning")
        return (t.dense, t.slice, t.light)

    def SetTuneCache(self, path):
        self._check(self._L.gvdb2_set_tune_cache(self._h, os.fsencode(path) if path else None), "SetTuneCache")

    def AutotuneScatter(self, kernel, num_pnts, chans, weight=1.0, attrs=None, trans=(0, 0, 0)):
        """ScatterKernel that times the scatter's candidate settings on this
        call, keeps the fastest and caches it; returns (dense, slice, light)."""
        wv = view_of(weight) if hasattr(weight, "data_ptr") else PointsView(None, 0, 0, 0)
        wc = 1.0 if hasattr(weight, "data_ptr") else float(weight)
        av = self._attr_array(attrs, len(chans))
        self._keep["scatter"] = (weight, attrs, av)
        t = Tuning()
        self._check(self._L.gvdb2_autotune_scatter(self._h, kernel, int(num_pnts), _f3(trans), wv, wc,
                                                   ctypes.cast(av, ctypes.c_void_p), self._chans(chans), len(chans),
                                                   ctypes.byref(t)), "AutotuneScatter")
        return (t.dense, t.slice, t.light)

    def AutotuneGather(self, kernel, num_pnts, chans, out=None, trans=(0, 0, 0)):
        """GatherKernel that times the gather's candidate settings on this
        call, keeps the fastest and caches it; returns (out, tuning)."""
        import torch
        if out is None:
            out = torch.empty((int(num_pnts), len(chans)), dtype=torch.float32, device=f"cuda:{self.device}")
        t = Tuning()
        self._check(self._L.gvdb2_autotune_gather(self._h, kernel, int(num_pnts), _f3(trans), self._chans(chans),
                                                  len(chans), ctypes.c_void_p(out.data_ptr()), out.stride(0),
                                                  ctypes.byref(t)), "AutotuneGather")
        return out, (t.dense, t.slice, t.light)

    def GatherKernelNoAlloc(self, kernel, num_pnts, chans, out, trans=(0, 0, 0)):
        """GatherKernel for callers that cannot allocate device memory once
        running: no device allocation at all (binning scratch is a fixed
        12.25 MiB array per GPU; at most 1,048,576 points and 32,768 active
        8^3 cells per call: bricks of 8^3 voxels, or an eighth as many of 16^3).  `out` is a caller-owned (N, nch) float32 CUDA
        tensor.  Calls whose GPU work overlaps share the scratch and race."""
        self._check(self._L.gvdb2_gather_kernel_noalloc(self._h, kernel, int(num_pnts), _f3(trans), self._chans(chans),
                                                        len(chans), ctypes.c_void_p(out.data_ptr()), out.stride(0)),
                    "GatherKernelNoAlloc")
        return out

    def ScatterDensityBackward(self, kernel, num_pnts, grad_chans, weight=1.0, attrs=None, trans=(0, 0, 0),
                               grad_pos=None, grad_weight=None, grad_attr=None):
        """Adjoint of ScatterKernel: from dL/dG in channels grad_chans, per-point
        dL/dpos (N,3), dL/dweight (N,) and dL/dattr (N,nch)."""
        import torch
        n, nch = int(num_pnts), len(grad_chans)
        dev = f"cuda:{self.device}"
        grad_pos = torch.empty((n, 3), dtype=torch.float32, device=dev) if grad_pos is None else grad_pos
        grad_weight = torch.empty((n,), dtype=torch.float32, device=dev) if grad_weight is None else grad_weight
        grad_attr = torch.empty((n, nch), dtype=torch.float32, device=dev) if grad_attr is None else grad_attr
        wv = view_of(weight) if hasattr(weight, "data_ptr") else PointsView(None, 0, 0, 0)
        wc = 1.0 if hasattr(weight, "data_ptr") else float(weight)
        av = self._attr_array(attrs, nch)
        self._check(self._L.gvdb2_scatter_kernel_backward(
            self._h, kernel, n, _f3(trans), wv, wc, ctypes.cast(av, ctypes.c_void_p), nch, self._chans(grad_chans),
            ctypes.c_void_p(grad_pos.data_ptr()), ctypes.c_void_p(grad_weight.data_ptr()),
            ctypes.c_void_p(grad_attr.data_ptr())), "ScatterDensityBackward")
        return grad_pos, grad_weight, grad_attr

    def GatherDensityBackward(self, kernel, num_pnts, chans, grad_out, grad_chans=None, trans=(0, 0, 0),
                              grad_pos=None):
        """Adjoint of GatherKernel: from dL/dout (N,nch), sets channels grad_chans
        to dL/dG (if given) and returns dL/dpos (N,3)."""
        import torch
        n = int(num_pnts)
        grad_out = grad_out.contiguous()
        grad_pos = torch.empty((n, 3), dtype=torch.float32, device=f"cuda:{self.device}") if grad_pos is None else grad_pos
        gch = None if grad_chans is None else self._chans(grad_chans)
        self._check(self._L.gvdb2_gather_kernel_backward(
            self._h, kernel, n, _f3(trans), self._chans(chans), len(chans), ctypes.c_void_p(grad_out.data_ptr()),
            gch, ctypes.c_void_p(grad_pos.data_ptr())), "GatherDensityBackward")
        return grad_pos

    # -- inspection ----------------------------------------------------------
    def info(self):
        inf = Info()
        self._check(self._L.gvdb2_get_info(self._h, ctypes.byref(inf)), "info")
        return inf

    def getNumTotalNodes(self, lev):
        return int(self.info().pool_count[lev])

    def getNumUsedNodes(self, lev):
        inf = self.info()
        return int(inf.used_leaves) if lev == 0 else int(inf.pool_count[lev])

    def nodes(self, lev):
        n = self.getNumTotalNodes(lev)
        out = np.zeros(n, NODE_DTYPE)
        if n:
            self._check(self._L.gvdb2_copy_nodes(self._h, lev, out.ctypes.data, n), "copy_nodes")
        return out

    def childlists(self, lev):
        inf = self.info()
        n = int(inf.pool_count[lev])
        r3 = int(inf.res[lev]) ** 3
        out = np.zeros((n, r3), np.uint64)
        if n:
            self._check(self._L.gvdb2_copy_childlists(self._h, lev, out.ctypes.data, n * r3), "copy_childlists")
        return out

    def atlas(self, chan):
        """Used slots' tiles of a channel, shape (slots, T, T, T) as (z, y, x)."""
        inf = self.info()
        s, t = int(inf.atlas_slots), int(inf.tile_res)
        out = np.zeros((s, t, t, t), np.float32)
        if s:
            self._check(self._L.gvdb2_copy_atlas(self._h, chan, out.ctypes.data, out.size), "copy_atlas")
        return out

    def atlas_map(self):
        n = int(self.info().atlas_capacity)
        out = np.zeros(n, AMAP_DTYPE)
        if n:
            self._check(self._L.gvdb2_copy_atlas_map(self._h, out.ctypes.data, n), "copy_atlas_map")
        return out

    def neighbors(self):
        n = self.getNumTotalNodes(0)
        out = np.zeros((n, 6), np.int32)
        if n:
            self._check(self._L.gvdb2_copy_neighbors(self._h, out.ctypes.data, 6 * n), "copy_neighbors")
        return out

    def point_nodes(self, num_pnts):
        n = int(num_pnts)
        nl = self.getNumTotalNodes(0)
        pnode = np.zeros(n, np.int32)
        poff = np.zeros(n, np.int32)
        gcnt = np.zeros(nl, np.int32)
        self._check(self._L.gvdb2_copy_point_nodes(self._h, pnode.ctypes.data, poff.ctypes.data, n,
                                                   gcnt.ctypes.data, nl), "copy_point_nodes")
        return pnode, poff, gcnt

    def subcell_points_fp16(self, length, vel=False):
        """The 16-bit list entries, (length, 3) uint16 (and velocities)."""
        import numpy as np
        q = np.zeros((max(length, 1), 3), np.uint16)
        qv = np.zeros((max(length, 1), 3), np.uint16) if vel else None
        self._check(self._L.gvdb2_copy_subcell_points_fp16(self._h, q.ctypes.data,
                                                           qv.ctypes.data if vel else None, int(length)),
                    "copy_subcell_points_fp16")
        return (q[:length], qv[:length]) if vel else q[:length]

    def subcells(self, count):
        cnt = np.zeros(count, np.int32)
        nid = np.zeros(count, np.int32)
        pos = np.zeros((count, 3), np.int32)
        self._check(self._L.gvdb2_copy_subcells(self._h, cnt.ctypes.data, nid.ctypes.data, pos.ctypes.data, count),
                    "copy_subcells")
        return cnt, nid, pos

    def atlas_tensor(self, chan):
        """Zero-copy torch view of a channel's used tiles, (slots, T, T, T)."""
        inf = self.info()
        ptr = ctypes.c_void_p()
        self._check(self._L.gvdb2_atlas_device_ptr(self._h, chan, ctypes.byref(ptr)), "atlas_device_ptr")
        s, t = int(inf.atlas_slots), int(inf.tile_res)
        return _wrap_device(ptr.value, (s, t, t, t), self.device)


def _wrap_device(ptr, shape, device):
    """Non-owning torch view of device memory (via the CUDA array interface)."""
    import torch

    class _Holder:
        pass
    h = _Holder()
    n = int(np.prod(shape))
    h.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}
    return torch.as_tensor(h, device=f"cuda:{device}").view(*shape)
