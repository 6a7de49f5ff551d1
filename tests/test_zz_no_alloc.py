"""gvdb2_gather_kernel_noalloc: the grid -> point gather for callers that
cannot allocate device memory once they are running (an application that
fixes its GPU memory budget at start-up, a real-time loop that forbids
allocation, an allocator owned by another framework).  Its binning scratch
is a fixed per-GPU device array, so it must give the same answer as
gvdb2_gather_kernel -- here on two calls in a row, the second with a
different point set, so stale scratch from the first call would show."""
import ctypes

import numpy as np
import pytest

from _helpers import REL_TOL, rel_err, shell_points

pytestmark = pytest.mark.gpu


def _volume(gvdb2_mod, pts, weights):
    import torch
    v = gvdb2_mod.VolumeGVDB(0)
    v.Configure(3, 3, 3, 3, 3)
    v.AddChannel(0, gvdb2_mod.T_FLOAT, 1)
    v.AddChannel(1, gvdb2_mod.T_FLOAT, 1)
    tp = torch.from_numpy(pts).cuda()
    tw = torch.from_numpy(weights).cuda()
    v.SetPoints(tp)
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    v.ScatterKernel(gvdb2_mod.KERNEL_CUBIC2, len(pts), [0, 1], attrs=[None, tw])
    v.UpdateApron()
    return v, (tp, tw)


def test_noalloc_gather_matches_gather_kernel_twice(gvdb2_mod):
    import torch
    from gvdb2 import _lib
    L = _lib.lib()
    pts = shell_points(300_000, seed=31)
    w = np.random.default_rng(32).uniform(0.5, 1.5, len(pts)).astype(np.float32)
    v, keep = _volume(gvdb2_mod, pts, w)
    second = pts[::3].copy()
    second[::11] += 400.0       # outside every brick
    second[1::11, 2] = 1.0e10   # NOHIT
    calls = [(pts, gvdb2_mod.KERNEL_CUBIC2, (0.0, 0.0, 0.0)), (second, gvdb2_mod.KERNEL_TENT1, (0.25, -0.5, 0.0))]
    chans = (ctypes.c_int * 2)(0, 1)
    for q, kernel, trans in calls:
        tq = torch.from_numpy(q).cuda()
        v.SetPoints(tq)
        want = v.GatherKernel(kernel, len(q), [0, 1], trans=trans)
        got = torch.full((len(q), 2), float("nan"), dtype=torch.float32, device="cuda")
        st = L.gvdb2_gather_kernel_noalloc(v._h, kernel, len(q), (ctypes.c_float * 3)(*trans), chans, 2,
                                           ctypes.c_void_p(got.data_ptr()), 2)
        assert st == 0, L.gvdb2_last_error(v._h)
        torch.cuda.synchronize()
        g, r = got.cpu().numpy(), want.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert rel_err(g, r) < REL_TOL
    del keep


def test_noalloc_rejects_more_points_than_its_scratch(gvdb2_mod):
    import torch
    from gvdb2 import _lib
    L = _lib.lib()
    pts = shell_points(50_000, seed=33)
    v, keep = _volume(gvdb2_mod, pts, np.ones(len(pts), np.float32))
    big = np.repeat(pts, 21, axis=0)[: (1 << 20) + 1]
    tb = torch.from_numpy(np.ascontiguousarray(big)).cuda()
    v.SetPoints(tb)
    out = torch.empty((len(big), 1), dtype=torch.float32, device="cuda")
    chans = (ctypes.c_int * 1)(0)
    st = L.gvdb2_gather_kernel_noalloc(v._h, gvdb2_mod.KERNEL_TENT1, len(big), None, chans, 1,
                                       ctypes.c_void_p(out.data_ptr()), 1)
    assert st == 7  # GVDB2_ERR_CAPACITY
    assert b"1,048,576" in L.gvdb2_last_error(v._h)
    del keep


def test_noalloc_gather_16cubed_bricks_twice(gvdb2_mod):
    """Bricks of 16^3 voxels hold 8 cells each; the cell-order binning of the
    scratch array must agree with gvdb2_gather_kernel on two calls in a row."""
    import torch
    from gvdb2 import _lib
    L = _lib.lib()
    pts = shell_points(200_000, seed=34)
    v = gvdb2_mod.VolumeGVDB(0)
    v.Configure(3, 3, 3, 3, 4)
    v.AddChannel(0, gvdb2_mod.T_FLOAT, 1)
    tp = torch.from_numpy(pts).cuda()
    v.SetPoints(tp)
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    v.ScatterKernel(gvdb2_mod.KERNEL_CUBIC2, len(pts), [0])
    v.UpdateApron()
    chans = (ctypes.c_int * 1)(0)
    for q, kernel in ((pts, gvdb2_mod.KERNEL_CUBIC2), (pts[1::2].copy(), gvdb2_mod.KERNEL_TENT1)):
        tq = torch.from_numpy(q).cuda()
        v.SetPoints(tq)
        want = v.GatherKernel(kernel, len(q), [0])
        got = torch.full((len(q), 1), float("nan"), dtype=torch.float32, device="cuda")
        st = L.gvdb2_gather_kernel_noalloc(v._h, kernel, len(q), None, chans, 1, ctypes.c_void_p(got.data_ptr()), 1)
        assert st == 0, L.gvdb2_last_error(v._h)
        torch.cuda.synchronize()
        g, r = got.cpu().numpy(), want.cpu().numpy()
        assert np.all(np.isfinite(g))
        assert rel_err(g, r) < REL_TOL
    # a refused call (unknown kernel, missing channel) launches nothing
    out = torch.full((len(pts), 1), 7.0, dtype=torch.float32, device="cuda")
    v.SetPoints(tp)
    for kernel, ch in ((9, 0), (gvdb2_mod.KERNEL_TENT1, 5)):
        bad = (ctypes.c_int * 1)(ch)
        st = L.gvdb2_gather_kernel_noalloc(v._h, kernel, len(pts), None, bad, 1, ctypes.c_void_p(out.data_ptr()), 1)
        assert st == 1  # GVDB2_ERR_ARG
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
    del tp


def test_noalloc_rejects_more_cells_than_its_scratch(gvdb2_mod):
    """More than 32,768 active 8^3 cells is refused before anything is
    written: the output keeps its contents."""
    import torch
    from gvdb2 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(35)
    pts = rng.uniform(8.0, 1016.0, (60_000, 3)).astype(np.float32)  # one isolated brick per point, mostly
    v = gvdb2_mod.VolumeGVDB(0)
    v.Configure(3, 3, 3, 3, 3)
    v.AddChannel(0, gvdb2_mod.T_FLOAT, 1)
    tp = torch.from_numpy(pts).cuda()
    v.SetPoints(tp)
    v.RebuildTopology(len(pts), 0.0)
    v.UpdateAtlas()
    assert int(v.info().atlas_slots) > 32_768
    out = torch.full((len(pts), 1), 7.0, dtype=torch.float32, device="cuda")
    chans = (ctypes.c_int * 1)(0)
    st = L.gvdb2_gather_kernel_noalloc(v._h, gvdb2_mod.KERNEL_TENT1, len(pts), None, chans, 1,
                                       ctypes.c_void_p(out.data_ptr()), 1)
    assert st == 7  # GVDB2_ERR_CAPACITY
    assert b"32,768" in L.gvdb2_last_error(v._h)
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())
    del tp
