"""Kernel splats and gathers on bricks larger than 8^3 (Configure(3,3,3,3,4)
for 16^3 bricks, Configure(3,3,3,4,5) for 32^3) against the FP64 oracle.
The GPU kernels work on 8^3 cells of a brick, so these cases exercise the
cell decode, the cell bins, partials that cross cell and brick faces, and
halo tiles staged from the neighbouring cells of the same and of other
bricks."""
import ctypes

import numpy as np
import pytest

from _helpers import REL_TOL, apron_self_consistent, interior, make_oracle, rel_err, shell_points
from test_gpu_topology import gpu_volume

pytestmark = pytest.mark.gpu

CFGS = [(3, 3, 3, 3, 4), (3, 3, 3, 4, 5)]


def both(gvdb2_mod, oracle_mod, pts, chans, cfg, radius=2.0):
    o = make_oracle(oracle_mod, cfg, chans=chans)
    assert o.rebuild_topology(pts, radius) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts, cfg, chans=chans)
    v.RebuildTopology(len(pts), radius)
    v.UpdateAtlas()
    return v, o


@pytest.mark.parametrize("cfg", CFGS)
@pytest.mark.parametrize("kernel", [1, 2])
def test_scatter_gather_large_bricks(gvdb2_mod, oracle_mod, cfg, kernel):
    import torch
    p = shell_points(40_000, seed=41)
    n = len(p)
    rng = np.random.default_rng(42)
    w = rng.uniform(0.5, 1.5, n).astype(np.float32)
    at = rng.standard_normal(n).astype(np.float32)
    v, o = both(gvdb2_mod, oracle_mod, p, [0, 1], cfg)
    res = 1 << cfg[4]
    tw, ta = torch.from_numpy(w).cuda(), torch.from_numpy(at).cuda()
    v.ScatterKernel(kernel, n, [0, 1], weight=tw, attrs=[None, ta])
    o.scatter_kernel(kernel, p, [0, 1], weight=w, attrs=[None, at])
    # the splat takes only the 8^3 cells that hold points
    assert int(v.info().splat_cells) == len(np.unique(np.floor(p).astype(np.int64) >> 3, axis=0))
    for c in (0, 1):
        g, r = interior(v.atlas(c), 1), interior(o.atlas(c), 1)
        assert g.shape[1] == res
        assert rel_err(g, r) < REL_TOL, f"channel {c}"
    v.UpdateApron(-1, 0.25)
    o.update_apron(0, 0.25)
    o.update_apron(1, 0.25)
    tiles = v.atlas(0)
    slot_leaf = v.atlas_map()["mLeafID"][:tiles.shape[0]]
    pos = v.nodes(0)["mPos"][slot_leaf]
    assert apron_self_consistent(tiles, None, pos, res, 1, 0.25) == len(pos) * ((res + 2) ** 3 - res ** 3)
    got = v.GatherKernel(kernel, n, [0, 1]).cpu().numpy()
    want = o.gather_kernel(kernel, p, [0, 1])
    assert rel_err(got, want) < REL_TOL


@pytest.mark.parametrize("cfg", CFGS)
@pytest.mark.parametrize("kernel", [1, 2])
def test_adjoints_large_bricks(gvdb2_mod, oracle_mod, cfg, kernel):
    import torch
    p = shell_points(30_000, seed=43)
    n = len(p)
    w = np.random.default_rng(44).uniform(0.5, 1.5, n).astype(np.float32)
    v, o = both(gvdb2_mod, oracle_mod, p, [0, 1, 2], cfg, radius=3.0)
    res = 1 << cfg[4]
    s = int(v.info().atlas_slots)
    g = np.zeros((s, res + 2, res + 2, res + 2), np.float32)
    g[:, 1:-1, 1:-1, 1:-1] = np.random.default_rng(45).standard_normal((s, res, res, res)).astype(np.float32)
    v.atlas_tensor(1).copy_(torch.from_numpy(g).cuda())
    buf = (ctypes.c_double * g.size).from_address(o.L.orc_atlas(o.h, 1))
    np.frombuffer(buf, np.float64).reshape(g.shape)[:] = g
    tw = torch.from_numpy(w).cuda()
    gp, gw, _ = v.ScatterDensityBackward(kernel, n, [1], weight=tw)
    ogp, ogw, _ = o.scatter_kernel_backward(kernel, p, [0], [1], weight=w)
    assert rel_err(gp.cpu().numpy(), ogp) < REL_TOL
    assert rel_err(gw.cpu().numpy(), ogw) < REL_TOL
    v.ScatterKernel(kernel, n, [0], weight=tw)
    o.scatter_kernel(kernel, p, [0], weight=w)
    dout = np.random.default_rng(46).standard_normal((n, 1)).astype(np.float32)
    gpos = v.GatherDensityBackward(kernel, n, [0], torch.from_numpy(dout).cuda(), grad_chans=[2])
    ogpos = o.gather_kernel_backward(kernel, p, [0], dout.astype(np.float64), grad_chans=[2])
    assert rel_err(gpos.cpu().numpy(), ogpos) < REL_TOL
    assert rel_err(interior(v.atlas(2), 1), interior(o.atlas(2), 1)) < REL_TOL


def test_deterministic_large_bricks(gvdb2_mod, oracle_mod):
    import torch
    p = shell_points(40_000, seed=47)
    at = np.sin(0.1 * p[:, 0]).astype(np.float32)
    v, o = both(gvdb2_mod, oracle_mod, p, [0, 1], (3, 3, 3, 3, 4))
    ta = torch.from_numpy(at).cuda()
    v.SetDeterministic(True)
    runs = []
    for _ in range(3):
        v.ScatterKernel(2, len(p), [0, 1], attrs=[None, ta])
        runs.append((v.atlas(0).tobytes(), v.atlas(1).tobytes()))
    assert all(r == runs[0] for r in runs[1:])
    o.scatter_kernel(2, p, [0, 1], attrs=[None, at])
    assert rel_err(interior(v.atlas(1), 1), interior(o.atlas(1), 1)) < REL_TOL


def test_noalloc_gather_large_bricks(gvdb2_mod, oracle_mod):
    import torch
    from gvdb2 import _lib
    L = _lib.lib()
    p = shell_points(40_000, seed=48)
    v, o = both(gvdb2_mod, oracle_mod, p, [0], (3, 3, 3, 3, 4))
    v.ScatterKernel(2, len(p), [0])
    v.UpdateApron(0)
    want = v.GatherKernel(2, len(p), [0])
    got = torch.full((len(p), 1), float("nan"), dtype=torch.float32, device="cuda")
    st = L.gvdb2_gather_kernel_noalloc(v._h, 2, len(p), (ctypes.c_float * 3)(0, 0, 0), (ctypes.c_int * 1)(0), 1,
                                       ctypes.c_void_p(got.data_ptr()), 1)
    assert st == 0, L.gvdb2_last_error(v._h)
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), want.cpu().numpy())
