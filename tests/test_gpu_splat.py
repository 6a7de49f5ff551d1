"""GPU parity of the splat path against the FP64 oracle: kernel scatter,
apron (bit-exact copies), gathers, reference-mode ScatterDensity and the
voxel-centric GatherDensity / GatherLevelSet (through the C-ABI)."""
import numpy as np
import pytest

from _helpers import REL_TOL, apron_self_consistent, interior, make_oracle, rel_err, shell_points
from test_gpu_topology import gpu_volume

pytestmark = pytest.mark.gpu


def lattice(n_side=(48, 12, 48), seed=1):
    import gvdb2.workloads as wl
    return wl.dam_block(sites=n_side, spacing=(1.0, 2.0, 1.0), origin=(64.0, 64.0, 64.0), seed=seed)


def both(gvdb2_mod, oracle_mod, pts, chans, radius=2.0, cfg=(3, 3, 3, 3, 3)):
    o = make_oracle(oracle_mod, cfg, chans=chans)
    assert o.rebuild_topology(pts, radius) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts, cfg, chans=chans)
    v.RebuildTopology(len(pts), radius)
    v.UpdateAtlas()
    return v, o


@pytest.mark.parametrize("kernel", [1, 2])
def test_scatter_matches_oracle(gvdb2_mod, oracle_mod, kernel):
    import torch
    p, vel = lattice()
    n = len(p)
    chans = [0, 1, 2, 3]
    v, o = both(gvdb2_mod, oracle_mod, p, chans)
    w = np.random.default_rng(5).uniform(0.5, 1.5, n).astype(np.float32)
    tw = torch.from_numpy(w).cuda()
    tv = torch.from_numpy(vel).cuda()
    v.ScatterKernel(kernel, n, chans, weight=tw, attrs=[None, (tv, 0), (tv, 1), (tv, 2)])
    o.scatter_kernel(kernel, p, chans, weight=w, attrs=[None, vel[:, 0], vel[:, 1], vel[:, 2]])
    for c in chans:
        g = interior(v.atlas(c), 1)
        r = interior(o.atlas(c), 1)
        e = rel_err(g, r)
        assert e < REL_TOL, f"channel {c}: rel err {e:.3e}"


@pytest.mark.parametrize("kernel", [1, 2])
def test_gather_matches_oracle(gvdb2_mod, oracle_mod, kernel):
    p = shell_points(200_000, seed=0)
    v, o = both(gvdb2_mod, oracle_mod, p, [0])
    v.ScatterKernel(kernel, len(p), [0])
    o.scatter_kernel(kernel, p, [0])
    v.UpdateApron(0)
    o.update_apron(0)
    g = v.GatherKernel(kernel, len(p), [0]).cpu().numpy()
    r = o.gather_kernel(kernel, p, [0])
    assert rel_err(g, r) < REL_TOL


def test_apron_bit_exact(gvdb2_mod, oracle_mod):
    p = shell_points(60_000, seed=2)
    v, o = both(gvdb2_mod, oracle_mod, p, [0])
    v.ScatterKernel(2, len(p), [0])
    o.scatter_kernel(2, p, [0])
    v.UpdateApron(0, 0.25)
    o.update_apron(0, 0.25)
    tiles = v.atlas(0)
    slot_leaf = v.atlas_map()["mLeafID"][:tiles.shape[0]]
    pos = v.nodes(0)["mPos"][slot_leaf]
    # every apron voxel is a bit copy of its owner's interior voxel (or boundval)
    checked = apron_self_consistent(tiles, None, pos, 8, 1, 0.25)
    assert checked == len(pos) * (1000 - 512)
    assert rel_err(tiles, o.atlas(0)) < REL_TOL


def test_apron_faces(gvdb2_mod, oracle_mod):
    p = shell_points(60_000, seed=3)
    v, o = both(gvdb2_mod, oracle_mod, p, [0])
    v.ScatterKernel(1, len(p), [0])
    o.scatter_kernel(1, p, [0])
    v.UpdateNeighbors()
    o.update_neighbors()
    v.UpdateApronFaces(0)
    o.update_apron_faces(0)
    assert rel_err(v.atlas(0), o.atlas(0)) < REL_TOL


def test_reference_scatter_density(gvdb2_mod, oracle_mod):
    # collision-light input: one point per voxel corner region
    p = shell_points(30_000, seed=4)
    v, o = both(gvdb2_mod, oracle_mod, p, [0], radius=0.0)
    v.ClearChannel(0)
    o.clear_channel(0)
    v.InsertPoints(len(p))
    v.ScatterDensity(len(p), 1.0, 1.0, (0, 0, 0), True)
    pnode, _, _ = o.insert_points(p)
    o.scatter_density(p, 1.0, 1.0, (0, 0, 0), True, pnode)
    assert rel_err(v.atlas(0), o.atlas(0)) < REL_TOL
    v.UpdateApron(0)
    o.update_apron(0)
    assert rel_err(v.atlas(0), o.atlas(0)) < REL_TOL


@pytest.mark.parametrize("levelset", [False, True])
def test_voxel_gathers(gvdb2_mod, oracle_mod, levelset):
    p = shell_points(80_000, seed=6)
    v, o = both(gvdb2_mod, oracle_mod, p, [0])
    v.ClearChannel(0)
    o.clear_channel(0)
    ln = v.InsertPointsSubcell(4, len(p), 2.0)
    assert ln == o.insert_points_subcell(4, p, 2.0)
    if levelset:
        v.GatherLevelSet(4, len(p), 1.0, (0, 0, 0), ln, 0)
        o.gather_level_set(4, 1.0, 0)
    else:
        v.GatherDensity(4, len(p), 1.0, (0, 0, 0), ln, 0)
        o.gather_density(4, 1.0, 0)
    assert rel_err(interior(v.atlas(0), 1), interior(o.atlas(0), 1)) < REL_TOL


def test_deterministic_mode_bit_reproducible(gvdb2_mod, oracle_mod):
    p, vel = lattice(seed=7)
    v, o = both(gvdb2_mod, oracle_mod, p, [0, 1])
    import torch
    tv = torch.from_numpy(vel).cuda()
    v.SetDeterministic(True)
    runs = []
    for _ in range(3):
        v.ScatterKernel(2, len(p), [0, 1], attrs=[None, (tv, 0)])
        runs.append((v.atlas(0).copy(), v.atlas(1).copy()))
    for r in runs[1:]:
        assert r[0].tobytes() == runs[0][0].tobytes()
        assert r[1].tobytes() == runs[0][1].tobytes()
    o.scatter_kernel(2, p, [0, 1], attrs=[None, vel[:, 0]])
    assert rel_err(interior(runs[0][0], 1), interior(o.atlas(0), 1)) < REL_TOL
    assert rel_err(interior(runs[0][1], 1), interior(o.atlas(1), 1)) < REL_TOL


def test_points_outside_gather_zero(gvdb2_mod, oracle_mod):
    import torch
    p = shell_points(20_000, seed=8)
    v, o = both(gvdb2_mod, oracle_mod, p, [0])
    v.ScatterKernel(1, len(p), [0])
    q = p.copy()
    q[::7] += 700.0
    q[1::7, 2] = 1.0e10
    tq = torch.from_numpy(q).cuda()
    v.SetPoints(tq)
    out = v.GatherKernel(1, len(q), [0]).cpu().numpy()
    assert np.all(out[::7] == 0) and np.all(out[1::7] == 0)


@pytest.mark.parametrize("kernel", [1, 2])
def test_adjoints_match_oracle(gvdb2_mod, oracle_mod, kernel):
    import torch
    p = shell_points(50_000, seed=9)
    n = len(p)
    w = np.random.default_rng(10).uniform(0.5, 1.5, n).astype(np.float32)
    v, o = both(gvdb2_mod, oracle_mod, p, [0, 1, 2], radius=3.0)
    inf = v.info()
    s = int(inf.atlas_slots)
    g = np.zeros((s, 10, 10, 10), np.float32)
    g[:, 1:9, 1:9, 1:9] = np.random.default_rng(11).standard_normal((s, 8, 8, 8)).astype(np.float32)
    v.atlas_tensor(1).copy_(torch.from_numpy(g).cuda())
    import ctypes
    buf = (ctypes.c_double * g.size).from_address(o.L.orc_atlas(o.h, 1))
    np.frombuffer(buf, np.float64).reshape(g.shape)[:] = g
    tw = torch.from_numpy(w).cuda()
    gp, gw, ga = v.ScatterDensityBackward(kernel, n, [1], weight=tw)
    ogp, ogw, oga = o.scatter_kernel_backward(kernel, p, [0], [1], weight=w)
    assert rel_err(gp.cpu().numpy(), ogp) < REL_TOL
    assert rel_err(gw.cpu().numpy(), ogw) < REL_TOL
    # gather adjoint
    v.ScatterKernel(kernel, n, [0], weight=tw)
    o.scatter_kernel(kernel, p, [0], weight=w)
    dout = np.random.default_rng(12).standard_normal((n, 1)).astype(np.float32)
    gpos = v.GatherDensityBackward(kernel, n, [0], torch.from_numpy(dout).cuda(), grad_chans=[2])
    ogpos = o.gather_kernel_backward(kernel, p, [0], dout.astype(np.float64), grad_chans=[2])
    assert rel_err(gpos.cpu().numpy(), ogpos) < REL_TOL
    assert rel_err(interior(v.atlas(2), 1), interior(o.atlas(2), 1)) < REL_TOL
