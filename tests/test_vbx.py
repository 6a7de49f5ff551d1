"""VBX files (GVDB_FILESPEC.txt; SaveVBX V:1626-1768, LoadVBX V:507-685).

On the CPU, the oracle's restatement of the reference's writer and reader
(oracle/vbx.py) round-trips a volume.  On the GPU, libgvdb2's SaveVBX writes
the file that restatement writes for the same volume (every header field,
node field compared by the parity tests, child list and atlas voxel), and
LoadVBX restores a volume whose topology, atlas and gathers equal the
original's."""
import ctypes

import numpy as np
import pytest

import vbx
from _helpers import NODE_FIELDS, make_oracle, shell_points

# file order: pre-translation, Euler angles, scale, translation
XF = ((1.5, -2.0, 0.25), (0.0, 30.0, 0.0), (2.0, 2.0, 2.0), (10.0, 0.0, -5.0))


def pattern(slots, t, c):
    i = np.arange(slots * t ** 3, dtype=np.float64).reshape(slots, t, t, t)
    return (np.sin(0.37 * i + c) * 100.0).astype(np.float32)


def oracle_volume(oracle_mod, pts, cfg, nchan):
    o = make_oracle(oracle_mod, cfg, chans=list(range(nchan)))
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    s, t = o.atlas_slots(), o.tile_res()
    for c in range(nchan):
        buf = (ctypes.c_double * (s * t ** 3)).from_address(o.L.orc_atlas(o.h, c))
        np.frombuffer(buf, np.float64)[:] = pattern(s, t, c).ravel()
    return o


def assert_same_file(a, b):
    for k in ("major", "minor", "transform", "grids", "offsets", "dtype", "components", "compression", "voxelsize",
              "leafcnt", "leafdim", "apron", "nchan", "atlas_bytes", "topology", "reuse", "layout", "subdim",
              "atlas_res", "levels", "root", "level_table", "size"):
        assert a[k] == b[k], k
    for l in range(a["levels"]):
        for f in NODE_FIELDS:
            assert np.array_equal(a["nodes"][l][f], b["nodes"][l][f]), (l, f)
        assert np.array_equal(a["clists"][l].ravel(), b["clists"][l].ravel()), l
    for x, y in zip(a["atlases"], b["atlases"]):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_oracle_vbx_round_trip(oracle_mod, tmp_path):
    pts = shell_points(20_000, seed=71)
    o = oracle_volume(oracle_mod, pts, (3, 3, 3, 3, 3), 2)
    st = vbx.state_of(o, 2, XF)
    path = tmp_path / "o.vbx"
    vbx.write(path, st)
    r = vbx.read(path)
    assert r["end"] == r["size"]
    assert (r["major"], r["minor"], r["grids"], r["nchan"]) == (1, 11, 1, 2)
    assert np.allclose(np.array(r["transform"]), np.array(XF))
    assert r["leafcnt"] == len(st["nodes"][0]) and r["root"] == st["depth"] << 8
    t = o.tile_res()
    assert r["atlas_res"] == tuple(n * t for n in st["subdim"])
    assert r["atlas_bytes"] == 4 * np.prod(r["atlas_res"])
    for l in range(5):
        assert np.array_equal(r["nodes"][l], st["nodes"][l])
        if l > 0:
            assert np.array_equal(r["clists"][l].ravel(), st["clists"][l].ravel())
    nx, ny, _ = st["subdim"]
    for c in range(2):
        a = r["atlases"][c]
        for s in range(len(st["tiles"][c])):
            bx, by, bz = s % nx, (s // nx) % ny, s // (nx * ny)
            assert np.array_equal(a[bz * t:(bz + 1) * t, by * t:(by + 1) * t, bx * t:(bx + 1) * t], st["tiles"][c][s])


def _gpu_volume(gvdb2_mod, pts, cfg, nchan, o):
    import torch
    from test_gpu_topology import gpu_volume
    v = gpu_volume(gvdb2_mod, pts, cfg, chans=list(range(nchan)))
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    s, t = int(v.info().atlas_slots), int(v.info().tile_res)
    for c in range(nchan):
        v.atlas_tensor(c).copy_(torch.from_numpy(pattern(s, t, c)).cuda())
    v.SetTransform(XF[0], XF[2], XF[1], XF[3])
    return v


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [(3, 3, 3, 3, 3), (3, 3, 3, 4, 5)])
def test_save_vbx_matches_restatement(gvdb2_mod, oracle_mod, tmp_path, cfg):
    pts = shell_points(20_000, seed=72)
    o = oracle_volume(oracle_mod, pts, cfg, 2)
    v = _gpu_volume(gvdb2_mod, pts, cfg, 2, o)
    v.SaveVBX(tmp_path / "gpu.vbx")
    vbx.write(tmp_path / "ref.vbx", vbx.state_of(o, 2, XF))
    assert_same_file(vbx.read(tmp_path / "gpu.vbx"), vbx.read(tmp_path / "ref.vbx"))


@pytest.mark.gpu
def test_load_vbx_restores_the_volume(gvdb2_mod, oracle_mod, tmp_path):
    import torch
    pts = shell_points(20_000, seed=73)
    cfg = (3, 3, 3, 3, 3)
    o = oracle_volume(oracle_mod, pts, cfg, 2)
    v = _gpu_volume(gvdb2_mod, pts, cfg, 2, o)
    v.UpdateApron(-1, 0.0)
    v.SaveVBX(tmp_path / "a.vbx")
    w = gvdb2_mod.VolumeGVDB(0)
    w.LoadVBX(tmp_path / "a.vbx")
    assert w.GetTransform() == (XF[0], XF[2], XF[1], XF[3])
    a, b = v.info(), w.info()
    for k in ("depth", "top_level", "used_leaves", "atlas_slots", "tile_res", "apron"):
        assert getattr(a, k) == getattr(b, k), k
    assert list(a.pool_count) == list(b.pool_count)
    for l in range(int(a.depth) + 1):
        for f in NODE_FIELDS:
            assert np.array_equal(v.nodes(l)[f], w.nodes(l)[f]), (l, f)
    for c in range(2):
        assert np.array_equal(v.atlas(c), w.atlas(c))
    # the loaded volume serves the point path as the original does
    t = torch.from_numpy(pts).cuda()
    w.SetPoints(t)
    g0 = v.GatherKernel(gvdb2_mod.KERNEL_CUBIC2, len(pts), [0, 1])
    g1 = w.GatherKernel(gvdb2_mod.KERNEL_CUBIC2, len(pts), [0, 1])
    assert torch.equal(g0, g1)
    # and saves back to the same file
    w.SaveVBX(tmp_path / "b.vbx")
    assert (tmp_path / "a.vbx").read_bytes() == (tmp_path / "b.vbx").read_bytes()
    # a file written by the restatement loads as well
    vbx.write(tmp_path / "r.vbx", vbx.state_of(o, 2, XF))
    u = gvdb2_mod.VolumeGVDB(0)
    u.LoadVBX(tmp_path / "r.vbx")
    for c in range(2):
        assert np.array_equal(u.atlas(c), o.atlas(c).astype(np.float32))
