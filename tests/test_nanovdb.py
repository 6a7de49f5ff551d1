"""NanoVDB-form export (ExportToNanoVDB, gNanoVDB/gvdb_export_nanovdb.cpp:
379-700; ProcessLeaf / ProcessInternalNode, cuda_export_nanovdb.cu:76-362;
ProcessGridExtents, gvdb_export_nanovdb.cpp:204-327).

On the CPU, the oracle's restatement (oracle/nanovdb.py) is checked against
what the tree and atlas say directly: every leaf's values are its atlas
brick in (x*T + y)*T + z order, every child-mask bit of a node names the
child whose corner sits at that slot, and the root's box and range cover the
leaves.  On the GPU, libgvdb2's export equals the restatement byte for byte,
for float and Vec3f grids, three tree shapes, a transform, and a volume with
stale leaves after incremental rebuilds."""
import ctypes

import numpy as np
import pytest

import nanovdb as nvo
from _helpers import make_oracle, shell_points

XF = ((1.5, -2.0, 0.25), (10.0, 30.0, -45.0), (2.0, 2.0, 0.5), (10.0, 0.0, -5.0))  # pre-translation, angles, scale, translation


def pattern(slots, t, c):
    i = np.arange(slots * t ** 3, dtype=np.float64).reshape(slots, t, t, t)
    return (np.sin(0.37 * i + c) * 100.0 - 20.0 * c).astype(np.float32)


def fill_oracle_atlas(o, nchan):
    s, t = o.atlas_slots(), o.tile_res()
    for c in range(nchan):
        buf = (ctypes.c_double * (s * t ** 3)).from_address(o.L.orc_atlas(o.h, c))
        np.frombuffer(buf, np.float64)[:] = pattern(s, t, c).ravel()


def oracle_volume(oracle_mod, pts, cfg, nchan):
    o = make_oracle(oracle_mod, cfg, chans=list(range(nchan)))
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    fill_oracle_atlas(o, nchan)
    return o


@pytest.mark.parametrize("cfg,nv", [((3, 3, 3, 3, 3), 1), ((3, 3, 5, 4, 3), 3), ((3, 3, 3, 4, 2), 1)])
def test_oracle_export_follows_the_tree(oracle_mod, cfg, nv):
    pts = shell_points(6_000, seed=81)  # radius 100 about 128: level-2 nodes in every shape
    o = oracle_volume(oracle_mod, pts, cfg, nv)
    assert o.pool_count(2) > 0
    st = nvo.state_of(o, list(range(nv)), XF)
    bg = (0.5, -1.0, 2.0)[:nv]
    p = nvo.parse(nvo.export(st, bg, "shell", 1, nv))
    g = p["grid"]
    ld = st["logdim"]
    counts = [len(st["nodes"][l]) for l in range(3)]
    rec, sec, total = nvo.layout(ld, counts, nv)
    assert g["magic"] == nvo.MAGIC and g["total_bytes"] == total and g["value_type"] == nv
    assert g["count"] == tuple(counts) + (1,) and g["section"] == tuple(sec) and g["record_bytes"] == tuple(rec)
    assert g["name"].rstrip(b"\0") == b"shell" and g["grid_class"] == 1
    T0 = 1 << ld[0]
    a = st["apron"]
    nodes0 = st["nodes"][0]
    live = np.nonzero(st["leaf_slot"] >= 0)[0]
    assert len(live) == len(nodes0)  # a full rebuild leaves no stale leaf
    # leaves: values are the atlas brick, x slowest and z fastest
    for i in live[:: max(1, len(live) // 25)]:
        s = st["leaf_slot"][i]
        body = p["rec0"][i, nvo.HEADER + T0 ** 3 // 8:nvo.HEADER + T0 ** 3 // 8 + 4 * nv * T0 ** 3]
        vals = body.view(np.float32).reshape(T0 ** 3, nv)
        for x, y, z in ((0, 0, 0), (T0 - 1, 0, 1), (1, T0 - 1, 2), (T0 - 1, T0 - 1, T0 - 1), (2, 1, 0)):
            for c in range(nv):
                assert vals[(x * T0 + y) * T0 + z, c] == st["tiles"][c][s, z + a, y + a, x + a]
        h = p["hdr0"][i]
        assert list(h["bbox_min"]) == list(nodes0["mPos"][i]) and list(h["bbox_dif"]) == [T0] * 3
        assert np.array_equal(h["vmin"][:nv], vals.min(axis=0)) and np.array_equal(h["vmax"][:nv], vals.max(axis=0))
        assert np.all(p["rec0"][i, nvo.HEADER:nvo.HEADER + T0 ** 3 // 8] == 0xFF)
    # nodes: a child-mask bit at slot (x, y, z) names the child whose corner is there
    for lev in (1, 2):
        T = 1 << ld[lev]
        span = 1 << sum(ld[:lev])  # voxels per child slot
        kids = st["nodes"][lev - 1]
        for i in range(len(st["nodes"][lev])):
            raw = p["rec%d" % lev][i]
            cmask = np.unpackbits(raw[nvo.HEADER + T ** 3 // 8:nvo.HEADER + T ** 3 // 4], bitorder="little").astype(bool)
            assert not raw[nvo.HEADER:nvo.HEADER + T ** 3 // 8].any()
            table = raw[nvo.HEADER + T ** 3 // 4:nvo.HEADER + T ** 3 // 4 + 4 * nv * T ** 3].view(np.uint32).reshape(-1, nv)
            corner = np.array(st["nodes"][lev]["mPos"][i])
            js = np.nonzero(cmask)[0]
            assert len(js) > 0
            for j in js:
                x, y, z = j // (T * T), (j // T) % T, j % T
                c = int(table[j, 0])
                assert list(kids["mPos"][c]) == list(corner + np.array([x, y, z]) * span)
            empty = np.nonzero(~cmask)[0][:50]
            assert np.all(table[empty].view(np.float32) == np.asarray(bg, np.float32))
            h = p["hdr%d" % lev][i]
            assert h["offset"] == len(st["nodes"][lev]) - i
    # root: box and range over the leaves, tiles in key order
    assert np.all(np.diff(p["tiles"]["key"].astype(np.float64)) >= 0)
    allv = np.stack([p["hdr0"]["vmin"][:, :nv].min(axis=0), p["hdr0"]["vmax"][:, :nv].max(axis=0)])
    assert np.array_equal(np.array(g["vmin"][:nv], np.float32), allv[0])
    assert np.array_equal(np.array(g["vmax"][:nv], np.float32), np.maximum(allv[1], nvo.FLT_MIN) if nv == 1 else allv[1])
    pos = nodes0["mPos"]
    assert list(g["bbox"][:3]) == list(pos.min(axis=0)) and list(g["bbox"][3:]) == list(pos.max(axis=0) + T0)
    assert g["active_voxels"] == counts[0] * T0 ** 3 and g["tile_count"] == counts[2]


def test_oracle_transform_matches_a_double_precision_matrix():
    """The float32 matrix equals T Rz Ry Rx S PT built in float64."""
    pt, ang, sc, t = [np.array(x, np.float64) for x in XF]
    r = np.radians(ang)
    cx, sx, cy, sy, cz, sz = np.cos(r[0]), np.sin(r[0]), np.cos(r[1]), np.sin(r[1]), np.cos(r[2]), np.sin(r[2])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    A = Rz @ Ry @ Rx @ np.diag(sc)
    M = np.eye(4)
    M[:3, :3] = A
    M[:3, 3] = A @ pt + t
    got = nvo.transform_matrix(XF).reshape(4, 4).T  # column-major
    assert np.allclose(got, M, atol=2e-5)
    assert np.array_equal(nvo.transform_matrix(((0, 0, 0), (0, 0, 0), (1, 1, 1), (0, 0, 0))).reshape(4, 4), np.eye(4))


def test_oracle_tile_keys_sign_extend():
    """A negative corner's shifted value sign-extends into the higher key
    fields, as uint64_t(ijk >> shift) does (gvdb_export_nanovdb.cpp:273-275)."""
    assert nvo.tile_key([512, 1024, 1536], 9) == 3 | 2 << 21 | 1 << 42
    k = nvo.tile_key([-5000, 4096, 0], 9)
    assert k >> 42 == (1 << 22) - 10 and (k >> 21) & ((1 << 21) - 1) == 8 and k & ((1 << 21) - 1) == 0
    assert nvo.tile_key([0, 0, -1], 12) == (1 << 64) - 1  # z = -1 fills every field


# ---------------------------------------------------------------- GPU parity
XF_FIELDS = ("index_to_world", "voxel_size", "world_bbox")


def assert_same_export(got, want):
    """Every field and byte equal; the transform's float fields within 1e-6
    relative (host cosf/sinf and double arithmetic on both sides)."""
    pg, pw = nvo.parse(got), nvo.parse(want)
    for k, w in pw["grid"].items():
        if k in XF_FIELDS:
            assert np.allclose(pg["grid"][k], w, rtol=1e-6, atol=1e-6), k
        else:
            assert pg["grid"][k] == w, k
    assert np.array_equal(pg["tiles"], pw["tiles"])
    for l in range(3):
        bad = np.nonzero((pg[f"rec{l}"] != pw[f"rec{l}"]).any(axis=1))[0]
        assert len(bad) == 0, (l, bad[:5], pg[f"hdr{l}"][bad[0]], pw[f"hdr{l}"][bad[0]])
    assert len(got) == len(want)


def gpu_volume_like(gvdb2_mod, pts, cfg, nchan, xf=XF):
    import torch
    from test_gpu_topology import gpu_volume
    v = gpu_volume(gvdb2_mod, pts, cfg, chans=list(range(nchan)))
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    fill_gpu_atlas(v, nchan)
    v.SetTransform(xf[0], xf[2], xf[1], xf[3])
    return v


def fill_gpu_atlas(v, nchan):
    import torch
    s, t = int(v.info().atlas_slots), int(v.info().tile_res)
    for c in range(nchan):
        v.atlas_tensor(c).copy_(torch.from_numpy(pattern(s, t, c)).cuda())


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [(3, 3, 3, 3, 3), (3, 3, 5, 4, 3), (3, 3, 3, 4, 5), (3, 3, 3, 4, 2)])
@pytest.mark.parametrize("nv", [1, 3])
def test_export_matches_restatement(gvdb2_mod, oracle_mod, cfg, nv):
    pts = shell_points(6_000 if cfg[4] < 5 else 3_000, seed=82)
    o = oracle_volume(oracle_mod, pts, cfg, nv)
    v = gpu_volume_like(gvdb2_mod, pts, cfg, nv)
    bg = (0.25, -3.0, 7.5)[:nv]
    got = v.ExportToNanoVDB(list(range(nv)), bg, "points", 2).cpu().numpy().tobytes()
    want = nvo.export(nvo.state_of(o, list(range(nv)), XF), bg, "points", 2, nv)
    assert_same_export(got, want)


@pytest.mark.gpu
def test_export_after_incremental_rebuilds(gvdb2_mod, oracle_mod):
    """Stale leaves (kept in the pool by incremental rebuilds) are zero
    records; the live tree matches the restatement byte for byte."""
    import torch
    import gvdb2.workloads as wl
    from test_gpu_topology import _drift_steps, gpu_volume
    p, vel = wl.dam_block(sites=(48, 12, 48), origin=(40.0, 40.0, 40.0), seed=11)
    cfg = (3, 3, 3, 3, 3)
    o = make_oracle(oracle_mod, cfg, chans=[0, 1, 2])
    v = gpu_volume(gvdb2_mod, p, cfg, chans=[0, 1, 2])
    for q in _drift_steps(p, vel, 5):
        assert o.rebuild_topology(q, 2.0) == 0
        t = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        v.SetPoints(t)
        v._pts = t
        v.RebuildTopology(len(q), 2.0)
        o.update_atlas()
        v.UpdateAtlas()
    assert o.pool_count(0) > o.used_leaves()  # stale leaves exist
    fill_oracle_atlas(o, 3)
    fill_gpu_atlas(v, 3)
    st = nvo.state_of(o, [0, 1, 2])
    for chans in ([1], [0, 1, 2]):
        got = v.ExportToNanoVDB(chans, 0.0).cpu().numpy().tobytes()
        want = nvo.export(dict(st, tiles=[st["tiles"][c] for c in chans]), 0.0, "", 0, len(chans))
        assert_same_export(got, want)
    rec0 = nvo.parse(got)["rec0"]
    stale = np.nonzero(st["leaf_slot"] < 0)[0]
    assert len(stale) and not rec0[stale].any()


@pytest.mark.gpu
def test_export_refusals(gvdb2_mod, oracle_mod):
    import torch
    from test_gpu_topology import gpu_volume
    pts = shell_points(4_000, seed=83)
    v = gpu_volume(gvdb2_mod, pts, (3, 3, 3, 3, 3), chans=[0])
    v.RebuildTopology(len(pts), 2.0)
    with pytest.raises(gvdb2_mod.GvdbError) as e:  # no atlas for this topology yet
        v.ExportToNanoVDB([0])
    assert e.value.status == 3
    v.UpdateAtlas()
    L, h = v._L, v._h
    size = ctypes.c_size_t()
    assert L.gvdb2_nanovdb_size(h, 2, ctypes.byref(size)) == 1  # value type neither float nor vec3f
    assert L.gvdb2_nanovdb_size(h, 1, ctypes.byref(size)) == 0
    buf = torch.empty(int(size.value), dtype=torch.uint8, device="cuda")
    ch = (ctypes.c_int * 1)(0)
    bg = (ctypes.c_float * 1)(0.0)
    ptr = ctypes.c_void_p(buf.data_ptr())
    assert L.gvdb2_export_nanovdb(h, 1, ch, bg, b"", 0, ptr, int(size.value) - 1) == 7  # capacity
    assert L.gvdb2_export_nanovdb(h, 1, (ctypes.c_int * 1)(5), bg, b"", 0, ptr, int(size.value)) == 1  # no channel 5
    assert L.gvdb2_export_nanovdb(h, 1, ch, bg, b"", 0, ctypes.c_void_p(buf.data_ptr() + 4), int(size.value)) == 1
    assert L.gvdb2_export_nanovdb(h, 1, ch, bg, b"", 0, ptr, int(size.value)) == 0
    w = gpu_volume(gvdb2_mod, pts, (3, 3, 3, 3, 1), chans=[0])  # 2^1 leaves: outside the reference's tables
    with pytest.raises(gvdb2_mod.GvdbError) as e:
        w.ExportToNanoVDB([0])
    assert e.value.status == 4
