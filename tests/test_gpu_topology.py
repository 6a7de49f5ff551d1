"""GPU parity of the topology path against the oracle: bit-exact node
pools, child lists, atlas map and point insertion (through the C-ABI)."""
import numpy as np
import pytest

from _helpers import assert_nodes_equal, make_oracle, shell_points

pytestmark = pytest.mark.gpu


def gpu_volume(gvdb2_mod, pts, cfg=(3, 3, 3, 3, 3), chans=(0,), apron=1):
    import torch
    v = gvdb2_mod.VolumeGVDB(0)
    v.Configure(*cfg)
    for c in chans:
        v.AddChannel(c, gvdb2_mod.T_FLOAT, apron)
    t = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).cuda()
    v.SetPoints(t)
    v._pts = t
    return v


def compare_topology(v, o):
    inf = v.info()
    d = o.depth()
    assert inf.depth == d
    assert inf.top_level == o.top_level()
    a, b = o.bbox()
    assert np.array_equal(np.array(inf.posmin[:], np.float32), a)
    assert np.array_equal(np.array(inf.posmax[:], np.float32), b)
    for lev in range(5):
        assert inf.pool_count[lev] == o.pool_count(lev), f"pool count level {lev}"
    assert inf.used_leaves == o.used_leaves()
    for lev in range(d + 1):
        assert_nodes_equal(v.nodes(lev), o.nodes(lev), lev)
        if lev >= 1:
            assert np.array_equal(v.childlists(lev), o.childlists(lev)), f"child lists level {lev}"


@pytest.mark.parametrize("cfg,radius,n", [
    ((3, 3, 3, 3, 3), 2.0, 200_000),
    ((3, 3, 3, 3, 3), 0.0, 50_000),
    ((3, 3, 3, 3, 3), 1.0, 50_000),
    ((3, 3, 3, 4, 4), 2.0, 100_000),
    ((3, 3, 3, 3, 2), 1.5, 30_000),
])
def test_full_rebuild_bit_exact(gvdb2_mod, oracle_mod, cfg, radius, n):
    pts = shell_points(n, seed=0)
    o = make_oracle(oracle_mod, cfg)
    assert o.rebuild_topology(pts, radius) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts, cfg)
    v.RebuildTopology(n, radius)
    v.UpdateAtlas()
    compare_topology(v, o)
    inf = v.info()
    assert inf.atlas_slots == o.atlas_slots()
    assert tuple(inf.atlas_subdim) == o.atlas_subdim()
    assert np.array_equal(v.atlas_map(), o.atlas_map())


def test_translation_and_negative_points(gvdb2_mod, oracle_mod):
    rng = np.random.default_rng(21)
    pts = shell_points(40_000, seed=1, r_in=30, r_out=34, center=(40.0, 40.0, 40.0))
    pts[:500] -= 60.0  # some points land at negative coordinates (lev-255 keys)
    orig = (3.25, 1.0, 0.5)
    o = make_oracle(oracle_mod)
    assert o.rebuild_topology(pts, 2.0, orig) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts)
    v.RebuildTopology(len(pts), 2.0, orig)
    v.UpdateAtlas()
    compare_topology(v, o)
    del rng


def test_second_rebuild_is_full_again(gvdb2_mod, oracle_mod):
    # mCurrDepth starts at -1, so the second call also takes the full path
    pts = shell_points(30_000, seed=2)
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, pts)
    for _ in range(2):
        assert o.rebuild_topology(pts, 2.0) == 0
        v.RebuildTopology(len(pts), 2.0)
    o.update_atlas()
    v.UpdateAtlas()
    compare_topology(v, o)


def test_depth_errors(gvdb2_mod):
    pts = np.full((100, 3), 3.0, np.float32)  # extents inside one brick
    v = gpu_volume(gvdb2_mod, pts)
    with pytest.raises(gvdb2_mod.GvdbError) as e:
        v.RebuildTopology(100, 0.0)
    assert e.value.status == 2


def test_empty_point_set(gvdb2_mod):
    v = gpu_volume(gvdb2_mod, np.zeros((1, 3), np.float32))
    with pytest.raises(gvdb2_mod.GvdbError):
        v.RebuildTopology(0, 2.0)  # empty extents: smaller than one brick


def test_insert_points(gvdb2_mod, oracle_mod):
    pts = shell_points(100_000, seed=3)
    pts[::1000, 2] = 1.0e10  # NOHIT
    pts[1::1000] += 500.0    # outside every brick
    o = make_oracle(oracle_mod)
    keep = np.ones(len(pts), bool)
    keep[::1000] = False
    keep[1::1000] = False
    good = pts[keep]  # the topology is built without the NOHIT and far-away points
    assert o.rebuild_topology(good, 2.0) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, good)
    v.RebuildTopology(len(good), 2.0)
    v.UpdateAtlas()
    import torch
    t = torch.from_numpy(pts).cuda()
    v.SetPoints(t)
    v.InsertPoints(len(pts), (0, 0, 0), prefix=True)
    pnode, poff, gcnt = v.point_nodes(len(pts))
    opnode, _, ogcnt = o.insert_points(pts)
    assert np.array_equal(pnode, opnode)
    assert np.array_equal(gcnt, ogcnt)
    # poff is an atomic order inside each leaf: a permutation of 0..count-1
    ok = pnode >= 0
    order = np.lexsort((poff[ok], pnode[ok]))
    leaves = pnode[ok][order]
    starts = np.concatenate([[0], np.cumsum(np.bincount(leaves, minlength=len(gcnt)))[:-1]])
    expect = np.arange(len(leaves)) - starts[leaves]
    assert np.array_equal(poff[ok][order], expect)


def test_neighbor_table(gvdb2_mod, oracle_mod):
    pts = shell_points(50_000, seed=4)
    o = make_oracle(oracle_mod)
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    o.update_neighbors()
    v = gpu_volume(gvdb2_mod, pts)
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    v.UpdateNeighbors()
    assert np.array_equal(v.neighbors(), o.neighbors())


def test_subcells(gvdb2_mod, oracle_mod):
    pts = shell_points(60_000, seed=5)
    o = make_oracle(oracle_mod)
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts)
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    ln = v.InsertPointsSubcell(4, len(pts), 2.0)
    oln = o.insert_points_subcell(4, pts, 2.0)
    assert ln == oln
    cnt, nid, pos = v.subcells(o.used_leaves() * 8)
    ocnt, onid, opos = o.subcells()
    assert np.array_equal(cnt, ocnt)
    assert np.array_equal(nid, onid)
    assert np.array_equal(pos, opos)


def _drift_steps(pts, vel, steps):
    for _ in range(steps):
        yield pts
        pts = pts + np.array([6.0, 0.0, 0.0], np.float32) + np.float32(0.2) * vel  # empties trailing bricks


@pytest.mark.parametrize("radius", [2.0, 0.5])
def test_incremental_rebuild_bit_exact(gvdb2_mod, oracle_mod, radius):
    """Third and later RebuildTopology calls take the incremental branch
    (V:1212-1217): appended nodes, flags, links and delinks match the oracle
    bit for bit, stale leaves included."""
    import gvdb2.workloads as wl
    p, vel = wl.dam_block(sites=(48, 12, 48), origin=(40.0, 40.0, 40.0), seed=11)
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, p)
    stale_seen = False
    for step, q in enumerate(_drift_steps(p, vel, 5)):
        assert o.rebuild_topology(q, radius) == 0
        import torch
        t = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        v.SetPoints(t)
        v._pts = t
        v.RebuildTopology(len(q), radius)
        compare_topology(v, o)
        o.update_atlas()
        v.UpdateAtlas()
        assert np.array_equal(v.atlas_map(), o.atlas_map())
        assert_nodes_equal(v.nodes(0), o.nodes(0), 0)
        stale_seen |= o.pool_count(0) > o.used_leaves()
    assert stale_seen


def test_accumulate_topology_bit_exact(gvdb2_mod, oracle_mod):
    """AccumulateTopology (V:1158-1178) keeps the flags of earlier leaves."""
    a = shell_points(20_000, seed=7, r_in=20, r_out=24, center=(60.0, 60.0, 60.0))
    b = shell_points(20_000, seed=8, r_in=20, r_out=24, center=(90.0, 60.0, 60.0))
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, a)
    import torch
    for q in (a, a, b):
        assert o.accumulate_topology(q, 2.0, (0, 0, 0), 1) == 0
        t = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        v.SetPoints(t)
        v._pts = t
        v.AccumulateTopology(len(q), 2.0, (0, 0, 0), 1)
        compare_topology(v, o)


def test_splat_after_incremental(gvdb2_mod, oracle_mod):
    """Splat and gather see only the linked leaves once stale leaves exist."""
    import gvdb2.workloads as wl
    import torch
    from _helpers import REL_TOL, rel_err
    p, vel = wl.dam_block(sites=(32, 8, 32), origin=(40.0, 40.0, 40.0), seed=12)
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, p)
    for q in _drift_steps(p, vel, 4):
        assert o.rebuild_topology(q, 2.0) == 0
        t = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        v.SetPoints(t)
        v._pts = t
        v.RebuildTopology(len(q), 2.0)
    assert o.pool_count(0) > o.used_leaves()
    o.update_atlas()
    v.UpdateAtlas()
    o.clear_channel(0)
    v.ClearChannel(0)
    o.scatter_kernel(gvdb2_mod.KERNEL_TENT1, q, [0])
    v.ScatterKernel(gvdb2_mod.KERNEL_TENT1, len(q), [0])
    assert rel_err(v.atlas(0), o.atlas(0)) <= REL_TOL
    got = v.GatherKernel(gvdb2_mod.KERNEL_TENT1, len(q), [0]).cpu().numpy()
    want = o.gather_kernel(gvdb2_mod.KERNEL_TENT1, q, [0])
    assert rel_err(got, want) <= REL_TOL


def test_sparse_extent_takes_hash_path(gvdb2_mod, oracle_mod):
    """Two clusters 100,000 voxels apart: the level-0 brick grid of their
    bounding box (12,500^3 bricks) is far past the bitmap limit, so the
    rebuild takes the hash-set path; topology still matches bit for bit."""
    a = shell_points(20_000, seed=31, r_in=20, r_out=24, center=(200.0, 200.0, 200.0))
    b = shell_points(20_000, seed=32, r_in=20, r_out=24, center=(100_200.0, 100_200.0, 100_200.0))
    pts = np.concatenate([a, b]).astype(np.float32)
    cfg = (4, 4, 4, 4, 3)
    o = make_oracle(oracle_mod, cfg)
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts, cfg)
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    compare_topology(v, o)
    assert np.array_equal(v.atlas_map(), o.atlas_map())


def test_large_extent_bitmaps_bit_exact(gvdb2_mod, oracle_mod):
    """Two clusters 4,000 voxels apart: their level-0 brick grid (about
    500^3 bricks) is within the bitmap limit but past the size where the
    parent levels and the compaction run over words across the GPU; the
    node pools, child lists and atlas map still match bit for bit, for a
    full rebuild with extra bricks and for one without (radius 0.5)."""
    a = shell_points(20_000, seed=41, r_in=20, r_out=24, center=(200.0, 260.0, 230.0))
    b = shell_points(20_000, seed=42, r_in=20, r_out=24, center=(4_200.0, 3_900.0, 4_100.0))
    pts = np.concatenate([a, b]).astype(np.float32)
    for radius in (2.0, 0.5):
        o = make_oracle(oracle_mod)
        assert o.rebuild_topology(pts, radius) == 0
        o.update_atlas()
        v = gpu_volume(gvdb2_mod, pts)
        v.RebuildTopology(len(pts), radius)
        v.UpdateAtlas()
        compare_topology(v, o)
        assert np.array_equal(v.atlas_map(), o.atlas_map())


def test_compact_pools_bit_exact(gvdb2_mod, oracle_mod):
    """CompactPools after incremental rebuilds left delinked nodes: pools,
    child lists and atlas map match the oracle's compaction bit for bit, and
    so do the incremental rebuilds and the scatter that follow."""
    import torch
    import gvdb2.workloads as wl
    p, vel = wl.dam_block(sites=(48, 12, 48), origin=(40.0, 40.0, 40.0), seed=11)
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, p)
    for step, q in enumerate(_drift_steps(p, vel, 6)):
        assert o.rebuild_topology(q, 2.0) == 0
        t = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        v.SetPoints(t)
        v._pts = t
        v.RebuildTopology(len(q), 2.0)
        if step == 3:
            assert o.pool_count(0) > o.used_leaves()
            o.compact_pools()
            v.CompactPools()
            assert o.pool_count(0) == o.used_leaves()
        compare_topology(v, o)
        o.update_atlas()
        v.UpdateAtlas()
        assert np.array_equal(v.atlas_map(), o.atlas_map())


def test_compute_bounds_bit_exact(gvdb2_mod, oracle_mod):
    """FinishTopology(bounds) = ComputeBounds (V:1792-1816): the box of the
    flagged leaves seeded with leaf 0's corner, after a full rebuild and
    after incremental rebuilds that leave stale (unflagged) leaves in the
    pool; getVolMin/getVolMax return it, and mVoxResMax only grows."""
    import torch
    import gvdb2.workloads as wl
    p, vel = wl.dam_block(sites=(48, 12, 48), origin=(40.0, 40.0, 40.0), seed=12)
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, p)
    res_max = np.zeros(3, np.float32)
    stale_seen = False
    for q in _drift_steps(p, vel, 5):
        assert o.rebuild_topology(q, 2.0) == 0
        t = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        v.SetPoints(t)
        v._pts = t
        v.RebuildTopology(len(q), 2.0)
        v.FinishTopology(True, True)
        lo, hi = o.compute_bounds()
        assert np.array_equal(np.array(v.getVolMin(), np.float32), lo)
        assert np.array_equal(np.array(v.getVolMax(), np.float32), hi)
        res_max = np.maximum(res_max, hi - lo)
        assert np.array_equal(np.array(v.info().vox_res_max[:], np.float32), res_max)
        stale_seen |= o.pool_count(0) > o.used_leaves()
    assert stale_seen
