"""InsertPointsSubcell_FP16 / GatherLevelSet_FP16 / GetMinMaxVel against the
FP64 oracle: the same subcell counts, 16-bit entries within one unit (the
oracle divides exactly, libgvdb2 with the reference's approximate
division), the level set within REL_TOL, and the two list kinds kept
apart."""
import numpy as np
import pytest

from _helpers import REL_TOL, fp16_level_set_tol, interior, make_oracle, rel_err, shell_points
from test_gpu_topology import gpu_volume

pytestmark = pytest.mark.gpu


def sort_groups(entries, cnt):
    """Each column of each subcell list sorted on its own: entries that
    differ by one unit keep |a - b| <= 1 after it (a lexicographic order
    could pair different points)."""
    out = entries.copy()
    off = np.r_[0, np.cumsum(cnt)[:-1]]
    for a, c in zip(off.tolist(), cnt.tolist()):
        out[a:a + c] = np.sort(out[a:a + c], axis=0)
    return out


@pytest.mark.parametrize("cfg", [(3, 3, 3, 3, 3), (3, 3, 3, 4, 5)])
def test_fp16_lists_and_level_set(gvdb2_mod, oracle_mod, cfg):
    import torch
    pts = shell_points(50_000, seed=61)
    vel = np.random.default_rng(62).normal(0.0, 2.0, pts.shape).astype(np.float32)
    o = make_oracle(oracle_mod, cfg, chans=[0])
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts, cfg, chans=[0])
    tv = torch.from_numpy(vel).cuda()
    v.SetPoints(v._pts, tv)
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    v.GetMinMaxVel(len(pts))
    o.get_min_max_vel(vel)
    ln = v.InsertPointsSubcell_FP16(4, len(pts), 2.0)
    oln = o.insert_points_subcell_fp16(4, pts, 2.0, vel=vel)
    assert ln == oln > 0
    m = int(o.used_leaves()) * (v.info().res[0] // 4) ** 3
    cnt, nid, pos = v.subcells(m)
    ocnt, onid, opos = o.subcells()
    assert np.array_equal(cnt, ocnt) and np.array_equal(nid, onid) and np.array_equal(pos, opos)
    q, qv = v.subcell_points_fp16(ln, vel=True)
    _, oq, oqv = o.subcell_lists()
    for got, want in ((q, oq), (qv, oqv)):
        d = np.abs(sort_groups(got, cnt).astype(np.int32) -
                   sort_groups(want, ocnt).astype(np.int32))
        assert d.max() <= 1
        assert np.mean(d == 0) > 0.99
    v.GatherLevelSet_FP16(4, len(pts), 1.0, (0, 0, 0), ln, 0)
    o.gather_level_set_fp16(4, 1.0, 0)
    want = interior(o.atlas(0), 1)
    # an entry one unit apart moves a point by one quantization step
    assert np.abs(interior(v.atlas(0), 1) - want).max() <= fp16_level_set_tol(pts, want, units=1)
    # the float gathers refuse the 16-bit lists, and the other way round
    with pytest.raises(gvdb2_mod.GvdbError):
        v.GatherLevelSet(4, len(pts), 1.0, (0, 0, 0), ln, 0)
    v.InsertPointsSubcell(4, len(pts), 2.0)
    with pytest.raises(gvdb2_mod.GvdbError):
        v.GatherLevelSet_FP16(4, len(pts), 1.0, (0, 0, 0), ln, 0)


def test_level_set_on_32_bricks(gvdb2_mod, oracle_mod):
    """4^3 subcells take a warp each, so bricks of 32^3 voxels are served too."""
    pts = shell_points(30_000, seed=63)
    cfg = (3, 3, 3, 4, 5)
    o = make_oracle(oracle_mod, cfg, chans=[0, 1])
    assert o.rebuild_topology(pts, 2.0) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, pts, cfg, chans=[0, 1])
    v.RebuildTopology(len(pts), 2.0)
    v.UpdateAtlas()
    ln = v.InsertPointsSubcell(4, len(pts), 2.0)
    assert ln == o.insert_points_subcell(4, pts, 2.0)
    v.GatherLevelSet(4, len(pts), 1.0, (0, 0, 0), ln, 0)
    o.gather_level_set(4, 1.0, 0)
    v.GatherDensity(4, len(pts), 1.0, (0, 0, 0), ln, 1)
    o.gather_density(4, 1.0, 1)
    assert rel_err(interior(v.atlas(0), 1), interior(o.atlas(0), 1)) < REL_TOL
    assert rel_err(interior(v.atlas(1), 1), interior(o.atlas(1), 1)) < REL_TOL
