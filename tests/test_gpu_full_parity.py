"""GPU-vs-oracle parity at the full sizes of the two plain configurations,
voxel by voxel and point by point (the oracle finishes each in seconds):

* the dynamic SPH-like step: 4,194,304 jittered lattice points in the
  256x128x256-voxel dam block, advected p += 0.1 v three times through the
  reference's state machine (two full rebuilds, then an incremental one that
  keeps stale leaves), Configure(3,3,3,3,3), activation radius 2; then the
  cubic scatter of mass and momentum into 4 channels, UpdateApron and the
  cubic gather of the 3 velocity channels;
* the plain small case: 1,000,000 shell points (radius 96-100, seed 0),
  RebuildTopology(N, 2), the tent scatter, UpdateApron and the tent gather;
  and the reference's own point path on the same points: InsertPoints +
  ScatterDensity (distFunc, expand) and InsertPointsSubcell + GatherDensity.

Topology (node pools, child lists, atlas map) and apron copies are compared
bit for bit; float channels and gathers within REL_TOL of the FP64 oracle.
"""
import numpy as np
import pytest

from _helpers import REL_TOL, apron_self_consistent, interior, make_oracle, rel_err
from test_gpu_topology import compare_topology, gpu_volume

pytestmark = pytest.mark.gpu

DT = np.float32(0.1)
RADIUS = 2.0


@pytest.fixture(scope="module")
def dam_run(gvdb2_mod, oracle_mod):
    """Both sides through three advect + RebuildTopology steps of the state
    machine; topology compared after every step."""
    import torch
    import gvdb2.workloads as wl
    p0, vel = wl.dam_block()
    assert len(p0) == 4_194_304
    chans = [0, 1, 2, 3]
    o = make_oracle(oracle_mod, chans=chans)
    v = gpu_volume(gvdb2_mod, p0, chans=chans)
    tp = v._pts
    tv = torch.from_numpy(vel).cuda()
    p = p0
    per_step = []
    for _ in range(3):
        p = (p + DT * vel).astype(np.float32)
        tp.copy_(torch.from_numpy(p))  # both sides advect with the same float32 rounding
        v.SetPoints(tp)
        v.RebuildTopology(len(p), RADIUS)
        v.UpdateAtlas()
        assert o.rebuild_topology(p, RADIUS) == 0
        o.update_atlas()
        compare_topology(v, o)
        assert np.array_equal(v.atlas_map(), o.atlas_map())
        inf = v.info()
        per_step.append((int(inf.pool_count[0]), int(inf.used_leaves)))
    return v, o, p, vel, tv, per_step


def test_dam_block_topology_through_the_state_machine(dam_run):
    _, _, _, _, _, per_step = dam_run
    # the third rebuild is incremental: the pool keeps the stale leaves
    assert per_step[2][0] >= per_step[2][1]


def test_dam_block_scatter_apron_gather_match_oracle(dam_run):
    v, o, p, vel, tv, _ = dam_run
    n = len(p)
    K = 2  # cubic B-spline
    attrs_gpu = [None, (tv, 0), (tv, 1), (tv, 2)]
    v.ScatterKernel(K, n, [0, 1, 2, 3], weight=1.0, attrs=attrs_gpu)
    o.scatter_kernel(K, p, [0, 1, 2, 3], attrs=[None, vel[:, 0], vel[:, 1], vel[:, 2]])
    for c in range(4):
        e = rel_err(interior(v.atlas(c), 1), interior(o.atlas(c), 1))
        assert e < REL_TOL, f"channel {c}: interior rel err {e:.3e}"
    v.UpdateApron(-1, 0.0)
    for c in range(4):
        o.update_apron(c, 0.0)
    tiles = v.atlas(1)
    slot_leaf = v.atlas_map()["mLeafID"][:tiles.shape[0]]
    pos = v.nodes(0)["mPos"][slot_leaf]
    assert apron_self_consistent(tiles, None, pos, 8, 1, 0.0) == len(pos) * (1000 - 512)
    for c in range(4):
        e = rel_err(v.atlas(c), o.atlas(c))
        assert e < REL_TOL, f"channel {c}: tile rel err {e:.3e}"
    g = v.GatherKernel(K, n, [1, 2, 3]).cpu().numpy()
    r = o.gather_kernel(K, p, [1, 2, 3])
    for c in range(3):
        e = rel_err(g[:, c], r[:, c])
        assert e < REL_TOL, f"gathered velocity {c}: rel err {e:.3e}"


@pytest.fixture(scope="module")
def shell_run(gvdb2_mod, oracle_mod):
    import gvdb2.workloads as wl
    p = wl.plain_small()
    assert len(p) == 1_000_000
    o = make_oracle(oracle_mod, chans=[0, 1])
    v = gpu_volume(gvdb2_mod, p, chans=[0, 1])
    v.RebuildTopology(len(p), RADIUS)
    v.UpdateAtlas()
    assert o.rebuild_topology(p, RADIUS) == 0
    o.update_atlas()
    compare_topology(v, o)
    assert np.array_equal(v.atlas_map(), o.atlas_map())
    return v, o, p


def test_plain_shell_kernel_path_matches_oracle(shell_run):
    v, o, p = shell_run
    n = len(p)
    K = 1  # tent
    v.ScatterKernel(K, n, [0])
    o.scatter_kernel(K, p, [0])
    assert rel_err(interior(v.atlas(0), 1), interior(o.atlas(0), 1)) < REL_TOL
    v.UpdateApron(0, 0.0)
    o.update_apron(0, 0.0)
    assert rel_err(v.atlas(0), o.atlas(0)) < REL_TOL
    g = v.GatherKernel(K, n, [0]).cpu().numpy()
    r = o.gather_kernel(K, p, [0])
    assert rel_err(g, r) < REL_TOL


def test_plain_shell_reference_path_matches_oracle(shell_run):
    v, o, p = shell_run
    n = len(p)
    v.ClearChannel(0)
    o.clear_channel(0)
    v.InsertPoints(n)
    pnode, _, gcnt = o.insert_points(p)
    got_pnode, _, got_gcnt = v.point_nodes(n)
    assert np.array_equal(got_pnode, pnode)
    assert np.array_equal(got_gcnt[:len(gcnt)], gcnt)
    v.ScatterDensity(n, 1.0, 1.0, (0, 0, 0), True)
    o.scatter_density(p, 1.0, 1.0, (0, 0, 0), True, pnode)
    assert rel_err(v.atlas(0), o.atlas(0)) < REL_TOL
    v.ClearChannel(1)
    o.clear_channel(1)
    ln = v.InsertPointsSubcell(4, n, RADIUS)
    assert ln == o.insert_points_subcell(4, p, RADIUS)
    v.GatherDensity(4, n, 1.0, (0, 0, 0), ln, 1)
    o.gather_density(4, 1.0, 1)
    assert rel_err(interior(v.atlas(1), 1), interior(o.atlas(1), 1)) < REL_TOL
