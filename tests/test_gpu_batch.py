"""Batched clouds: several point clouds packed into one volume must give,
cloud by cloud, exactly what a volume of their own gives.  With stable
(deterministic) binning a cell adds its points in the same order either way,
so the checks are bit for bit, forward and adjoint:
  - the same bricks and atlas tiles (apron included);
  - the same gathered values;
  - the same dL/dG grids;
  - the same per-point gradients."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CFG = (3, 3, 3, 3, 3)
SPACE_LOG2 = 10  # every cloud lives in [0, 1024)^3


def clouds(seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for n, sigma, centre in ((3_000, 8.0, 512.0), (40_000, 30.0, 480.0), (12_000, 15.0, 20.0),
                             (60_000, 45.0, 700.0), (7_500, 20.0, 1000.0)):
        c = rng.normal(centre, sigma, (n, 3)) + rng.uniform(-10, 10, 3)
        # clouds 2 and 4 reach the faces of their space: activation boxes
        # are clamped there exactly as in a volume of their own
        out.append(np.clip(c, 0.25, 1023.5).astype(np.float32))
    return out


def run(gvdb2_mod, pts_list, kernel, batched):
    """Rebuild, splat 2 channels, apron, gather, then both adjoints (the
    gathered values as dL/dout, dL/dG into channels 2-3); returns per cloud
    (brick positions, {brick pos: tile per channel}, per-point arrays)."""
    import torch
    attrs = [np.sin(0.05 * p[:, 0]).astype(np.float32) for p in pts_list]
    results = []
    vols = []
    if batched:
        v = gvdb2_mod.VolumeGVDB(0)
        v.SetDeterministic(True)
        v.Configure(*CFG)
        for c in range(4):
            v.AddChannel(c, gvdb2_mod.T_FLOAT, 1)
        dev = [torch.from_numpy(p).cuda() for p in pts_list]
        first = v.BatchPoints(dev, SPACE_LOG2)
        groups = [(v, first, dev)]
    else:
        groups = []
        for p in pts_list:
            v = gvdb2_mod.VolumeGVDB(0)
            v.SetDeterministic(True)
            v.Configure(*CFG)
            for c in range(4):
                v.AddChannel(c, gvdb2_mod.T_FLOAT, 1)
            t = torch.from_numpy(p).cuda()
            v.SetPoints(t)
            groups.append((v, np.array([0, len(p)], np.int64), [t]))
    for v, first, keep in groups:
        n = int(first[-1])
        attr = torch.from_numpy(np.concatenate(attrs[len(results):len(results) + len(first) - 1])).cuda()
        v.RebuildTopology(n, 2.0)
        v.UpdateAtlas()
        for c in range(4):
            v.ClearChannel(c)
        v.ScatterKernel(kernel, n, [0, 1], weight=1.0, attrs=[None, attr])
        v.UpdateApron(-1, 0.25)
        out_t = v.GatherKernel(kernel, n, [0, 1])
        gp_gather = v.GatherDensityBackward(kernel, n, [0, 1], out_t, grad_chans=[2, 3])
        gp_scatter, g_w, g_a = v.ScatterDensityBackward(kernel, n, [2, 3], weight=1.0, attrs=[None, attr])
        per_point = np.concatenate([out_t.cpu().numpy(), gp_gather.cpu().numpy(), gp_scatter.cpu().numpy(),
                                    g_w.cpu().numpy()[:, None], g_a.cpu().numpy()], axis=1)
        amap = v.atlas_map()
        tiles = [v.atlas(c) for c in range(4)]
        slots = int(v.info().atlas_slots)
        for k in range(len(first) - 1):
            o = np.array(v.BatchOrigin(k) if batched else (0, 0, 0))
            pos = amap["mPos"][:slots]
            mine = np.all((pos >= o) & (pos < o + (1 << SPACE_LOG2)), axis=1)
            bricks = {tuple(q): s for s, q in enumerate((pos - o).tolist()) if mine[s]}
            results.append((set(bricks), {b: [tiles[c][s] for c in range(4)] for b, s in bricks.items()},
                            per_point[first[k]:first[k + 1]]))
        vols.append((v, keep))
    return results


@pytest.mark.parametrize("kernel_name", ["KERNEL_CUBIC2", "KERNEL_TENT1"])
def test_batch_equals_per_cloud_volumes(gvdb2_mod, kernel_name):
    kernel = getattr(gvdb2_mod, kernel_name)
    pts = clouds()
    solo = run(gvdb2_mod, pts, kernel, batched=False)
    both = run(gvdb2_mod, pts, kernel, batched=True)
    assert len(solo) == len(both) == len(pts)
    for c, ((b0, t0, g0), (b1, t1, g1)) in enumerate(zip(solo, both)):
        assert b0 == b1, f"cloud {c}: brick sets differ"
        for b in b0:
            for ch in range(4):
                assert np.array_equal(t0[b][ch].view(np.uint32), t1[b][ch].view(np.uint32)), (c, b, ch)
        assert np.array_equal(g0.view(np.uint32), g1.view(np.uint32)), f"cloud {c}: per-point values differ"


def test_batch_origin_layout(gvdb2_mod):
    import torch
    v = gvdb2_mod.VolumeGVDB(0)
    v.Configure(*CFG)
    v.AddChannel(0, gvdb2_mod.T_FLOAT, 1)
    pts = [torch.full((10, 3), 500.0, device="cuda") for _ in range(9)]
    first = v.BatchPoints(pts, SPACE_LOG2)
    assert first.tolist() == list(range(0, 100, 10))
    # 9 clouds -> a 3x3x3 grid of 2048-voxel blocks, x fastest
    assert v.BatchOrigin(0) == (0, 0, 0)
    assert v.BatchOrigin(1) == (2048, 0, 0)
    assert v.BatchOrigin(3) == (0, 2048, 0)
    assert v.BatchOrigin(8) == (4096, 4096, 0)
    with pytest.raises(gvdb2_mod.GvdbError):
        v.BatchOrigin(9)
