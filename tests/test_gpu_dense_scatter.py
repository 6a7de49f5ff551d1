"""GPU parity of the scatter's dense cells (cells of 512 points or more,
splatted into fixed-point partial sums that the owner-computes pass merges):
both kernels, 1 to 4 channels, weights and attributes over a wide range of
magnitudes, cells split over several CTAs (more than 4096 points), dense
and sparse cells side by side, batched clouds against volumes of their
own, and bit-reproducibility in deterministic mode (fixed-point partials)."""
import numpy as np
import pytest

from _helpers import REL_TOL, interior, make_oracle, rel_err
from test_gpu_topology import gpu_volume

pytestmark = pytest.mark.gpu


def dense_block(sites=(64, 64, 64), spacing=0.5, seed=3):
    import gvdb2.workloads as wl
    return wl.dam_block(sites=sites, spacing=(spacing, spacing, spacing), origin=(64.0, 64.0, 64.0), seed=seed)


def volumes(gvdb2_mod, oracle_mod, p, chans, radius=2.0):
    o = make_oracle(oracle_mod, chans=chans)
    assert o.rebuild_topology(p, radius) == 0
    o.update_atlas()
    v = gpu_volume(gvdb2_mod, p, chans=chans)
    v.RebuildTopology(len(p), radius)
    v.UpdateAtlas()
    return v, o


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("nch", [1, 2, 3, 4])
def test_dense_scatter_matches_oracle(gvdb2_mod, oracle_mod, kernel, nch):
    import torch
    p, vel = dense_block()
    n = len(p)
    chans = list(range(nch))
    v, o = volumes(gvdb2_mod, oracle_mod, p, chans)
    w = np.random.default_rng(5).uniform(0.5, 1.5, n).astype(np.float32)
    tw = torch.from_numpy(w).cuda()
    tv = torch.from_numpy(vel).cuda()
    attrs_g = [None, (tv, 0), (tv, 1), (tv, 2)][:nch]
    attrs_o = [None, vel[:, 0], vel[:, 1], vel[:, 2]][:nch]
    v.ScatterKernel(kernel, n, chans, weight=tw, attrs=attrs_g)
    o.scatter_kernel(kernel, p, chans, weight=w, attrs=attrs_o)
    for c in chans:
        e = rel_err(interior(v.atlas(c), 1), interior(o.atlas(c), 1))
        assert e < REL_TOL, f"channel {c}: rel err {e:.3e}"


@pytest.mark.parametrize("kernel", [1, 2])
def test_dense_giant_cells_and_wide_range(gvdb2_mod, oracle_mod, kernel):
    """64 points a voxel (32,768 a cell: 8 CTAs each) and amounts spread
    over 12 decades."""
    import torch
    p, vel = dense_block(sites=(64, 64, 64), spacing=0.25, seed=4)
    n = len(p)
    v, o = volumes(gvdb2_mod, oracle_mod, p, [0, 1])
    rng = np.random.default_rng(6)
    w = (10.0 ** rng.uniform(-6, 6, n)).astype(np.float32)
    tw = torch.from_numpy(w).cuda()
    tv = torch.from_numpy(vel).cuda()
    v.ScatterKernel(kernel, n, [0, 1], weight=tw, attrs=[None, (tv, 0)])
    o.scatter_kernel(kernel, p, [0, 1], weight=w, attrs=[None, vel[:, 0]])
    for c in (0, 1):
        e = rel_err(interior(v.atlas(c), 1), interior(o.atlas(c), 1))
        assert e < REL_TOL, f"channel {c}: rel err {e:.3e}"


def blob(n, sigma, centre, seed):
    rng = np.random.default_rng(seed)
    return np.clip(rng.normal(centre, sigma, (n, 3)), 0.25, 1023.5).astype(np.float32)


@pytest.mark.parametrize("kernel", [1, 2])
def test_mixed_dense_and_sparse_cells(gvdb2_mod, oracle_mod, kernel):
    """A Gaussian blob: cells of up to ~20,000 points at its centre, a few
    points in its outskirts; dense and owner-computed cells meet."""
    import torch
    p = blob(400_000, 6.0, 300.0, 11)
    n = len(p)
    attr = np.cos(0.1 * p[:, 1]).astype(np.float32)
    v, o = volumes(gvdb2_mod, oracle_mod, p, [0, 1])
    v.SetDeterministic(True)
    ta = torch.from_numpy(attr).cuda()
    v.ScatterKernel(kernel, n, [0, 1], weight=1.0, attrs=[None, ta])
    o.scatter_kernel(kernel, p, [0, 1], attrs=[None, attr])
    for c in (0, 1):
        e = rel_err(interior(v.atlas(c), 1), interior(o.atlas(c), 1))
        assert e < REL_TOL, f"channel {c}: rel err {e:.3e}"


def test_mixed_density_batched_identical_to_own_volumes(gvdb2_mod):
    """Two blobs with dense centres, batched and each in a volume of its own:
    the same tiles bit for bit (deterministic binning)."""
    import torch
    clouds = [blob(300_000, 5.0, 500.0, 12), blob(150_000, 9.0, 480.0, 13)]
    tiles = []
    for batched in (True, False):
        vols = []
        if batched:
            v = gvdb2_mod.VolumeGVDB(0)
            v.SetDeterministic(True)
            v.Configure(3, 3, 3, 3, 3)
            v.AddChannel(0, gvdb2_mod.T_FLOAT, 1)
            dev = [torch.from_numpy(c).cuda() for c in clouds]
            first = v.BatchPoints(dev, 10)
            vols.append((v, int(first[-1]), dev, [v.BatchOrigin(k) for k in range(len(clouds))]))
        else:
            for c in clouds:
                v = gvdb2_mod.VolumeGVDB(0)
                v.SetDeterministic(True)
                v.Configure(3, 3, 3, 3, 3)
                v.AddChannel(0, gvdb2_mod.T_FLOAT, 1)
                t = torch.from_numpy(c).cuda()
                v.SetPoints(t)
                vols.append((v, len(c), [t], [(0, 0, 0)]))
        got = {}
        for k, (v, n, keep, origins) in enumerate(vols):
            v.RebuildTopology(n, 2.0)
            v.UpdateAtlas()
            v.ScatterKernel(2, n, [0], weight=1.0)
            amap = v.atlas_map()
            slots = int(v.info().atlas_slots)
            pos = amap["mPos"][:slots]
            t = v.atlas(0)
            for ci, o in enumerate(origins):
                cid = ci if batched else k
                o = np.array(o)
                mine = np.all((pos >= o) & (pos < o + 1024), axis=1)
                for s in np.nonzero(mine)[0]:
                    got[(cid, tuple((pos[s] - o).tolist()))] = t[s].tobytes()
        tiles.append(got)
    assert tiles[0].keys() == tiles[1].keys()
    assert all(tiles[0][k] == tiles[1][k] for k in tiles[0])


@pytest.mark.parametrize("spacing", [0.5, 0.25])
def test_dense_deterministic_mode_bit_reproducible(gvdb2_mod, oracle_mod, spacing):
    """Deterministic mode: the dense cells' fixed-point partials (one CTA a
    cell, and 8 CTAs a cell at spacing 0.25) and the whole grid are the same
    bit for bit from call to call, with the bins made again each time."""
    import torch
    p, vel = dense_block(spacing=spacing, seed=9)
    n = len(p)
    v, o = volumes(gvdb2_mod, oracle_mod, p, [0, 1])
    tv = torch.from_numpy(vel).cuda()
    v.SetDeterministic(True)
    runs = []
    for _ in range(3):
        v.SetPoints(v._pts)  # bins made again
        v.ScatterKernel(2, n, [0, 1], attrs=[None, (tv, 1)])
        runs.append((v.atlas(0).tobytes(), v.atlas(1).tobytes()))
    assert all(r == runs[0] for r in runs[1:])
    o.scatter_kernel(2, p, [0, 1], attrs=[None, vel[:, 1]])
    g = np.frombuffer(runs[0][1], np.float32).reshape(v.atlas(1).shape)
    assert rel_err(interior(g, 1), interior(o.atlas(1), 1)) < REL_TOL
