"""Size-independent properties of the kernel splat and gather, checked at the
full size of the dynamic workload (4,194,304 jittered lattice points in the
256 x 128 x 256-voxel dam block, 8^3 bricks, activation radius 2), where the
FP64 oracle would take minutes per call.  Each property holds exactly in the
oracle on a smaller lattice of the same layout:

* power-of-two homogeneity: amounts times 2 give channel values times 2, bit
  for bit (every product and sum of the splat scales exactly by a power of
  two, and both channels of one call add their records in the same order);
* the adjoint identity <scatter(a), g> = <a, gather(g)> over the interior
  voxels: the gather is the transpose of the scatter, taps outside the active
  bricks being dropped by one and read as 0 by the other;
* partition of unity: the taps of every point lie in active bricks (radius-2
  activation covers the cubic stencil) and their weights sum to 1, so the
  scattered mass is the number of points and a field of ones gathers to 1;
* run-to-run reproducibility of the default scatter over the same bins, and
  of a full re-binning in deterministic mode.
"""
import numpy as np
import pytest

from _helpers import REL_TOL
from test_gpu_topology import gpu_volume

pytestmark = pytest.mark.gpu

RADIUS = 2.0


@pytest.fixture(scope="module")
def dam(gvdb2_mod):
    import torch
    import gvdb2.workloads as wl
    p, vel = wl.dam_block()  # 256 x 64 x 256 sites
    assert len(p) == 4_194_304
    v = gpu_volume(gvdb2_mod, p, chans=[0, 1, 2])
    v.RebuildTopology(len(p), RADIUS)
    v.UpdateAtlas()
    rng = torch.Generator(device="cuda").manual_seed(11)
    a = torch.rand(len(p), device="cuda", generator=rng) + 0.5  # amounts in [0.5, 1.5)
    vx = torch.from_numpy(np.ascontiguousarray(vel[:, :1])).cuda()
    return v, len(p), a, vx


def inner(t):
    """Interior voxels of (slots, T, T, T) tiles with a 1-voxel apron (the
    scatter writes these; aprons keep whatever they held)."""
    return t[:, 1:-1, 1:-1, 1:-1]


def interior_sum(t, other=None):
    x = inner(t).double()
    if other is not None:
        x = x * inner(other).double()
    return float(x.sum())


@pytest.mark.parametrize("kernel", [1, 2])
def test_full_size_power_of_two_homogeneity(dam, kernel):
    import torch
    v, n, a, vx = dam
    both = torch.cat([vx, 2.0 * vx], dim=1).contiguous()  # doubling is exact
    v.ScatterKernel(kernel, n, [0, 2], weight=a, attrs=[(both, 0), (both, 1)])
    once, twice = inner(v.atlas_tensor(0)).clone(), inner(v.atlas_tensor(2)).clone()
    assert float(once.abs().max()) > 0.0
    assert torch.equal(2.0 * once, twice)


@pytest.mark.parametrize("kernel", [1, 2])
def test_full_size_adjoint_identity(dam, kernel):
    import torch
    v, n, a, _ = dam
    v.ScatterKernel(kernel, n, [0], weight=a)
    g = v.atlas_tensor(1)
    g.copy_(torch.rand(g.shape, device="cuda", generator=torch.Generator(device="cuda").manual_seed(12)))
    lhs = interior_sum(v.atlas_tensor(0), g)
    out = v.GatherKernel(kernel, n, [1])
    rhs = float((a.double() * out[:, 0].double()).sum())
    assert abs(lhs - rhs) <= REL_TOL * abs(rhs), f"<scatter(a), g> = {lhs!r}, <a, gather(g)> = {rhs!r}"


@pytest.mark.parametrize("kernel", [1, 2])
def test_full_size_partition_of_unity(dam, kernel):
    v, n, _, _ = dam
    v.ScatterKernel(kernel, n, [0], weight=1.0)
    mass = interior_sum(v.atlas_tensor(0))
    assert abs(mass - n) <= REL_TOL * n, f"scattered mass {mass!r} for {n} points"
    v.atlas_tensor(1).fill_(1.0)
    out = v.GatherKernel(kernel, n, [1])
    err = float((out[:, 0].double() - 1.0).abs().max())
    assert err <= REL_TOL, f"gather of ones: max |out - 1| = {err:.3e}"


def test_full_size_scatter_reproducible(dam):
    import torch
    v, n, a, vx = dam
    runs = []
    for _ in range(2):
        v.ScatterKernel(2, n, [0, 2], weight=a, attrs=[None, (vx, 0)])
        runs.append((inner(v.atlas_tensor(0)).clone(), inner(v.atlas_tensor(2)).clone()))
    assert torch.equal(runs[0][0], runs[1][0]) and torch.equal(runs[0][1], runs[1][1])
    # deterministic mode: every call re-bins the points (SetPoints drops the
    # bins) and still gives the same bits
    v.SetDeterministic(True)
    det = []
    for _ in range(2):
        v.SetPoints(v._pts)
        v.ScatterKernel(2, n, [0, 2], weight=a, attrs=[None, (vx, 0)])
        det.append((inner(v.atlas_tensor(0)).clone(), inner(v.atlas_tensor(2)).clone()))
    v.SetDeterministic(False)
    assert torch.equal(det[0][0], det[1][0]) and torch.equal(det[0][1], det[1][1])
    assert float((det[0][0] - runs[0][0]).abs().max()) <= REL_TOL * float(runs[0][0].abs().max())
