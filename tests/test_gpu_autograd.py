"""The adjoint kernels composed by torch.autograd (the ScatterFn / GatherFn
wrappers of tests/_autograd.py) against a dense FP64 restatement of the same
splat and gather differentiated by torch itself.  The loss

    L = sum_p c_p * gather(scatter(w))_p + 1/2 * sum_v rho_v^2

sends gradients to the positions through both the gather and the scatter,
and to the weights through the scatter.  The dense restatement agrees with
the FP64 oracle's adjoints to float64 rounding on this lattice."""
import numpy as np
import pytest

from _autograd import DenseGrid, GatherFn, ScatterFn, inner
from _helpers import REL_TOL, rel_err
from test_gpu_topology import gpu_volume

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4  # relative to the largest gradient component


@pytest.mark.parametrize("kernel", [1, 2])
def test_autograd_composes_adjoints(gvdb2_mod, kernel):
    import torch
    import gvdb2.workloads as wl
    p, _ = wl.dam_block(sites=(48, 12, 48), seed=1)
    n = len(p)
    w = np.random.default_rng(5).uniform(0.5, 1.5, n).astype(np.float32)
    c = np.random.default_rng(6).standard_normal(n).astype(np.float32)
    v = gpu_volume(gvdb2_mod, p, chans=[0, 1, 2, 3])
    v.RebuildTopology(n, 2.0)
    v.UpdateAtlas()

    pos = v._pts.requires_grad_(True)  # the tensor the volume holds from SetPoints
    wt = torch.from_numpy(w).cuda().requires_grad_(True)
    ct = torch.from_numpy(c).cuda()
    grid = ScatterFn.apply(pos, wt, v, kernel, 0, 3)
    out = GatherFn.apply(pos, grid, v, kernel, 1, 2)
    fit = (ct * out).sum()
    energy = 0.5 * (inner(grid).double() ** 2).sum()
    loss = fit.double() + energy
    gp, gw = torch.autograd.grad(loss, [pos, wt])

    pd = torch.from_numpy(p.astype(np.float64)).requires_grad_(True)
    wd = torch.from_numpy(w.astype(np.float64)).requires_grad_(True)
    dense = DenseGrid(pd, kernel)
    rho = dense.scatter(wd)
    ref = (torch.from_numpy(c.astype(np.float64)) * dense.gather(rho)).sum() + 0.5 * (rho * rho).sum()
    rp, rw = torch.autograd.grad(ref, [pd, wd])

    scale = float((ct * out).abs().sum().detach()) + float(energy.detach())
    assert abs(float(loss.detach()) - float(ref.detach())) <= REL_TOL * scale
    assert rel_err(gp.cpu().numpy(), rp.numpy()) < GRAD_TOL
    assert rel_err(gw.cpu().numpy(), rw.numpy()) < GRAD_TOL
