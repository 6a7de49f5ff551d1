"""torch.autograd wrappers of the kernel splat and gather, for the tests only.

Forward runs ScatterKernel / GatherKernel and backward runs the adjoint
kernels (ScatterDensityBackward / GatherDensityBackward) through the C-ABI,
so that torch's autograd composes them like any other op.  The point set is
the tensor the volume got in SetPoints: its topology and binning come from
it, and the backward kernels recompute the point -> cell mapping from it
instead of storing it.

Also a dense FP64 restatement of the same splat and gather in plain torch
(voxel centres at i + 0.5; tent taps floor(x - 0.5) + {0, 1}, cubic B-spline
taps floor(x - 0.5) + {-1, 0, 1, 2}), whose gradients come from torch's own
autograd: the reference the wrapped adjoints are checked against.
"""
import torch


def inner(tiles, apron=1):
    """Interior voxels of (slots, T, T, T) tiles."""
    return tiles[:, apron:-apron, apron:-apron, apron:-apron]


class ScatterFn(torch.autograd.Function):
    """grid = splat of `weight` at `pos` into channel `chan` of volume `v`,
    returned as the channel's used tiles (slots, T, T, T); only interior
    voxels depend on the inputs.  Backward writes dL/dgrid into channel
    `grad_chan` and returns dL/dpos, dL/dweight."""

    @staticmethod
    def forward(ctx, pos, weight, v, kernel, chan, grad_chan):
        w = weight.detach().float().contiguous()
        v.ScatterKernel(kernel, pos.shape[0], [chan], weight=w)
        ctx.save_for_backward(w)
        ctx.args = (v, kernel, grad_chan, pos.shape[0])
        return v.atlas_tensor(chan).clone()

    @staticmethod
    def backward(ctx, g_grid):
        v, kernel, grad_chan, n = ctx.args
        (w,) = ctx.saved_tensors
        v.atlas_tensor(grad_chan).copy_(g_grid)
        gp, gw, _ = v.ScatterDensityBackward(kernel, n, [grad_chan], weight=w)
        return gp, gw, None, None, None, None


class GatherFn(torch.autograd.Function):
    """out[p] = sample of `grid` (slots, T, T, T) at pos[p]: the grid is
    copied into channel `chan`, which must still hold it when backward runs.
    Backward writes dL/dgrid (interior voxels; the gather reads no apron)
    into channel `grad_chan` and returns dL/dpos, dL/dgrid."""

    @staticmethod
    def forward(ctx, pos, grid, v, kernel, chan, grad_chan, apron=1):
        v.atlas_tensor(chan).copy_(grid)
        out = v.GatherKernel(kernel, pos.shape[0], [chan])
        ctx.args = (v, kernel, chan, grad_chan, pos.shape[0], apron)
        return out[:, 0].clone()

    @staticmethod
    def backward(ctx, g_out):
        v, kernel, chan, grad_chan, n, apron = ctx.args
        go = g_out.reshape(n, 1).float().contiguous()
        gp = v.GatherDensityBackward(kernel, n, [chan], go, grad_chans=[grad_chan])
        g = v.atlas_tensor(grad_chan)
        g_grid = torch.zeros_like(g)
        inner(g_grid, apron).copy_(inner(g, apron))
        return gp, g_grid, None, None, None, None, None


# ---------------------------------------------------------------------------
# dense FP64 restatement
# ---------------------------------------------------------------------------

def dense_taps(pos, kernel):
    """First tap (N, 3) and per-axis weights (N, 3, K) of the tent (kernel 1,
    K = 2) or cubic B-spline (kernel 2, K = 4); the weights are
    differentiable in pos."""
    u = pos - 0.5
    b = torch.floor(u).detach()
    t = u - b
    if kernel == 1:
        return b.long(), torch.stack([1.0 - t, t], dim=-1)
    s = 1.0 - t
    w = torch.stack([s * s * s, (3.0 * t - 6.0) * t * t + 4.0, ((-3.0 * t + 3.0) * t + 3.0) * t + 1.0, t * t * t],
                    dim=-1) / 6.0
    return b.long() - 1, w


class DenseGrid:
    """A dense (Z, Y, X) grid of voxels lo .. lo + shape - 1 covering every
    tap of `pos` (N, 3), with the tap indices and weights of each point."""

    def __init__(self, pos, kernel):
        first, w = dense_taps(pos, kernel)
        k = w.shape[-1]
        self.lo = first.min(dim=0).values
        hi = first.max(dim=0).values + k
        self.shape = tuple(int(s) for s in (hi - self.lo).flip(0))  # (Z, Y, X)
        off = torch.arange(k)
        ix, iy, iz = [(first[:, a, None] - self.lo[a]) + off for a in range(3)]
        Z, Y, X = self.shape
        self.idx = ((iz[:, :, None, None] * Y + iy[:, None, :, None]) * X + ix[:, None, None, :]).reshape(len(pos), -1)
        self.w = (w[:, 2, :, None, None] * w[:, 1, None, :, None] * w[:, 0, None, None, :]).reshape(len(pos), -1)

    def scatter(self, weight):
        vals = (weight[:, None] * self.w).reshape(-1)
        rho = torch.zeros(self.shape[0] * self.shape[1] * self.shape[2], dtype=vals.dtype)
        return rho.index_add(0, self.idx.reshape(-1), vals)

    def gather(self, rho):
        return (rho[self.idx] * self.w).sum(dim=1)
