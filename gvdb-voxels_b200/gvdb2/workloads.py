"""Seeded synthetic point sets with the shapes, sizes and value distributions
of the five benchmark configurations.  The reference ships no dataset for
this path, so these generators stand in for one.

Every generator returns float32 arrays; positions are in voxel (index-space)
units.
"""
import numpy as np

SHELL_CENTER = (128.0, 128.0, 128.0)


def shell(n, seed, r_in, r_out, center=SHELL_CENTER):
    """n points uniform in a spherical shell r in [r_in, r_out)."""
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    r = (r_in ** 3 + u * (r_out ** 3 - r_in ** 3)) ** (1.0 / 3.0)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p = np.asarray(center, np.float64) + d * r[:, None]
    return p.astype(np.float32)


def plain_small(n=1_000_000, seed=0):
    """Config 0: uniform shell, centre (128,128,128), radius 96-100, weight 1."""
    return shell(n, seed, 96.0, 100.0)


def diff_target(n=1_000_000, seed=2):
    """Config 2 target set: shell radius 90-104."""
    return shell(n, seed, 90.0, 104.0)


def dam_block(sites=(256, 64, 256), spacing=(1.0, 2.0, 1.0), origin=(64.0, 64.0, 64.0), seed=1, jitter=0.1):
    """Config 1: jittered lattice filling a dam block; sites[0] x sites[1] x
    sites[2] points (x fastest), site i at origin + (i + 0.5) * spacing plus
    U(-jitter, jitter); velocity ~ N(0, 1).

    The default 256 x 64 x 256 sites at spacing (1, 2, 1) fill the
    256 x 128 x 256-voxel block with exactly 4,194,304 points; the
    16,777,216-point variant is sites (256, 256, 256) at spacing (1, 0.5, 1).
    """
    rng = np.random.default_rng(seed)
    sx, sy, sz = sites
    n = sx * sy * sz
    ix = np.arange(sx, dtype=np.float32)
    iy = np.arange(sy, dtype=np.float32)
    iz = np.arange(sz, dtype=np.float32)
    z, y, x = np.meshgrid(iz, iy, ix, indexing="ij")
    p = np.empty((n, 3), np.float32)
    p[:, 0] = origin[0] + (x.ravel() + 0.5) * spacing[0]
    p[:, 1] = origin[1] + (y.ravel() + 0.5) * spacing[1]
    p[:, 2] = origin[2] + (z.ravel() + 0.5) * spacing[2]
    p += rng.uniform(-jitter, jitter, (n, 3)).astype(np.float32)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    return p, vel


def batched_clouds(count=64, seed=3, lo=1e4, hi=2e6, space=1024.0):
    """Config 3: `count` Gaussian blobs with sizes log-uniform in [lo, hi],
    sigma ~ U(8, 64), centred in their own `space`^3 index space."""
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)
    sigmas = rng.uniform(8.0, 64.0, count)
    clouds = []
    for c in range(count):
        p = rng.normal(space / 2, sigmas[c], (int(sizes[c]), 3))
        p = np.clip(p, 0.0, np.nextafter(space, 0))
        clouds.append(p.astype(np.float32))
    return clouds, sigmas


def gaussian_mixture(n=67_108_864, seed=4, comps=32, space=4096.0, chunk=1 << 24):
    """Config 4: `comps`-component equal-weight Gaussian mixture, sigma ~
    U(8, 64), means U[0, space)^3; points outside [0, space)^3 are rejected
    and redrawn.  Velocity ~ N(0, 2^2)."""
    rng = np.random.default_rng(seed)
    means = rng.uniform(0.0, space, (comps, 3))
    sig = rng.uniform(8.0, 64.0, comps)
    out = np.empty((n, 3), np.float32)
    got = 0
    while got < n:
        m = min(chunk, n - got)
        k = rng.integers(0, comps, m)
        p = means[k] + rng.standard_normal((m, 3)) * sig[k][:, None]
        ok = np.all((p >= 0.0) & (p < space), axis=1)
        p = p[ok]
        take = min(p.shape[0], n - got)
        out[got:got + take] = p[:take]
        got += take
    vel = (rng.standard_normal((n, 3)) * 2.0).astype(np.float32)
    return out, vel
