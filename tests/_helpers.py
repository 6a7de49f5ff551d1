"""Shared set-up for the parity tests: the same configuration and points
are run through the oracle (CPU) and, in GPU tests, through libgvdb2."""
import numpy as np

NODE_FIELDS = ("mLev", "mFlags", "mPos", "mValue", "mParent", "mChildList")
UNDEF64 = np.uint64(0xFFFFFFFFFFFFFFFF)

# Tolerance for float32 channels against the FP64 oracle: max |a-b| / max |b|.
REL_TOL = 1e-5


def fp16_level_set_tol(pts, ref, units=0):
    """Largest difference allowed between level sets gathered from 16-bit
    subcell lists: two float spacings at the largest coordinate -- the
    dequantized position q / 65535 * range + min is rounded to a float of
    that magnitude, and the approximate division of a --use_fast_math build
    rounds it differently from an exact one -- plus `units` quantization
    steps (entries that may differ by that many units: an exact division
    against an approximate one) plus REL_TOL of the values."""
    import numpy as np
    lo = np.maximum(pts.min(0) - 1.0, 0.0)  # the bounding box the entries are quantized over
    hi = np.maximum(pts.max(0) + 2.0, 0.0)
    step = float((hi - lo).max()) / 65535.0
    return (2.0 * float(np.spacing(np.float32(np.abs(pts).max()))) + units * step +
            REL_TOL * float(np.abs(ref).max()))


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-30)
    return float(np.max(np.abs(a - b))) / den if a.size else 0.0


def assert_nodes_equal(got, want, lev):
    assert got.shape == want.shape, f"level {lev}: {got.shape} nodes vs {want.shape}"
    for f in NODE_FIELDS:
        g, w = got[f], want[f]
        if not np.array_equal(g, w):
            bad = np.nonzero(np.any((g != w).reshape(len(g), -1), axis=1))[0]
            raise AssertionError(f"level {lev} field {f}: {len(bad)} nodes differ, first {bad[:5]}: "
                                 f"{g[bad[:3]]} vs {w[bad[:3]]}")


def make_oracle(oracle_mod, cfg=(3, 3, 3, 3, 3), chans=(0,), apron=1):
    o = oracle_mod.Oracle()
    o.configure(*cfg)
    for c in chans:
        o.add_channel(c, apron)
    return o


def shell_points(n, seed=0, r_in=96.0, r_out=100.0, center=(128.0, 128.0, 128.0)):
    import gvdb2.workloads as wl
    return wl.shell(n, seed, r_in, r_out, center)


def interior(tiles, apron):
    """Interior voxels of (slots, T, T, T) tiles."""
    t = tiles.shape[1]
    return tiles[:, apron:t - apron, apron:t - apron, apron:t - apron]


def apron_self_consistent(tiles, nodes0, slot_leaf_pos, res, apron, boundval=0.0):
    """Check every apron voxel equals (bit for bit) the interior voxel of the
    brick that owns its position, or boundval; returns the number checked.
    tiles: (slots, T, T, T) as (z, y, x); slot_leaf_pos: brick corner per slot."""
    tiles = np.asarray(tiles, np.float32)
    pos = np.asarray(slot_leaf_pos, np.int64)
    index = {tuple(p): i for i, p in enumerate(pos.tolist())}
    checked = 0
    a = apron
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dx == dy == dz == 0:
                    continue
                d = np.array([dx, dy, dz])
                nb = np.array([index.get(tuple(p), -1) for p in (pos + d * res).tolist()])
                sl_self, sl_nb = [], []
                for ax in (2, 1, 0):  # tile axes are (z, y, x)
                    dd = d[ax]
                    lo = {-1: 0, 0: a, 1: a + res}[dd]
                    hi = lo + (a if dd else res)
                    sl_self.append(slice(lo, hi))
                    sl_nb.append(slice(lo - dd * res, hi - dd * res))
                got = tiles[(slice(None),) + tuple(sl_self)]
                want = np.where((nb >= 0)[:, None, None, None], tiles[np.maximum(nb, 0)][(slice(None),) + tuple(sl_nb)],
                                np.float32(boundval))
                assert np.array_equal(got.view(np.uint32), want.astype(np.float32).view(np.uint32)), (dx, dy, dz)
                checked += got.size
    return checked
