"""The kernel splats' autotuner (gvdb2_autotune_scatter / _gather) and its
on-disk cache.

On the CPU: the cache file's entries round-trip through the library's
host-only cache calls, replace by key, refuse invalid settings and keys.
On the GPU: every candidate setting the autotuner tries gives the oracle's
scatter and gather within the splat tolerance on a point set with dense,
medium and light cells; the autotuner leaves the fastest on the volume,
writes it under the call's class, and a second volume with
GVDB2_OPT_AUTOTUNE takes it from the file and reproduces the first
volume's results bit for bit in deterministic mode."""
import ctypes

import numpy as np
import pytest

from _helpers import REL_TOL, interior, make_oracle, rel_err


def _lib():
    import gvdb2._lib as L
    return L.lib(), L.Tuning


def test_cache_round_trip(tmp_path):
    lib, Tuning = _lib()
    path = str(tmp_path / "tune.txt").encode()
    a, b = Tuning(1024, 2048, 16), Tuning(0, 4096, 32)
    assert lib.gvdb2_tune_cache_put(path, b"dev/148|scatter|k2|c4|r8|d10", ctypes.byref(a), 2.5) == 0
    assert lib.gvdb2_tune_cache_put(path, b"dev/148|gather|k2|c3|r8|d4", ctypes.byref(b), 0.75) == 0
    t, ms = Tuning(), ctypes.c_float()
    assert lib.gvdb2_tune_cache_get(path, b"dev/148|scatter|k2|c4|r8|d10", ctypes.byref(t), ctypes.byref(ms)) == 0
    assert (t.dense, t.slice, t.light, ms.value) == (1024, 2048, 16, 2.5)
    # replace by key; the other entry stays
    c = Tuning(256, 8192, 8)
    assert lib.gvdb2_tune_cache_put(path, b"dev/148|scatter|k2|c4|r8|d10", ctypes.byref(c), 1.5) == 0
    assert lib.gvdb2_tune_cache_get(path, b"dev/148|scatter|k2|c4|r8|d10", ctypes.byref(t), None) == 0
    assert (t.dense, t.slice, t.light) == (256, 8192, 8)
    assert lib.gvdb2_tune_cache_get(path, b"dev/148|gather|k2|c3|r8|d4", ctypes.byref(t), None) == 0
    assert (t.dense, t.slice, t.light) == (0, 4096, 32)
    lines = open(path.decode()).read().splitlines()
    assert len(lines) == 2 and all(len(ln.split("\t")) == 2 for ln in lines)
    # absent key, invalid settings and keys
    assert lib.gvdb2_tune_cache_get(path, b"nope", ctypes.byref(t), None) == 3
    for bad in (Tuning(100, 4096, 32), Tuning(512, 1000, 32), Tuning(512, 4096, 33), Tuning(512, 4096, -1)):
        assert lib.gvdb2_tune_cache_put(path, b"k", ctypes.byref(bad), 1.0) == 1
    assert lib.gvdb2_tune_cache_put(path, b"a\tb", ctypes.byref(a), 1.0) == 1
    assert lib.gvdb2_tune_cache_get(str(tmp_path / "missing.txt").encode(), b"k", ctypes.byref(t), None) == 3


def _mixed_points():
    """A Gaussian blob (cells of thousands of points at its centre) inside a
    sparse shell (cells of a few points)."""
    from _helpers import shell_points
    rng = np.random.default_rng(21)
    blob = np.clip(rng.normal(128.0, 5.0, (150_000, 3)), 1.0, 254.0).astype(np.float32)
    shell = shell_points(30_000, seed=22, r_in=60, r_out=70)
    return np.concatenate([blob, shell]).astype(np.float32)


SCATTER_CANDIDATES = [(0, 4096)] + [(d, s) for d in (256, 512, 1024, 2048) for s in (2048, 4096, 8192)]


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [1, 2])
def test_every_candidate_matches_oracle(gvdb2_mod, oracle_mod, kernel):
    import torch
    from test_gpu_topology import gpu_volume
    p = _mixed_points()
    n = len(p)
    w = np.random.default_rng(23).uniform(0.5, 2.0, n).astype(np.float32)
    chans = [0, 1]
    o = make_oracle(oracle_mod, chans=chans)
    assert o.rebuild_topology(p, 2.0) == 0
    o.update_atlas()
    o.scatter_kernel(kernel, p, chans, weight=w, attrs=[None, p[:, 0].copy()])
    want = [interior(o.atlas(c), 1) for c in chans]
    for c in chans:
        o.update_apron(c)
    g_want = o.gather_kernel(kernel, p, chans)
    v = gpu_volume(gvdb2_mod, p, chans=chans)
    v.RebuildTopology(n, 2.0)
    v.UpdateAtlas()
    tw = torch.from_numpy(w).cuda()
    tp = torch.from_numpy(p).cuda()
    for dense, slc in SCATTER_CANDIDATES:
        v.SetTuning(dense, slc, 32)
        v.ScatterKernel(kernel, n, chans, weight=tw, attrs=[None, (tp, 0)])
        for c in chans:
            e = rel_err(interior(v.atlas(c), 1), want[c])
            assert e < REL_TOL, f"dense {dense} slice {slc} channel {c}: rel err {e:.3e}"
    v.UpdateApron(-1, 0.0)
    for light in (0, 8, 16, 32):
        v.SetTuning(512, 4096, light)
        g = v.GatherKernel(kernel, n, chans).cpu().numpy()
        e = rel_err(g, g_want)
        assert e < REL_TOL, f"light {light}: rel err {e:.3e}"
    with pytest.raises(gvdb2_mod.GvdbError):
        v.SetTuning(512, 4000, 32)  # not a multiple of 128


@pytest.mark.gpu
def test_autotune_caches_and_reapplies(gvdb2_mod, tmp_path):
    import torch
    from test_gpu_topology import gpu_volume
    p = _mixed_points()
    n = len(p)
    path = str(tmp_path / "tune.txt")
    K = gvdb2_mod.KERNEL_CUBIC2

    def volume():
        v = gpu_volume(gvdb2_mod, p, chans=[0, 1, 2])
        v.SetDeterministic(True)
        v.SetTuneCache(path)
        v.RebuildTopology(n, 2.0)
        v.UpdateAtlas()
        return v

    tp = torch.from_numpy(p).cuda()
    attrs = [None, (tp, 0), (tp, 1)]
    a = volume()
    ts = a.AutotuneScatter(K, n, [0, 1, 2], weight=1.0, attrs=attrs)
    assert a.GetTuning()[:2] == ts[:2]
    _, tg = a.AutotuneGather(K, n, [0, 1, 2])
    assert a.GetTuning() == (ts[0], ts[1], tg[2])
    lines = open(path).read().splitlines()
    assert len(lines) == 2 and {ln.split("|")[1] for ln in lines} == {"scatter", "gather"}
    # results of the tuned volume are those of a plain call with its setting
    ref = [a.atlas(c).copy() for c in range(3)]
    g_ref = a.GatherKernel(K, n, [0, 1, 2]).cpu().numpy()

    b = volume()
    b.SetAutotune(True)
    b.SetTuning(512, 4096, 32)
    b.ScatterKernel(K, n, [0, 1, 2], weight=1.0, attrs=attrs)
    assert b.GetTuning()[:2] == ts[:2]
    g = b.GatherKernel(K, n, [0, 1, 2]).cpu().numpy()
    assert b.GetTuning() == a.GetTuning()
    for c in range(3):
        assert np.array_equal(b.atlas(c), ref[c])
    assert np.array_equal(g, g_ref)
