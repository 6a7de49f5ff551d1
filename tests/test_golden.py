"""Parity against golden vectors from the reference's own CUDA kernels.

tests/golden/make_golden.py replays the gvdb-voxels kernels on a B200
(oracle/ref_driver.cu) and stores every intermediate result of four seeded
cases. The CPU tests pin the oracle to those vectors. The GPU tests run the
same sequences through libgvdb2's C-ABI.

Equality rules:
  - topology, atlas assignment, neighbour table, point->brick assignment and
    subcell lists are compared bit for bit;
  - the 16-bit subcell entries of InsertPointsSubcell_FP16 too, for libgvdb2,
    which quantizes with the same approximate division as the reference's
    --use_fast_math build; the oracle divides exactly (IEEE), so an entry
    may differ from the reference's by one unit there;
  - float channels are compared within REL_TOL. The reference is built with
    --use_fast_math. Level sets from 16-bit lists also allow two float
    spacings at the coordinates' magnitude (fp16_level_set_tol).
  - the reference leaves two things undefined, so only their defined part is
    compared:
      - the brick coordinates of unused atlas-map entries;
      - the order of points inside one brick or subcell, which follows its
        atomics.
"""
import os

import numpy as np
import pytest

import make_golden as mg
from _helpers import REL_TOL, assert_nodes_equal, fp16_level_set_tol, interior, rel_err

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {c["name"]: c for c in mg.cases()}


def load(name):
    return np.load(os.path.join(HERE, name + ".npz"))


def last_points(g):
    return g[f"pts{int(g['npts_sets']) - 1}"]


def test_fixture_inputs_match_generator():
    """The committed fixtures hold exactly the points the generator makes."""
    for name, c in CASES.items():
        g = load(name)
        assert int(g["npts_sets"]) == len(c["pts"])
        for k, p in enumerate(c["pts"]):
            assert np.array_equal(g[f"pts{k}"], p), (name, k)
        mg.check_inputs(c)


def assert_atlas_map_equal(got, want):
    assert len(got) == len(want)
    assert np.array_equal(got["mLeafID"], want["mLeafID"])
    used = want["mLeafID"] >= 0
    assert np.array_equal(got["mPos"][used], want["mPos"][used])


def sort_groups(entries, off, cnt, by_column=False):
    """Entries of each subcell list in lexicographic order, or each column
    sorted on its own (entries that may differ by one unit can swap places
    in a lexicographic order; per column, sorting keeps |a - b| <= 1)."""
    out = entries.copy()
    for a, c in zip(off.tolist(), cnt.tolist()):
        blk = out[a:a + c]
        out[a:a + c] = np.sort(blk, axis=0) if by_column else blk[np.lexsort(blk.T[::-1])]
    return out


def assert_poff_permutation(pnode, poff):
    """poff numbers the points of each brick 0..count-1 in some order."""
    ok = pnode >= 0
    order = np.lexsort((poff[ok], pnode[ok]))
    pn, po = pnode[ok][order], poff[ok][order]
    starts = np.r_[0, np.nonzero(np.diff(pn))[0] + 1]
    rank = np.arange(len(pn)) - np.repeat(starts, np.diff(np.r_[starts, len(pn)]))
    assert np.array_equal(po, rank)


class Steps:
    """One golden sequence, driven through either the oracle or libgvdb2."""

    def __init__(self, g, case):
        self.g = g
        self.case = case
        self.ops = case["ops"]
        self.pts = last_points(g)
        self.n = len(self.pts)

    def check(self, run):
        g = self.g
        cnt = g["counts_topology"]
        depth = int(cnt[7])
        for k in range(int(g["npts_sets"])):
            run.rebuild(g[f"pts{k}"], float(g["radius"]))
        assert run.depth() == depth and run.top_level() == int(cnt[8])
        assert [run.pool_count(l) for l in range(5)] == cnt[:5].tolist()
        assert run.used_leaves() == int(cnt[5])
        for lev in range(depth + 1):
            assert_nodes_equal(run.nodes(lev), g[f"nodes{lev}"], lev)
            if lev > 0:
                assert np.array_equal(run.childlists(lev), g[f"clist{lev}"]), f"child lists level {lev}"
        run.update_atlas()
        assert run.atlas_slots() == int(g["counts_atlas"][6])
        assert_nodes_equal(run.nodes(0), g["nodes0_atlas"], 0)
        assert_atlas_map_equal(run.atlas_map(), g["atlas_map"])
        if "subcell_fp16" in self.ops:
            self.check_fp16(run)
        if "insert" not in self.ops:
            return
        for c in range(self.case["chans"]):
            run.clear(c)
        pnode, poff, gcnt = run.insert(self.pts)
        assert np.array_equal(pnode, g["pnode"])
        assert np.array_equal(gcnt[:len(g["gcnt"])], g["gcnt"])
        assert_poff_permutation(pnode, poff)
        if "scatter" not in self.ops:
            return
        run.scatter(self.pts, pnode)
        assert rel_err(run.tiles(0), g["tiles_scatter"]) <= REL_TOL
        run.neighbors_update()
        assert np.array_equal(run.neighbors(), g["neighbors"])
        run.faces(0)
        assert rel_err(run.tiles(0), g["tiles_faces"]) <= REL_TOL
        run.apron(0, mg.APRON_SCATTER_BOUND)
        assert rel_err(run.tiles(0), g["tiles_apron_scatter"]) <= REL_TOL
        ln = run.subcell(self.pts)
        assert ln == int(g["sc_len"])
        sc_cnt, sc_nid = run.subcell_lists(len(g["sc_cnt"]))
        assert np.array_equal(sc_cnt, g["sc_cnt"]) and np.array_equal(sc_nid, g["sc_nid"])
        run.levelset(ln)
        assert rel_err(interior(run.tiles(0), 1), interior(g["tiles_levelset"], 1)) <= REL_TOL
        run.apron(mg.LEVELSET["chan"], mg.APRON_LEVELSET_BOUND)
        assert rel_err(run.tiles(0), g["tiles_apron_levelset"]) <= REL_TOL
        run.density(ln)
        assert rel_err(interior(run.tiles(1), 1), interior(g["tiles_density"], 1)) <= REL_TOL


    def check_fp16(self, run):
        g = self.g
        ln = run.subcell_fp16(self.pts)
        assert ln == int(g["sc16_len"])
        cnt, nid = run.subcell_lists(len(g["sc16_cnt"]))
        assert np.array_equal(cnt, g["sc16_cnt"]) and np.array_equal(nid, g["sc16_nid"])
        by_column = run.Q16_TOL > 0
        q = sort_groups(run.fp16_entries(ln), g["sc16_off"], g["sc16_cnt"], by_column)
        ref = sort_groups(g["sc16_q"], g["sc16_off"], g["sc16_cnt"], by_column)
        diff = np.abs(q.astype(np.int32) - ref.astype(np.int32))
        assert diff.max() <= run.Q16_TOL, f"16-bit entries differ by up to {diff.max()}"
        run.levelset_fp16(ln)
        want = interior(g["tiles_levelset_fp16"], 1)
        tol = fp16_level_set_tol(self.pts, want, run.Q16_TOL)
        assert np.abs(interior(run.tiles(0), 1) - want).max() <= tol
        run.apron(mg.LEVELSET["chan"], mg.APRON_LEVELSET_BOUND)
        assert np.abs(run.tiles(0) - g["tiles_apron_levelset_fp16"]).max() <= tol


class OracleRun:
    Q16_TOL = 1  # exact division against the reference's approximate one
    def __init__(self, oracle_mod, case):
        self.o = oracle_mod.Oracle()
        self.o.configure(*case["cfg"])
        for c in range(case["chans"]):
            self.o.add_channel(c, case["apron"])
        self.__dict__.update({k: getattr(self.o, k) for k in (
            "depth", "top_level", "pool_count", "used_leaves", "nodes", "childlists", "update_atlas",
            "atlas_slots", "atlas_map", "neighbors")})

    def rebuild(self, pts, radius):
        assert self.o.rebuild_topology(pts, radius) == 0

    def clear(self, c):
        self.o.clear_channel(c)

    def insert(self, pts):
        return self.o.insert_points(pts)

    def scatter(self, pts, pnode):
        s = mg.SCATTER
        self.o.scatter_density(pts, s["radius"], s["amp"], (0, 0, 0), s["expand"], pnode)

    def tiles(self, c):
        return self.o.atlas(c)

    def neighbors_update(self):
        self.o.update_neighbors()

    def faces(self, c):
        self.o.update_apron_faces(c)

    def apron(self, c, bound):
        self.o.update_apron(c, bound)

    def subcell(self, pts):
        return self.o.insert_points_subcell(mg.SUBCELL["size"], pts, mg.SUBCELL["radius"])

    def subcell_lists(self, m):
        cnt, nid, _ = self.o.subcells()
        return cnt, nid

    def levelset(self, ln):
        self.o.gather_level_set(mg.SUBCELL["size"], mg.LEVELSET["radius"], mg.LEVELSET["chan"])

    def density(self, ln):
        self.o.gather_density(mg.SUBCELL["size"], mg.DENSITY["radius"], mg.DENSITY["chan"])

    def subcell_fp16(self, pts):
        return self.o.insert_points_subcell_fp16(mg.SUBCELL["size"], pts, mg.SUBCELL["radius"])

    def fp16_entries(self, ln):
        return self.o.subcell_lists()[1]

    def levelset_fp16(self, ln):
        self.o.gather_level_set_fp16(mg.SUBCELL["size"], mg.LEVELSET["radius"], mg.LEVELSET["chan"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference(oracle_mod, name):
    Steps(load(name), CASES[name]).check(OracleRun(oracle_mod, CASES[name]))


class GpuRun:
    Q16_TOL = 0

    def __init__(self, gvdb2_mod, case):
        self.v = gvdb2_mod.VolumeGVDB(0)
        self.v.Configure(*case["cfg"])
        for c in range(case["chans"]):
            self.v.AddChannel(c, gvdb2_mod.T_FLOAT, case["apron"])
        self._t = None

    def _set(self, pts):
        import torch
        self._t = torch.from_numpy(np.ascontiguousarray(pts, np.float32)).cuda()
        self.v.SetPoints(self._t)
        return len(pts)

    def rebuild(self, pts, radius):
        self.v.RebuildTopology(self._set(pts), radius)

    def depth(self):
        return int(self.v.info().depth)

    def top_level(self):
        return int(self.v.info().top_level)

    def pool_count(self, lev):
        return self.v.getNumTotalNodes(lev)

    def used_leaves(self):
        return self.v.getNumUsedNodes(0)

    def nodes(self, lev):
        return self.v.nodes(lev)

    def childlists(self, lev):
        return self.v.childlists(lev)

    def update_atlas(self):
        self.v.UpdateAtlas()

    def atlas_slots(self):
        return int(self.v.info().atlas_slots)

    def atlas_map(self):
        return self.v.atlas_map()

    def clear(self, c):
        self.v.ClearChannel(c)

    def insert(self, pts):
        n = self._set(pts)
        self.v.InsertPoints(n)
        return self.v.point_nodes(n)

    def scatter(self, pts, pnode):
        s = mg.SCATTER
        self.v.ScatterDensity(len(pts), s["radius"], s["amp"], (0, 0, 0), s["expand"])

    def tiles(self, c):
        return self.v.atlas(c)

    def neighbors_update(self):
        self.v.UpdateNeighbors()

    def neighbors(self):
        return self.v.neighbors()

    def faces(self, c):
        self.v.UpdateApronFaces(c)

    def apron(self, c, bound):
        self.v.UpdateApron(c, bound)

    def subcell(self, pts):
        return self.v.InsertPointsSubcell(mg.SUBCELL["size"], len(pts), mg.SUBCELL["radius"])

    def subcell_lists(self, m):
        cnt, nid, _ = self.v.subcells(m)
        return cnt, nid

    def levelset(self, ln):
        self.v.GatherLevelSet(mg.SUBCELL["size"], len(self._t), mg.LEVELSET["radius"], (0, 0, 0), ln,
                              mg.LEVELSET["chan"])

    def density(self, ln):
        self.v.GatherDensity(mg.SUBCELL["size"], len(self._t), mg.DENSITY["radius"], (0, 0, 0), ln,
                             mg.DENSITY["chan"])

    def subcell_fp16(self, pts):
        return self.v.InsertPointsSubcell_FP16(mg.SUBCELL["size"], len(pts), mg.SUBCELL["radius"])

    def fp16_entries(self, ln):
        return self.v.subcell_points_fp16(ln)

    def levelset_fp16(self, ln):
        self.v.GatherLevelSet_FP16(mg.SUBCELL["size"], len(self._t), mg.LEVELSET["radius"], (0, 0, 0), ln,
                                   mg.LEVELSET["chan"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_reference(gvdb2_mod, name):
    Steps(load(name), CASES[name]).check(GpuRun(gvdb2_mod, CASES[name]))
