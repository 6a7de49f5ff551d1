"""Generates the golden vectors that pin the CPU oracle to the reference.

It replays the reference's own CUDA kernels on a B200. They sit in
oracle/_ref/libgvdbref.so, which `make -C oracle ref` compiles from the
gvdb-voxels kernel sources behind the host restatement in
oracle/ref_driver.cu. The script writes one compressed .npz per case into
--out (default tests/golden/). The replay library is prebuilt, so this
script reads nothing from the reference tree at run time.

Every input is seeded. Before any launch it is checked on the CPU against the
conditions under which the reference kernels stay in bounds:
  - every point is positive;
  - the points span at least two nodes one level below the root, so the
    kernels' top level is the root;
  - every box the point kernels visit lies inside the root node;
  - scatter inputs put at most one point in any voxel (the reference splat
    is an unsynchronised read-modify-write).

Run:  python tests/golden/make_golden.py [--out DIR] [--device 0]
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(REPO, "oracle", "_ref", "libgvdbref.so")

NODE_DTYPE = np.dtype([
    ("mLev", np.uint8), ("mFlags", np.uint8), ("mPriority", np.uint8), ("pad", np.uint8),
    ("mPos", np.int32, 3), ("mValue", np.int32, 3), ("mVRange", np.float32, 3),
    ("mParent", np.uint64), ("mChildList", np.uint64), ("mMask", np.uint64),
])
AMAP_DTYPE = np.dtype([("mPos", np.int32, 3), ("mLeafID", np.int32)])

# ---------------------------------------------------------------- cases


def _shell(n, seed, center, r_in, r_out):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = rng.uniform(r_in, r_out, size=(n, 1))
    return (np.asarray(center) + d * r).astype(np.float32)


def _one_per_voxel(p):
    _, first = np.unique(np.floor(p).astype(np.int64), axis=0, return_index=True)
    return p[np.sort(first)]


def _box(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)


def cases():
    """(name, config q4..q0, apron, channels, radius, points, ops)."""
    shell = _one_per_voxel(_shell(900, 11, (512.3, 511.6, 512.4), 17.0, 21.0))
    blob0 = _shell(700, 12, (511.2, 512.5, 510.8), 6.0, 26.0)
    drift = np.zeros_like(blob0)
    drift[: len(blob0) // 2, 0] = 5.25  # half of the cloud moves by 5.25 voxels in x
    blob1 = (blob0 + drift).astype(np.float32)
    return [
        dict(name="shell_splat_levelset", cfg=(3, 3, 3, 3, 3), apron=1, chans=2, radius=2.0, pts=[shell],
             ops=["topology", "atlas", "insert", "scatter", "faces", "apron_scatter", "subcell", "levelset",
                  "apron_levelset", "density"]),
        dict(name="incremental_drift", cfg=(3, 3, 3, 3, 3), apron=1, chans=1, radius=2.0,
             pts=[blob0, blob0, blob1], ops=["topology", "atlas"]),
        dict(name="leaf32_r3", cfg=(3, 3, 3, 4, 5), apron=1, chans=1, radius=3.0,
             pts=[_box(300, 13, 100.0, 1400.0)], ops=["topology", "atlas", "insert"]),
        dict(name="deep_r0", cfg=(3, 3, 3, 3, 3), apron=1, chans=1, radius=0.0,
             pts=[_box(400, 14, 100.0, 5000.0)], ops=["topology", "atlas", "insert"]),
        dict(name="blob_fp16", cfg=(3, 3, 3, 3, 3), apron=1, chans=1, radius=2.0,
             pts=[_shell(800, 15, (511.7, 512.2, 512.9), 4.0, 24.0)],
             ops=["topology", "atlas", "subcell_fp16", "levelset_fp16", "apron_levelset_fp16"]),
    ]


# Parameters of the point kernels, shared with the tests that read the goldens.
SCATTER = dict(radius=1.0, amp=1.0, expand=False)
APRON_SCATTER_BOUND = 0.25
SUBCELL = dict(size=4, radius=2.0)
LEVELSET = dict(radius=1.0, chan=0)
APRON_LEVELSET_BOUND = 3.0
DENSITY = dict(radius=1.0, chan=1)

# ---------------------------------------------------------- input checks


def _ranges(cfg):
    logdim = [cfg[4], cfg[3], cfg[2], cfg[1], cfg[0]]
    res = [1 << max(d, 1) for d in logdim]
    out, r = [], 1
    for l in range(5):
        r *= res[l]
        out.append(r)
    return out


def check_inputs(case):
    """CPU checks that keep every reference kernel of the case in bounds."""
    rng = _ranges(case["cfg"])
    margin = 3.0 * case["radius"] + 2.0 + SUBCELL["size"]
    depths = []
    for p in case["pts"]:
        assert np.all(p > 0), "non-positive point"
        lo = np.maximum(p.min(0) - 1, 0)
        hi = np.maximum(p.max(0) + 2, 0)
        depth = next(l for l in range(5) if np.all((lo.astype(int) // rng[l]) == (hi.astype(int) // rng[l])))
        assert 1 <= depth <= 4, f"depth {depth}"
        below = set(map(tuple, (p.astype(np.int64) // rng[depth - 1]).tolist()))
        assert len(below) >= 2, "points inside one node below the root: the top level would not be the root"
        root = (lo.astype(int) // rng[depth]) * rng[depth]
        assert np.all(p - margin >= root) and np.all(p + margin < root + rng[depth]), "box leaves the root"
        depths.append(depth)
    if "scatter" in case["ops"]:
        v = np.floor(case["pts"][-1]).astype(np.int64)
        assert len(np.unique(v, axis=0)) == len(v), "two points in one voxel"
    return depths


# ------------------------------------------------------------- replay


class Ref:
    def __init__(self, device):
        self.L = ctypes.CDLL(REF_LIB)
        L = self.L
        vp, i32, f32, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_longlong
        fp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
        sig = {
            "rd_create": (vp, [i32]), "rd_destroy": (None, [vp]),
            "rd_configure": (i32, [vp, i32, i32, i32, i32, i32]), "rd_add_channel": (i32, [vp, i32, i32]),
            "rd_set_points": (i32, [vp, vp, i32]), "rd_rebuild_topology": (i32, [vp, i32, f32, fp]),
            "rd_update_atlas": (i32, [vp]), "rd_clear_channel": (i32, [vp, i32]),
            "rd_request_full_rebuild": (i32, [vp]),
            "rd_insert_points": (i32, [vp, i32, fp]),
            "rd_copy_point_nodes": (i32, [vp, vp, vp, i32, vp, i32]),
            "rd_scatter_density": (i32, [vp, i32, f32, f32, fp, i32]),
            "rd_update_apron": (i32, [vp, i32, f32]), "rd_update_neighbors": (i32, [vp]),
            "rd_copy_neighbors": (i32, [vp, vp, i64]), "rd_update_apron_faces": (i32, [vp, i32]),
            "rd_insert_points_subcell": (i32, [vp, i32, i32, f32, fp, ip]),
            "rd_copy_subcells": (i32, [vp, vp, vp, vp, vp, i64, i64]),
            "rd_gather_density": (i32, [vp, i32, f32, i32, i32]),
            "rd_gather_level_set": (i32, [vp, i32, f32, i32, i32]),
            "rd_insert_points_subcell_fp16": (i32, [vp, i32, i32, f32, fp, ip]),
            "rd_copy_subcells_fp16": (i32, [vp, vp, i64]),
            "rd_gather_level_set_fp16": (i32, [vp, i32, f32, i32]),
            "rd_get_counts": (i32, [vp, vp]), "rd_copy_nodes": (i32, [vp, i32, vp, i64]),
            "rd_copy_childlists": (i32, [vp, i32, vp, i64]), "rd_copy_atlas_map": (i32, [vp, vp, i64]),
            "rd_copy_atlas_tiles": (i32, [vp, i32, vp, i64]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype, f.argtypes = r, a
        self.h = L.rd_create(device)
        assert self.h, "rd_create failed"

    def __call__(self, fn, *args):
        rc = getattr(self.L, fn)(self.h, *args)
        if rc:
            raise RuntimeError(f"{fn} returned {rc}")

    def close(self):
        self.L.rd_destroy(self.h)

    def counts(self):
        c = np.zeros(9, np.int64)
        self("rd_get_counts", c.ctypes.data)
        return c

    def nodes(self, lev, count):
        out = np.zeros(count, NODE_DTYPE)
        self("rd_copy_nodes", lev, out.ctypes.data, out.nbytes)
        return out

    def childlists(self, lev, count, res):
        out = np.zeros((count, res ** 3), np.uint64)
        self("rd_copy_childlists", lev, out.ctypes.data, out.nbytes)
        return out

    def tiles(self, chan, slots, t):
        out = np.zeros((slots, t, t, t), np.float32)
        self("rd_copy_atlas_tiles", chan, out.ctypes.data, out.size)
        return out


def _f3(v):
    return (ctypes.c_float * 3)(*v)


def run_case(case, device):
    depths = check_inputs(case)
    cfg = case["cfg"]
    res = [1 << max(d, 1) for d in (cfg[4], cfg[3], cfg[2], cfg[1], cfg[0])]
    out = dict(cfg=np.array(cfg), apron=case["apron"], radius=np.float32(case["radius"]))
    R = Ref(device)
    try:
        R("rd_configure", *cfg)
        for c in range(case["chans"]):
            R("rd_add_channel", c, case["apron"])
        zero = _f3((0, 0, 0))
        for k, p in enumerate(case["pts"]):
            p = np.ascontiguousarray(p, np.float32)
            out[f"pts{k}"] = p
            R("rd_set_points", p.ctypes.data, len(p))
            R("rd_rebuild_topology", len(p), float(case["radius"]), zero)
        pts = np.ascontiguousarray(case["pts"][-1], np.float32)
        n = len(pts)
        out["npts_sets"] = len(case["pts"])
        cnt = R.counts()
        depth = int(cnt[7])
        assert depth == depths[-1], (depth, depths)
        out["counts_topology"] = cnt
        for lev in range(depth + 1):
            out[f"nodes{lev}"] = R.nodes(lev, int(cnt[lev]))
            if lev > 0:
                out[f"clist{lev}"] = R.childlists(lev, int(cnt[lev]), res[lev])
        R("rd_update_atlas")
        cnt = R.counts()
        out["counts_atlas"] = cnt
        out["nodes0_atlas"] = R.nodes(0, int(cnt[0]))
        slots = int(cnt[6])
        t = res[0] + 2 * case["apron"]
        cap = 16 * 16 * int(np.ceil(max(slots, 1) / 256.0))
        amap = np.zeros(cap, AMAP_DTYPE)
        R("rd_copy_atlas_map", amap.ctypes.data, amap.nbytes // 4)
        out["atlas_map"] = amap
        ops = case["ops"]
        if "insert" in ops:
            for c in range(case["chans"]):
                R("rd_clear_channel", c)
            R("rd_insert_points", n, zero)
            pnode = np.zeros(n, np.int32)
            poff = np.zeros(n, np.int32)
            gcnt = np.zeros(max(slots, 1), np.int32)
            R("rd_copy_point_nodes", pnode.ctypes.data, poff.ctypes.data, n, gcnt.ctypes.data, slots)
            out["pnode"], out["poff"], out["gcnt"] = pnode, poff, gcnt[:slots]
        if "scatter" in ops:
            R("rd_scatter_density", n, SCATTER["radius"], SCATTER["amp"], zero, int(SCATTER["expand"]))
            out["tiles_scatter"] = R.tiles(0, slots, t)
        if "faces" in ops:
            R("rd_update_neighbors")
            nbr = np.zeros((int(cnt[0]), 6), np.int32)
            R("rd_copy_neighbors", nbr.ctypes.data, nbr.size)
            out["neighbors"] = nbr
            R("rd_update_apron_faces", 0)
            out["tiles_faces"] = R.tiles(0, slots, t)
        if "apron_scatter" in ops:
            R("rd_update_apron", 0, APRON_SCATTER_BOUND)
            out["tiles_apron_scatter"] = R.tiles(0, slots, t)
        if "subcell" in ops:
            ln = ctypes.c_int(0)
            R("rd_insert_points_subcell", SUBCELL["size"], n, SUBCELL["radius"], zero, ctypes.byref(ln))
            per = (res[0] // SUBCELL["size"]) ** 3
            m = per * int(cnt[5])
            sc_cnt = np.zeros(m, np.int32)
            sc_off = np.zeros(m, np.int32)
            sc_nid = np.zeros(m, np.int32)
            sc_pts = np.zeros((max(ln.value, 1), 3), np.float32)
            R("rd_copy_subcells", sc_cnt.ctypes.data, sc_off.ctypes.data, sc_nid.ctypes.data, sc_pts.ctypes.data,
              m, len(sc_pts))
            # order inside one subcell follows atomics: sort each list
            for s in range(m):
                a, b = sc_off[s], sc_off[s] + sc_cnt[s]
                blk = sc_pts[a:b]
                sc_pts[a:b] = blk[np.lexsort(blk.T[::-1])]
            out.update(sc_len=ln.value, sc_cnt=sc_cnt, sc_off=sc_off, sc_nid=sc_nid, sc_pts=sc_pts[:ln.value])
        if "levelset" in ops:
            R("rd_gather_level_set", n, LEVELSET["radius"], LEVELSET["chan"], 0)
            out["tiles_levelset"] = R.tiles(LEVELSET["chan"], slots, t)
        if "apron_levelset" in ops:
            R("rd_update_apron", LEVELSET["chan"], APRON_LEVELSET_BOUND)
            out["tiles_apron_levelset"] = R.tiles(LEVELSET["chan"], slots, t)
        if "density" in ops:
            R("rd_gather_density", n, DENSITY["radius"], DENSITY["chan"], 0)
            out["tiles_density"] = R.tiles(DENSITY["chan"], slots, t)
        if "subcell_fp16" in ops:
            ln = ctypes.c_int(0)
            R("rd_insert_points_subcell_fp16", SUBCELL["size"], n, SUBCELL["radius"], zero, ctypes.byref(ln))
            per = (res[0] // SUBCELL["size"]) ** 3
            m = per * int(cnt[5])
            sc_cnt = np.zeros(m, np.int32)
            sc_off = np.zeros(m, np.int32)
            sc_nid = np.zeros(m, np.int32)
            unused = np.zeros((1, 3), np.float32)  # the float lists are not written by the 16-bit insert
            R("rd_copy_subcells", sc_cnt.ctypes.data, sc_off.ctypes.data, sc_nid.ctypes.data, unused.ctypes.data,
              m, ln.value)
            q = np.zeros((max(ln.value, 1), 3), np.uint16)
            R("rd_copy_subcells_fp16", q.ctypes.data, len(q))
            for s in range(m):  # order inside one subcell follows atomics
                a, b = sc_off[s], sc_off[s] + sc_cnt[s]
                blk = q[a:b]
                q[a:b] = blk[np.lexsort(blk.T[::-1])]
            out.update(sc16_len=ln.value, sc16_cnt=sc_cnt, sc16_off=sc_off, sc16_nid=sc_nid, sc16_q=q[:ln.value])
        if "levelset_fp16" in ops:
            R("rd_gather_level_set_fp16", n, LEVELSET["radius"], LEVELSET["chan"])
            out["tiles_levelset_fp16"] = R.tiles(LEVELSET["chan"], slots, t)
        if "apron_levelset_fp16" in ops:
            R("rd_update_apron", LEVELSET["chan"], APRON_LEVELSET_BOUND)
            out["tiles_apron_levelset_fp16"] = R.tiles(LEVELSET["chan"], slots, t)
    finally:
        R.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--check-only", action="store_true", help="run the CPU input checks and exit")
    ap.add_argument("--only", default=None, help="generate this case only")
    a = ap.parse_args()
    for case in cases():
        if a.only and case["name"] != a.only:
            continue
        if a.check_only:
            print(case["name"], "depths", check_inputs(case))
            continue
        out = run_case(case, a.device)
        os.makedirs(a.out, exist_ok=True)
        path = os.path.join(a.out, case["name"] + ".npz")
        np.savez_compressed(path, **out)
        print(f"{case['name']}: {os.path.getsize(path)} bytes, counts {out['counts_atlas'].tolist()}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
