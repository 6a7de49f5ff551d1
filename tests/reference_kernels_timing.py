"""Times the reference's own CUDA kernels against libgvdb2 on one B200.

Both sides run the reference's point path on the same inputs:
RebuildTopology -> UpdateAtlas -> InsertPoints -> ScatterDensity ->
UpdateApron -> InsertPointsSubcell -> GatherDensity.

  - The reference runs as oracle/_ref/libgvdbref.so. That is the gvdb-voxels
    kernel module compiled for sm_100a behind the host restatement in
    oracle/ref_driver.cu (`make -C oracle ref`).
  - libgvdb2 runs the same calls through its C-ABI.

Inputs: the dynamic SPH-like workload. It has 4,194,304 points on a jittered
lattice filling a 256x128x256-voxel block, advected by 0.1*v before each
step. The reference's calls synchronise the device and include its host
loops (node allocation, pool commits, atlas assignment). So every stage on
both sides is timed as host wall time around the call, followed by a device
synchronise. Each stage reports the median over the timed steps.

The inputs satisfy the conditions under which the reference kernels stay in
bounds; make_golden.check_inputs tests them on the CPU before any launch.

Run (GPU box):  python tests/reference_kernels_timing.py [--steps 5] [--out F]
Prints one JSON object.
"""
import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, os.path.join(ROOT, "gvdb-voxels_b200"))

STAGES = ["rebuild", "atlas", "insert", "scatter", "apron", "subcell", "gather"]
RADIUS = 2.0          # RebuildTopology / InsertPointsSubcell radius
SPLAT_R = 1.0         # ScatterDensity / GatherDensity radius
SUBCELL = 4


def ref_pipeline(mg, pts_steps):
    import ctypes
    R = mg.Ref(0)
    R("rd_configure", 3, 3, 3, 3, 3)
    R("rd_add_channel", 0, 1)
    zero = (ctypes.c_float * 3)(0, 0, 0)
    times = {k: [] for k in STAGES}
    extra = {}
    for p in pts_steps:
        n = len(p)
        R("rd_set_points", p.ctypes.data, n)
        R("rd_request_full_rebuild")  # full branch every step, as the bench's RequestFullRebuild(true)
        t = {}
        t0 = time.perf_counter()
        R("rd_rebuild_topology", n, RADIUS, zero)
        t["rebuild"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        R("rd_update_atlas")
        R("rd_clear_channel", 0)
        t["atlas"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        R("rd_insert_points", n, zero)
        t["insert"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        R("rd_scatter_density", n, SPLAT_R, 1.0, zero, 0)
        t["scatter"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        R("rd_update_apron", 0, 0.0)
        t["apron"] = time.perf_counter() - t0
        ln = ctypes.c_int(0)
        t0 = time.perf_counter()
        R("rd_insert_points_subcell", SUBCELL, n, RADIUS, zero, ctypes.byref(ln))
        t["subcell"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        R("rd_gather_density", n, SPLAT_R, 0, 0)
        t["gather"] = time.perf_counter() - t0
        for k in STAGES:
            times[k].append(t[k])
        extra = {"counts": R.counts().tolist(), "subcell_len": ln.value}
    R.close()
    return times, extra


def our_pipeline(pts_steps):
    import torch
    import gvdb2
    v = gvdb2.VolumeGVDB(0)
    v.Configure(3, 3, 3, 3, 3)
    v.AddChannel(0, gvdb2.T_FLOAT, 1)
    times = {k: [] for k in STAGES}
    sync = torch.cuda.synchronize
    extra = {}
    for p in pts_steps:
        n = len(p)
        t_pts = torch.from_numpy(p).cuda()
        v.SetPoints(t_pts)
        sync()
        t = {}
        t0 = time.perf_counter()
        v.RequestFullRebuild(True)
        v.RebuildTopology(n, RADIUS)
        sync()
        t["rebuild"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        v.UpdateAtlas()
        v.ClearChannel(0)
        sync()
        t["atlas"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        v.InsertPoints(n)
        sync()
        t["insert"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        v.ScatterDensity(n, SPLAT_R, 1.0, (0, 0, 0), False)
        sync()
        t["scatter"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        v.UpdateApron(0, 0.0)
        sync()
        t["apron"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        ln = v.InsertPointsSubcell(SUBCELL, n, RADIUS)
        sync()
        t["subcell"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        v.GatherDensity(SUBCELL, n, SPLAT_R, (0, 0, 0), ln, 0)
        sync()
        t["gather"] = time.perf_counter() - t0
        for k in STAGES:
            times[k].append(t[k])
        inf = v.info()
        extra = {"counts": [int(inf.pool_count[l]) for l in range(5)], "used": int(inf.used_leaves),
                 "subcell_len": ln}
    v.close()
    return times, extra


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--sites", default="256,64,256")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    import make_golden as mg
    import gvdb2.workloads as wl
    sites = tuple(int(x) for x in a.sites.split(","))
    pos, vel = wl.dam_block(sites=sites)
    steps = []
    p = pos
    for _ in range(a.warmup + a.steps):
        p = (p + np.float32(0.1) * vel).astype(np.float32)
        steps.append(np.ascontiguousarray(p))
    case = dict(cfg=(3, 3, 3, 3, 3), radius=RADIUS, pts=steps, ops=[])
    mg.check_inputs(case)  # CPU: every kernel box inside the root, top level = root

    ref_t, ref_x = ref_pipeline(mg, steps)
    our_t, our_x = our_pipeline(steps)
    res = {"workload": f"dam block {sites[0]}x{sites[1]}x{sites[2]} sites = {len(pos)} points, advected 0.1*v per step",
           "steps_timed": a.steps, "timing": "host wall time around each synchronised call, median ms",
           "reference": {}, "ours": {}, "speedup": {}}
    for k in STAGES:
        r = 1e3 * statistics.median(ref_t[k][a.warmup:])
        o = 1e3 * statistics.median(our_t[k][a.warmup:])
        res["reference"][k] = round(r, 3)
        res["ours"][k] = round(o, 3)
        res["speedup"][k] = round(r / o, 2) if o > 0 else None
    rt, ot = sum(res["reference"].values()), sum(res["ours"].values())
    res["reference"]["total"] = round(rt, 3)
    res["ours"]["total"] = round(ot, 3)
    res["speedup"]["total"] = round(rt / ot, 2)
    res["points_per_s"] = {"reference": len(pos) / (rt / 1e3), "ours": len(pos) / (ot / 1e3)}
    res["check"] = {"reference": ref_x, "ours": our_x}
    txt = json.dumps(res)
    print(txt, flush=True)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
