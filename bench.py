"""Benchmark of the point -> sparse-volume step on B200.

Default workload (the dynamic step the throughput target is stated on):
16,777,216 points on a jittered lattice (256 x 256 x 256 sites at spacing
(1, 0.5, 1)) filling a 256x128x256-voxel dam block, velocity ~ N(0,1),
Configure(3,3,3,3,3) (8^3 bricks, apron 1), channels density + 3 x velocity.
One step: advect p += 0.1 v -> RebuildTopology(N, 2.0) -> UpdateAtlas ->
cubic B-spline scatter (r = 2) of mass and momentum -> UpdateApron -> cubic
gather of the 3 velocity channels back to the points.

`python bench.py [--gpus N --steps K --warmup W]` prints one JSON line.  At
N = 1 the line also carries the rest of the metric, each measured in the same
run: the 4,194,304-point dynamic step, the incremental topology state
machine, the adjoint step against the forward step, the 64 batched clouds
against a per-cloud loop, and the reference's own CUDA kernels against this
library on the reference's point path.
`--impl reference` times the reference's host path (ActivateSpace topology,
host atlas, CPU splat and gather) on all host cores instead: the reference's
host library does not build here (it needs GL), so this is the CPU
restatement of that path.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gvdb-voxels_b200"))

METRIC = "points/s rebuild+scatter+gather at <=1e-5 err, % HBM peak; adjoint & batched vs plain"
DT = 0.1
RADIUS = 2.0

WORKLOADS = {
    "dam16m": dict(sites=(256, 256, 256), spacing=(1.0, 0.5, 1.0),
                   desc="dynamic SPH-like step: 16,777,216-pt jittered lattice (256x256x256 sites, spacing 1,0.5,1) "
                        "in a 256x128x256-voxel block, cubic B-spline r=2, density+3 vel channels"),
    "dam": dict(sites=(256, 64, 256), spacing=(1.0, 2.0, 1.0),
                desc="dynamic SPH-like step: 4,194,304-pt jittered lattice (256x64x256 sites, spacing 1,2,1) "
                     "in a 256x128x256-voxel block, cubic B-spline r=2, density+3 vel channels"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="the main line only (no 4M, incremental, adjoint, "
                                                              "batched or reference-kernel legs)")
    ap.add_argument("--incremental", action="store_true", help="reference state machine instead of full rebuilds")
    ap.add_argument("--leg", default=None, choices=list(EXTRA_LEGS),
                    help="one extra leg of the main line, alone (the main line runs each in a child process)")
    ap.add_argument("--quick", action="store_true", help="timed steps only (no baseline, e2e or launch count)")
    ap.add_argument("--sites", default=None, help="lattice sites x,y,z (smaller cases for profiling)")
    ap.add_argument("--workload", default="dam16m", choices=["dam16m", "dam", "batched", "adjoint", "sparse67m"],
                    help="dam16m: the contract line (dynamic step, 16,777,216 points); dam: the same step on "
                         "4,194,304 points; batched: 64 clouds, batch vs per-cloud loop; adjoint: the "
                         "differentiable splat, adjoint vs forward; sparse67m: the large sparse scene "
                         "(67,108,864-point Gaussian mixture, 32^3 bricks, forward + adjoint)")
    ap.add_argument("--points", type=int, default=0, help="sparse67m: fewer points (smaller cases for profiling)")
    ap.add_argument("--clouds", type=int, default=0, help="batched: the first K clouds only (smaller cases for "
                                                             "profiling)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_points(a):
    """(positions, velocities, description) of the dam-block workload."""
    import gvdb2.workloads as wl
    w = WORKLOADS[a.workload]
    sites = tuple(int(x) for x in a.sites.split(",")) if a.sites else w["sites"]
    pos, vel = wl.dam_block(sites=sites, spacing=w["spacing"])
    desc = w["desc"] if not a.sites else f"{w['desc']} (reduced to {sites[0]}x{sites[1]}x{sites[2]} sites)"
    return pos, vel, desc


L2_BYTES = 126 * 1000 * 1000  # B200 L2


def static_config(a, n, ws):
    """The workload as both arms name it (no measured quantities)."""
    desc = WORKLOADS[a.workload]["desc"] if not a.sites else f"{a.workload} sites {a.sites}"
    return {"workload": desc, "points_per_gpu": int(n),
            "rebuild": "incremental state machine" if a.incremental else "full rebuild every step",
            "l2": (f"inputs larger than L2 (positions, velocities and gathered velocities: {36 * n / 1e6:.0f} MB "
                   "per step, atlas not counted)" if 36 * n > L2_BYTES else
                   "inputs smaller than L2 (a reduced case for profiling; not a benchmark line)"),
            "parallelism": f"replicas x{ws}"}


class Pipeline:
    """The benchmark step over libgvdb2 (through the VolumeGVDB mirror)."""

    def __init__(self, device, pos_host, vel_host, full_rebuild=True):
        import torch
        import gvdb2
        self.torch = torch
        self.gvdb2 = gvdb2
        self.dev = f"cuda:{device}"
        self.n = pos_host.shape[0]
        self.pos0 = torch.from_numpy(pos_host).to(self.dev)
        self.vel = torch.from_numpy(vel_host).to(self.dev)
        self.pos = self.pos0.clone()
        self.out = torch.empty((self.n, 3), dtype=torch.float32, device=self.dev)
        self.full = full_rebuild
        v = gvdb2.VolumeGVDB(device)
        v.Configure(3, 3, 3, 3, 3)
        for c in range(4):
            v.AddChannel(c, gvdb2.T_FLOAT, 1)
        v.SetPoints(self.pos)
        self.v = v
        self.attrs = [None, (self.vel, 0), (self.vel, 1), (self.vel, 2)]

    def reset(self):
        self.pos.copy_(self.pos0)

    def use_buffers(self, pos, vel, out):
        """Run the next steps on these device buffers (positions, velocities, gather output)."""
        self.pos, self.vel, self.out = pos, vel, out
        self.attrs = [None, (vel, 0), (vel, 1), (vel, 2)]
        self.v.SetPoints(pos)

    def step(self):
        v, n, K = self.v, self.n, self.gvdb2.KERNEL_CUBIC2
        self.pos.add_(self.vel, alpha=DT)  # advect (the simulation's own update)
        v.SetPoints(self.pos)  # positions changed in place: the binning is redone
        if self.full:
            v.RequestFullRebuild(True)
        v.RebuildTopology(n, RADIUS)
        v.UpdateAtlas()
        v.ScatterKernel(K, n, [0, 1, 2, 3], weight=1.0, attrs=self.attrs)
        v.UpdateApron(-1, 0.0)
        v.GatherKernel(K, n, [1, 2, 3], out=self.out)

    def geometry(self):
        inf = self.v.info()
        U = sum(int(inf.pool_count[l]) for l in range(5))
        CL = sum(int(inf.pool_count[l]) * 8 * int(inf.res[l]) ** 3 for l in range(1, 5))
        return {"B": int(inf.atlas_slots), "U": U, "CL": CL, "T": int(inf.tile_res) ** 3, "R3": int(inf.res[0]) ** 3}


# ----------------------------------------------------------------------------
# The reference's host path on the CPU: the cpu_baseline leg and the
# reference arm.  The reference's host library does not build here (GL), so
# its path runs as the C restatement: ActivateSpace at every brick of each
# point's activation box (the host topology build), the host atlas
# assignment, then the splat, apron and gather loops.
# ----------------------------------------------------------------------------
_SHM = {}


def _host_step(pos, vel):
    """One step of the workload on the host path over (pos, vel); seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    t0 = time.perf_counter()
    o = oracle.Oracle()
    o.configure(3, 3, 3, 3, 3)
    for c in range(4):
        o.add_channel(c, 1)
    p = (pos + np.float32(DT) * vel).astype(np.float32)
    o.activate_points(p, RADIUS)
    o.update_atlas()
    o.scatter_kernel(oracle.KERNEL_CUBIC2, p, [0, 1, 2, 3], attrs=[None, vel[:, 0], vel[:, 1], vel[:, 2]])
    for c in range(4):
        o.update_apron(c, 0.0)
    o.gather_kernel(oracle.KERNEL_CUBIC2, p, [1, 2, 3])
    o.close()
    return time.perf_counter() - t0


def _attach(name, n):
    import numpy as np
    from multiprocessing import shared_memory
    if name not in _SHM:
        shm = shared_memory.SharedMemory(name=name)
        _SHM[name] = (shm, np.ndarray((n, 6), np.float32, buffer=shm.buf))
    return _SHM[name][1]


def _host_task(args):
    name, n, start, count = args
    buf = _attach(name, n)
    pv = buf[start:start + count]
    return _host_step(pv[:, :3].copy(), pv[:, 3:].copy())


def cpu_baseline(pos, vel, n):
    """The host path single-threaded on a contiguous sub-block of n points."""
    n = min(n, len(pos))
    dt = _host_step(pos[:n].copy(), vel[:n].copy())
    return {"value": n / dt, "unit": "points/s", "cores": 1, "kind": "port",
            "sample": f"one step over the first {n} lattice points (a contiguous slab of the block): host "
                      "ActivateSpace topology, host atlas, CPU cubic splat, apron and gather, single-threaded",
            "seconds": round(dt, 3)}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    import multiprocessing as mp
    import numpy as np
    from multiprocessing import shared_memory
    pos, vel, _ = workload_points(a)
    n = len(pos)
    cores = os.cpu_count() or 1
    per = min(262_144, max(1, n // cores))
    shm = shared_memory.SharedMemory(create=True, size=n * 24)
    try:
        buf = np.ndarray((n, 6), np.float32, buffer=shm.buf)
        buf[:, :3] = pos
        buf[:, 3:] = vel
        del pos, vel
        stride = max(per, (n - per) // max(1, cores - 1))
        tasks = [(shm.name, n, min(k * stride, n - per), per) for k in range(cores)]
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores) as pool:
            for _ in range(a.warmup):
                pool.map(_host_task, tasks)
            times = []
            for _ in range(a.steps):
                t0 = time.perf_counter()
                pool.map(_host_task, tasks)
                times.append(time.perf_counter() - t0)
        del buf
    finally:
        shm.close()
        shm.unlink()
    total = sum(times)
    value = per * cores * a.steps / total
    sample = (f"{cores} processes, each one step over its own contiguous slab of {per} lattice points per "
              f"timed step: host ActivateSpace topology (single-threaded per volume, as the reference), host "
              f"atlas, CPU cubic splat, apron and gather")
    line = {"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * total / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": static_config(a, n, ws),
            "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def stage_times(pipe, reps=7):
    """Median device time of each stage (one launch each for the splats)."""
    import torch
    v, n, K = pipe.v, pipe.n, pipe.gvdb2.KERNEL_CUBIC2

    def timed(f):
        f()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            f()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    def topo():
        v.RequestFullRebuild(True)
        v.RebuildTopology(n, RADIUS)
        v.UpdateAtlas()

    out = {"topology": timed(topo)}
    v.GatherKernel(K, n, [1, 2, 3], out=pipe.out)  # bins for the stages below
    out["scatter"] = timed(lambda: v.ScatterKernel(K, n, [0, 1, 2, 3], weight=1.0, attrs=pipe.attrs))
    out["apron"] = timed(lambda: v.UpdateApron(-1, 0.0))
    out["gather"] = timed(lambda: v.GatherKernel(K, n, [1, 2, 3], out=pipe.out))

    def rebin_gather():
        v.SetPoints(pipe.pos)  # drops the cached binning
        v.GatherKernel(K, n, [1, 2, 3], out=pipe.out)
    out["binning"] = max(timed(rebin_gather) - out["gather"], 0.0)
    return out


def count_launches(pipe):
    """Kernels of libgvdb2 in one step (names in the gvdb2 namespace)."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        pipe.step()
        torch.cuda.synchronize()
    ours = 0
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA and "gvdb2" in e.name:
            ours += 1
    return ours


def e2e_pipelined(pipe, pos, vel, steps, barrier):
    """Device time of `steps` end-to-end steps with double-buffered copies.

    Step k computes on buffer set k % 2 on the volume's own stream.  The
    inputs of step k+1 are copied into the other set on a copy stream, after
    step k-1 has finished with that set.  Step k's gathered velocities go
    back to pinned host memory on a third stream.  Returns the time from the
    first input copy to the last read-back.
    """
    import torch
    n = pipe.n
    hpos = torch.from_numpy(pos).pin_memory()
    hvel = torch.from_numpy(vel).pin_memory()
    hout = [torch.empty((n, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
    bufs = [(torch.empty_like(pipe.pos), torch.empty_like(pipe.vel), torch.empty_like(pipe.out)) for _ in range(2)]
    compute, h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    pipe.v.SetStream(compute)

    def run(k_steps, e0=None, e1=None):
        in_ready = [torch.cuda.Event() for _ in range(2)]
        done = [torch.cuda.Event() for _ in range(2)]
        read = [torch.cuda.Event() for _ in range(2)]
        with torch.cuda.stream(h2d):
            if e0 is not None:
                e0.record(h2d)
            bufs[0][0].copy_(hpos, non_blocking=True)
            bufs[0][1].copy_(hvel, non_blocking=True)
            in_ready[0].record(h2d)
        for k in range(k_steps):
            cur, nxt = k % 2, (k + 1) % 2
            if k + 1 < k_steps:  # next step's inputs, once step k-1 is done with that set
                with torch.cuda.stream(h2d):
                    if k >= 1:
                        h2d.wait_event(done[nxt])
                    bufs[nxt][0].copy_(hpos, non_blocking=True)
                    bufs[nxt][1].copy_(hvel, non_blocking=True)
                    in_ready[nxt].record(h2d)
            compute.wait_event(in_ready[cur])
            if k >= 2:
                compute.wait_event(read[cur])  # step k-2's result has left this buffer
            with torch.cuda.stream(compute):
                pipe.use_buffers(*bufs[cur])
                pipe.step()
                done[cur].record(compute)
            with torch.cuda.stream(d2h):
                d2h.wait_event(done[cur])
                hout[cur].copy_(bufs[cur][2], non_blocking=True)
                read[cur].record(d2h)
        if e1 is not None:
            e1.record(d2h)

    run(3)  # warm-up
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    run(steps, e0, e1)
    barrier()
    return e0.elapsed_time(e1)


def timed_steps(pipe, steps, warmup):
    """Device ms of `steps` pipeline steps after `warmup` untimed ones."""
    import torch
    for _ in range(warmup):
        pipe.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        pipe.step()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_ours(a):
    import torch
    import torch.distributed as dist
    from gvdb2 import metrics

    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    pos, vel, desc = workload_points(a)
    cpu = None
    if rank == 0 and ws == 1 and not (a.no_cpu_baseline or a.quick):
        cpu = cpu_baseline(pos, vel, 4_194_304)

    pipe = Pipeline(local, pos, vel, full_rebuild=not a.incremental)
    n = pipe.n

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        from gvdb2 import shard
        return shard.max_over_ranks(x, device=f"cuda:{local}")

    # the sampler starts before the warm-up (its start-up stays out of the
    # timed region) and keeps sampling until the timed steps are done
    clocks = Clocks(local)
    clocks.start()
    for _ in range(max(3, a.warmup)):
        pipe.step()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        pipe.step()
    e1.record()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = n * a.steps * ws / (ms / 1e3)

    if a.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": ws, "steps": a.steps,
                              "ms_per_step": ms / a.steps, "quick": True, "workload": desc,
                              "bricks": pipe.geometry()["B"]}), flush=True)
        return 0

    # per-stage device times: each stage repeated on the launching stream,
    # CUDA events around it, median of `reps`
    geo = pipe.geometry()
    stage_ms = stage_times(pipe)
    sb = metrics.stage_bytes(N=n, B=geo["B"], U=geo["U"], C=4, Cw=4, G=3, T=geo["T"], R3=geo["R3"], CL=geo["CL"])
    peak, peak_kind = peaks()
    stages = {}
    for k in ("topology", "binning", "scatter", "apron", "gather"):
        gbs = sb[k] / (stage_ms[k] / 1e3) / 1e9 if stage_ms.get(k) else None
        stages[k] = {"ms": round(stage_ms.get(k, 0.0), 4), "alg_bytes": sb[k], "GBps": gbs,
                     "frac_of_peak": gbs / peak if gbs else None}
    dom = max(("scatter", "gather", "apron"), key=lambda k: stage_ms.get(k, 0.0))
    achieved = sb[dom] / (stage_ms[dom] / 1e3) / 1e9
    step_alg = sum(sb.values())
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": TRAFFIC_PER_BRICK[dom] * geo["B"] if dom in TRAFFIC_PER_BRICK else None,
                "kernel": STAGE_KERNELS[dom], "stage": dom, "peak_source": f"{peak_kind} (MEASURED_PEAKS hbm_gbs)",
                "traffic_source": TRAFFIC_SOURCE,
                "step": {"alg_bytes": step_alg, "achieved": step_alg / (ms / a.steps / 1e3) / 1e9,
                         "frac": step_alg / (ms / a.steps / 1e3) / 1e9 / peak}}

    # end to end through the public API: every step copies its inputs from
    # pinned host memory and reads its gathered velocities back.  Two device
    # buffer sets alternate, so the copies of one step run on their own
    # streams while the neighbouring step computes.
    barrier()
    e2e_ms = e2e_pipelined(pipe, pos, vel, a.steps, barrier)
    ms_e2e = max_over_ranks(e2e_ms)
    e2e = {"value": n * a.steps * ws / (ms_e2e / 1e3), "unit": "points/s", "h2d_bytes_per_step": 24 * n,
           "d2h_bytes_per_step": 12 * n, "overlap": "double-buffered: H2D, compute and D2H on separate streams"}
    pipe.use_buffers(pipe.pos, pipe.vel, pipe.out)
    pipe.v.SetStream(0)
    barrier()
    launches = count_launches(pipe) * a.steps
    extras = {}
    if rank == 0 and ws == 1 and not a.no_extras and not a.sites:
        del pipe
        torch.cuda.empty_cache()
        extras = run_extras(a)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "points/s", "n_gpus": ws, "steps": a.steps,
                "warmup": max(3, a.warmup), "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": static_config(a, n, ws),
                "geometry": {"bricks": geo["B"], "nodes": geo["U"],
                             "atlas_mb_per_channel": round(4 * geo["B"] * geo["T"] / 1e6, 1)},
                "roofline": roofline, "stages": stages, "clocks": clk, "e2e": e2e, "gpu_launches": launches,
                "cpu_baseline": cpu}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


# DRAM bytes (read + write) per brick of each stage's kernels, from an ncu
# capture of one launch of each kernel on the 2,097,152-point block at the
# default workload's density (128 x 128 x 128 lattice sites at spacing
# (1, 0.5, 1): 1,024 points per 8^3 cell, 3,240 bricks), divided by its
# bricks.  Traffic grows with the brick count at a fixed density, so a
# launch moves about this many bytes x bricks.
TRAFFIC_PER_BRICK = {
    # k_pack_amounts, k_scatter_part, k_scatter_cells, k_scatter_merge
    "scatter": ((33.6 + 1.0) + (66.8 + 14.0) + (8.9 + 7.4) + (88.4 + 4.6)) * 1e6 / 3240,
    # k_gather_tile, k_gather_light
    "gather": ((70.6 + 2.7) + (12.4 + 0.0)) * 1e6 / 3240,
}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 2,097,152-point block at the "
                  "16,777,216-point step's density, scaled by bricks")
STAGE_KERNELS = {"scatter": "scatter stage: k_pack_amounts<4> + k_scatter_part<cubic,4> (dense cells' partials) + "
                            "k_scatter_cells<cubic,4> (owner-computes) + k_scatter_merge<cubic,4>",
                 "gather": "k_gather_tile<cubic,fwd,3> + k_gather_light<cubic,fwd,3>", "apron": "k_apron"}


# ----------------------------------------------------------------------------
# the rest of the metric, each measured in the same run (N = 1)
# ----------------------------------------------------------------------------
EXTRA_LEGS = ("incremental", "config1_4m", "adjoint", "batched", "vs_ref_kernels", "nanovdb_export", "autotune")
# legs left out of the main line, with the reason (none)
HELD_LEGS = {}


def run_leg(name, warmup, workload="dam16m"):
    """One extra leg in this process; returns its result dict (the export
    leg runs on `workload` when it is a dam block, else on dam16m)."""
    if name == "incremental":
        import gvdb2.workloads as wl
        w = WORKLOADS["dam16m"]
        pos, vel = wl.dam_block(sites=w["sites"], spacing=w["spacing"])
        return extra_incremental(pos, vel, warmup)
    if name == "config1_4m":
        return extra_config1()
    if name == "adjoint":
        return measure_adjoint(steps=20, warmup=3)
    if name == "batched":
        return measure_batched(steps=3, warmup=1)
    if name == "vs_ref_kernels":
        return extra_ref_kernels()
    if name == "nanovdb_export":
        return extra_nanovdb(warmup, workload if workload in ("dam16m", "dam") else "dam16m")
    if name == "autotune":
        return extra_autotune()
    raise ValueError(name)


def run_extras(a):
    """The rest of the metric, each leg in a child process of its own (a
    failing leg reports an error and never takes the main line down)."""
    out = {}
    for name in EXTRA_LEGS:
        if name in HELD_LEGS:
            out[name] = {"error": HELD_LEGS[name]}
            continue
        cmd = [sys.executable, os.path.abspath(__file__), "--leg", name, "--warmup", str(a.warmup)]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            if r.returncode == 0 and lines:
                out[name] = json.loads(lines[-1])
            else:
                tail = (r.stderr.strip().splitlines() or ["no output"])[-1]
                out[name] = {"error": f"exit {r.returncode}: {tail}"[:300]}
        except subprocess.TimeoutExpired:
            out[name] = {"error": "timed out after 900 s"}
    summary = {}
    if isinstance(out.get("adjoint"), dict) and "adjoint_over_forward" in out["adjoint"]:
        summary["adjoint_over_forward"] = out["adjoint"]["adjoint_over_forward"]
    if isinstance(out.get("batched"), dict) and "speedup_vs_loop" in out["batched"]:
        summary["batched_over_loop"] = out["batched"]["speedup_vs_loop"]
    if isinstance(out.get("vs_ref_kernels"), dict) and "speedup_device" in out["vs_ref_kernels"]:
        summary["vs_ref_kernels_speedup"] = out["vs_ref_kernels"]["speedup_device"]
    if isinstance(out.get("nanovdb_export"), dict) and "float" in out["nanovdb_export"]:
        summary["nanovdb_export_ms"] = out["nanovdb_export"]["float"]["ms"]
    out.update(summary)
    return out


def extra_incremental(pos, vel, warmup):
    """The reference's state machine on the 16M-point step (the first two
    RebuildTopology calls full, incremental from the third, V:1181-1218):
    10 steps of the advect, timed after `warmup` steps, against the same
    steps with a full rebuild every step."""
    res = {}
    for name, full in (("incremental", False), ("full", True)):
        pipe = Pipeline(0, pos, vel, full_rebuild=full)
        ms = timed_steps(pipe, 10, max(3, warmup))
        inf = pipe.v.info()
        res[name] = {"ms_per_step": ms / 10, "value": pipe.n * 10 / (ms / 1e3), "leaves": int(inf.pool_count[0]),
                     "bricks": int(inf.atlas_slots)}
        del pipe
    res["incremental_over_full_speedup"] = res["full"]["ms_per_step"] / res["incremental"]["ms_per_step"]
    res["workload"] = "16,777,216-pt dam block, 10 timed advect steps (dt 0.1), stale leaves kept by the state machine"
    return res


def extra_nanovdb(warmup, wname="dam16m"):
    """ExportToNanoVDB of the 16M-point step's volume (after one step): a
    float grid of channel 0 (mass) and a Vec3f grid of channels 1-3
    (momentum), each call timed end to end on the host (the call returns
    with the buffer complete: device passes, one read-back of the level-2
    headers, the root finished on the host and written back).  Algorithmic
    bytes: the live bricks' interiors read from the atlas plus the buffer
    written."""
    import ctypes
    import torch
    import gvdb2.workloads as wl
    w = WORKLOADS[wname]
    pos, vel = wl.dam_block(sites=w["sites"], spacing=w["spacing"])
    pipe = Pipeline(0, pos, vel, full_rebuild=True)
    timed_steps(pipe, 1, 1)
    v = pipe.v
    inf = v.info()
    peak, kind = peaks()
    res = {"workload": w["desc"] + ", the volume after one step", "leaves": int(inf.pool_count[0]),
           "level1": int(inf.pool_count[1]), "level2": int(inf.pool_count[2]), "timed_calls": 10}
    for name, chans in (("float", [0]), ("vec3f", [1, 2, 3])):
        nv = len(chans)
        size = ctypes.c_size_t()
        v._check(v._L.gvdb2_nanovdb_size(v._h, nv, ctypes.byref(size)), "nanovdb_size")
        buf = torch.empty(int(size.value), dtype=torch.uint8, device=pipe.dev)
        ch, bg = (ctypes.c_int * nv)(*chans), (ctypes.c_float * nv)(*([0.0] * nv))

        def call():
            v._check(v._L.gvdb2_export_nanovdb(v._h, nv, ch, bg, wname.encode(), 0, ctypes.c_void_p(buf.data_ptr()),
                                               int(size.value)), "export_nanovdb")
        for _ in range(max(3, warmup)):
            call()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            call()
        ms = (time.perf_counter() - t0) * 1e3 / 10
        alg = int(inf.atlas_slots) * int(inf.res[0]) ** 3 * 4 * nv + int(size.value)
        res[name] = {"ms": ms, "buffer_bytes": int(size.value), "algorithmic_bytes": alg,
                     "gbs": alg / ms / 1e6, "frac_of_hbm": alg / ms / 1e6 / peak, "peak": f"{peak:.1f} GB/s {kind}"}
    return res


def extra_autotune():
    """The autotuner on the step's scatter (4 channels) and gather (3
    channels), at 16,777,216 points (1,024 a cell) and 4,194,304 points (256
    a cell), after one step: each call timed (CUDA events, 10 calls after 2)
    with the default setting, then tuned (gvdb2_autotune_scatter / _gather on
    the same call, cache in a temporary file), then timed again."""
    import tempfile
    import torch
    import gvdb2
    import gvdb2.workloads as wl

    def per_call(fn):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 10

    res = {}
    with tempfile.TemporaryDirectory() as td:
        for wname in ("dam16m", "dam"):
            w = WORKLOADS[wname]
            pos, vel = wl.dam_block(sites=w["sites"], spacing=w["spacing"])
            pipe = Pipeline(0, pos, vel, full_rebuild=True)
            timed_steps(pipe, 1, 1)
            v, n, K = pipe.v, pipe.n, gvdb2.KERNEL_CUBIC2
            v.SetTuneCache(os.path.join(td, "tune.txt"))

            def scat():
                v.ScatterKernel(K, n, [0, 1, 2, 3], weight=1.0, attrs=pipe.attrs)

            def gath():
                v.GatherKernel(K, n, [1, 2, 3], out=pipe.out)
            r = {"default": list(v.GetTuning()), "scatter_ms_default": per_call(scat),
                 "gather_ms_default": per_call(gath)}
            t0 = time.perf_counter()
            v.AutotuneScatter(K, n, [0, 1, 2, 3], weight=1.0, attrs=pipe.attrs)
            v.AutotuneGather(K, n, [1, 2, 3], out=pipe.out)
            r["tuning_s"] = time.perf_counter() - t0
            r["tuned"] = list(v.GetTuning())
            r["scatter_ms_tuned"] = per_call(scat)
            r["gather_ms_tuned"] = per_call(gath)
            res[wname] = r
            del pipe
    return res


def extra_config1():
    """The 4,194,304-point dynamic step (the configuration's own size)."""
    import gvdb2.workloads as wl
    pos, vel = wl.dam_block(sites=WORKLOADS["dam"]["sites"], spacing=WORKLOADS["dam"]["spacing"])
    pipe = Pipeline(0, pos, vel, full_rebuild=True)
    ms = timed_steps(pipe, 20, 3)
    return {"workload": WORKLOADS["dam"]["desc"], "ms_per_step": ms / 20, "value": pipe.n * 20 / (ms / 1e3),
            "unit": "points/s"}


def extra_ref_kernels(steps=3, warmup=1):
    """The reference's own CUDA kernels (the gvdb-voxels kernel module
    compiled for sm_100a behind its host restatement, the prebuilt replay
    library that also generated the golden vectors) against libgvdb2, both
    on the reference's point path on the same advected 4,194,304 dam points:
    RebuildTopology -> UpdateAtlas -> InsertPoints -> ScatterDensity ->
    UpdateApron -> InsertPointsSubcell -> GatherDensity.  Per stage: device
    time of the kernels, copies and fills (CUPTI), and host wall time
    around the synchronised call (the reference's stages include host loops
    and blocking copies)."""
    import ctypes
    import numpy as np
    import torch
    from torch.profiler import ProfilerActivity, profile
    import gvdb2
    import gvdb2.workloads as wl
    lib = os.path.join(ROOT, "oracle", "_ref", "libgvdbref.so")
    if not os.path.exists(lib):
        return {"unavailable": "the replay library of the reference's kernels was not built"}
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as mg
    stages = ["rebuild", "atlas", "insert", "scatter", "apron", "subcell", "gather"]
    pos, vel = wl.dam_block(sites=WORKLOADS["dam"]["sites"], spacing=WORKLOADS["dam"]["spacing"])
    pts = []
    p = pos
    for _ in range(warmup + steps):
        p = (p + np.float32(DT) * vel).astype(np.float32)
        pts.append(np.ascontiguousarray(p))
    mg.check_inputs(dict(cfg=(3, 3, 3, 3, 3), radius=RADIUS, pts=pts, ops=[]))  # every kernel box inside the root

    def timed_stage(f):
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            t0 = time.perf_counter()
            f()
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        dev = sum(e.device_time for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA) / 1e3
        return dev, wall * 1e3

    def ref_side():
        R = mg.Ref(0)
        R("rd_configure", 3, 3, 3, 3, 3)
        R("rd_add_channel", 0, 1)
        zero = (ctypes.c_float * 3)(0, 0, 0)
        ln = ctypes.c_int(0)
        calls = {
            "rebuild": lambda n: (R("rd_request_full_rebuild"), R("rd_rebuild_topology", n, RADIUS, zero)),
            "atlas": lambda n: (R("rd_update_atlas"), R("rd_clear_channel", 0)),
            "insert": lambda n: R("rd_insert_points", n, zero),
            "scatter": lambda n: R("rd_scatter_density", n, 1.0, 1.0, zero, 0),
            "apron": lambda n: R("rd_update_apron", 0, 0.0),
            "subcell": lambda n: R("rd_insert_points_subcell", 4, n, RADIUS, zero, ctypes.byref(ln)),
            "gather": lambda n: R("rd_gather_density", n, 1.0, 0, 0),
        }
        t = {k: [] for k in stages}
        for q in pts:
            R("rd_set_points", q.ctypes.data, len(q))
            for k in stages:
                t[k].append(timed_stage(lambda: calls[k](len(q))))
        leaves = int(R.counts()[0])
        R.close()
        return t, leaves, ln.value

    def our_side():
        v = gvdb2.VolumeGVDB(0)
        v.Configure(3, 3, 3, 3, 3)
        v.AddChannel(0, gvdb2.T_FLOAT, 1)
        box = {}
        calls = {
            "rebuild": lambda n: (v.RequestFullRebuild(True), v.RebuildTopology(n, RADIUS)),
            "atlas": lambda n: (v.UpdateAtlas(), v.ClearChannel(0)),
            "insert": lambda n: v.InsertPoints(n),
            "scatter": lambda n: v.ScatterDensity(n, 1.0, 1.0, (0, 0, 0), False),
            "apron": lambda n: v.UpdateApron(0, 0.0),
            "subcell": lambda n: box.__setitem__("len", v.InsertPointsSubcell(4, n, RADIUS)),
            "gather": lambda n: v.GatherDensity(4, n, 1.0, (0, 0, 0), box["len"], 0),
        }
        t = {k: [] for k in stages}
        for q in pts:
            tq = torch.from_numpy(q).cuda()
            v.SetPoints(tq)
            for k in stages:
                t[k].append(timed_stage(lambda: calls[k](len(q))))
        leaves = int(v.info().pool_count[0])
        v.close()
        return t, leaves, box["len"]

    rt, rleaves, rlen = ref_side()
    ot, oleaves, olen = our_side()
    res = {"workload": "reference point path on the 4,194,304-pt dam block, advected 0.1 v per step; "
                       f"{steps} timed steps after {warmup}",
           "timing": "device: CUPTI kernel+copy+fill time per stage; host: wall time around the synchronised call",
           "reference_ms": {}, "ours_ms": {}, "check": {"leaves": [rleaves, oleaves], "subcell_len": [rlen, olen]}}
    dev_r = dev_o = wall_r = wall_o = 0.0
    for k in stages:
        dr = statistics.median(x[0] for x in rt[k][warmup:])
        do = statistics.median(x[0] for x in ot[k][warmup:])
        hr = statistics.median(x[1] for x in rt[k][warmup:])
        ho = statistics.median(x[1] for x in ot[k][warmup:])
        res["reference_ms"][k] = {"device": round(dr, 4), "host_wall": round(hr, 4)}
        res["ours_ms"][k] = {"device": round(do, 4), "host_wall": round(ho, 4)}
        dev_r, dev_o, wall_r, wall_o = dev_r + dr, dev_o + do, wall_r + hr, wall_o + ho
    res["reference_ms"]["total"] = {"device": round(dev_r, 4), "host_wall": round(wall_r, 4)}
    res["ours_ms"]["total"] = {"device": round(dev_o, 4), "host_wall": round(wall_o, 4)}
    res["speedup_device"] = dev_r / dev_o if dev_o > 0 else None
    res["speedup_host_wall"] = wall_r / wall_o if wall_o > 0 else None
    return res


# ----------------------------------------------------------------------------
# batched clouds: one batched pass vs a per-cloud loop of the plain path
# ----------------------------------------------------------------------------
BATCH_SPACE_LOG2 = 10


BATCH_STAGES = ("rebuild", "atlas", "scatter", "apron", "gather", "gather_adjoint", "scatter_adjoint")


def batched_step(v, K, n, chans_fwd, grad_chan, go, mark=None):
    """Forward (rebuild, splat, apron, gather) and adjoint (gather adjoint into
    the gradient channel, then the splat adjoint) over the volume's points.
    `mark`, if given, is called after each of BATCH_STAGES (event records)."""
    mark = mark or (lambda: None)
    v.RequestFullRebuild(True)
    v.RebuildTopology(n, RADIUS)
    mark()
    v.UpdateAtlas()
    mark()
    v.ScatterKernel(K, n, chans_fwd, weight=1.0)
    mark()
    for c in chans_fwd:  # the aprons of the scattered channels
        v.UpdateApron(c, 0.0)
    mark()
    out = v.GatherKernel(K, n, chans_fwd, out=go[0])
    mark()
    v.GatherDensityBackward(K, n, chans_fwd, out, grad_chans=[grad_chan], grad_pos=go[1])
    mark()
    v.ScatterDensityBackward(K, n, [grad_chan], weight=1.0, grad_pos=go[2], grad_weight=go[3], grad_attr=go[4])
    mark()


def measure_batched(steps, warmup, env=None, nclouds=0):
    """The 64 clouds in one batched pass against a per-cloud loop.  Under
    torchrun the clouds are spread over the ranks (LPT by size, no data-path
    collective); each rank batches its own share and the time is the max
    over the ranks.  nclouds > 0 keeps the first nclouds clouds only."""
    import torch
    import gvdb2
    import gvdb2.workloads as wl
    from gvdb2 import shard
    env = env or shard.RankEnv()
    all_clouds, _ = wl.batched_clouds()
    if nclouds > 0:
        all_clouds = all_clouds[:nclouds]
    mine = shard.lpt_partition([len(c) for c in all_clouds], env.world)[env.rank]
    clouds = [all_clouds[i] for i in mine]
    dev = [torch.from_numpy(c).cuda() for c in clouds]
    total = sum(len(c) for c in clouds)
    job_total = sum(len(c) for c in all_clouds)
    K = gvdb2.KERNEL_CUBIC2

    def volume():
        v = gvdb2.VolumeGVDB(env.local)
        v.Configure(3, 3, 3, 3, 3)
        for c in range(2):
            v.AddChannel(c, gvdb2.T_FLOAT, 1)
        return v

    def outs(n):
        return [torch.empty((n, 1), device="cuda"), torch.empty((n, 3), device="cuda"),
                torch.empty((n, 3), device="cuda"), torch.empty((n,), device="cuda"),
                torch.empty((n, 1), device="cuda")]

    vb = volume()
    gob = outs(total)

    def step_batched():
        vb.BatchPoints(dev, BATCH_SPACE_LOG2)
        batched_step(vb, K, total, [0], 1, gob)

    vl = volume()
    gol = [outs(len(c)) for c in clouds]

    def step_loop():
        for c, t in enumerate(dev):
            vl.SetPoints(t)
            batched_step(vl, K, len(t), [0], 1, gol[c])

    def timed(f, k):
        import torch.distributed as dist
        for _ in range(max(1, warmup)):
            f()
        torch.cuda.synchronize()
        if env.world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            f()
        e1.record()
        torch.cuda.synchronize()
        if env.world > 1:
            dist.barrier()
        return shard.max_over_ranks(e0.elapsed_time(e1) / k, device=f"cuda:{env.local}")

    clocks = Clocks(env.local)
    clocks.start()
    ms_b = timed(step_batched, steps)
    ms_l = timed(step_loop, max(1, steps))
    clk = clocks.stop()
    # one more batched pass with an event after each stage (on the volume's
    # stream, which is torch's current one here)
    ev = [torch.cuda.Event(enable_timing=True)]
    ev[0].record()

    def mark():
        ev.append(torch.cuda.Event(enable_timing=True))
        ev[-1].record()
    vb.BatchPoints(dev, BATCH_SPACE_LOG2)
    mark()
    batched_step(vb, K, total, [0], 1, gob, mark)
    torch.cuda.synchronize()
    stages = {"pack": ev[0].elapsed_time(ev[1])}
    stages.update({name: ev[i + 1].elapsed_time(ev[i + 2]) for i, name in enumerate(BATCH_STAGES)})
    # identical results, cloud by cloud, with stable binning on both sides
    # (each cell then adds its points in the same order)
    vb.SetDeterministic(True)
    vl.SetDeterministic(True)
    first = vb.BatchPoints(dev, BATCH_SPACE_LOG2)
    batched_step(vb, K, total, [0], 1, gob)
    step_loop()
    same = all(bool(torch.equal(gob[0][first[c]:first[c + 1]], gol[c][0])) and
               bool(torch.equal(gob[2][first[c]:first[c + 1]], gol[c][2])) for c in range(len(clouds)))
    same = shard.max_over_ranks(0.0 if same else 1.0, device=f"cuda:{env.local}") == 0.0
    bricks = int(vb.info().used_leaves)
    del vb, vl
    return {"workload": f"batched: {len(all_clouds)} Gaussian clouds, {job_total} points, sizes log-uniform in "
                        "[1e4, 2e6], each in its own 1024^3 space; cubic B-spline r=2, density; forward + adjoint",
            "value": job_total / (ms_b / 1e3), "unit": "points/s", "ms_per_step": ms_b,
            "per_cloud_loop": {"value": job_total / (ms_l / 1e3), "ms_per_step": ms_l},
            "batched_stage_ms": stages, "bricks": bricks,
            "speedup_vs_loop": ms_l / ms_b, "identical_to_loop": same, "n_gpus": env.world,
            "scaling": "strong", "parallelism": f"clouds over {env.world} ranks (LPT by size)", "steps": steps,
            "clocks": clk}


def run_batched(a):
    import torch
    from gvdb2 import shard
    env = shard.RankEnv.from_env()
    torch.cuda.set_device(env.local)
    if env.world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = measure_batched(a.steps, a.warmup, env, a.clouds)
    if env.rank == 0:
        line = {"metric": METRIC}
        line.update(res)
        line.update({"data": "synthetic", "dtype": "f32"})
        print(json.dumps(line), flush=True)
    if env.world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------
# differentiable splat: adjoint step vs forward step
# ----------------------------------------------------------------------------
def measure_adjoint(steps, warmup):
    """1,000,000 shell points splatted with the tent kernel into their own
    topology; loss = sum over voxels of (rho - rho_target)^2 plus the sum of
    the density gathered back at the points.  Forward = splat + loss +
    gather; adjoint = gather adjoint + loss gradient + splat adjoint (grads
    to positions and weights)."""
    import torch
    import gvdb2
    import gvdb2.workloads as wl
    K = gvdb2.KERNEL_TENT1
    src = torch.from_numpy(wl.plain_small()).cuda()
    tgt = torch.from_numpy(wl.diff_target()).cuda()
    n, nt = len(src), len(tgt)
    v = gvdb2.VolumeGVDB(0)
    v.Configure(3, 3, 3, 3, 3)
    for c in range(3):
        v.AddChannel(c, gvdb2.T_FLOAT, 1)
    v.SetPoints(src)
    v.RebuildTopology(n, RADIUS)
    v.UpdateAtlas()
    for c in range(3):
        v.ClearChannel(c)
    v.SetPoints(tgt)
    v.ScatterKernel(K, nt, [1])  # target density in the source topology (points outside it drop out)
    v.SetPoints(src)
    rho, rho_t, grad = v.atlas_tensor(0), v.atlas_tensor(1), v.atlas_tensor(2)
    out = torch.empty((n, 1), device="cuda")
    ones = torch.ones((n, 1), device="cuda")
    gp_g = torch.empty((n, 3), device="cuda")
    gp_s = torch.empty((n, 3), device="cuda")
    gw = torch.empty((n,), device="cuda")
    ga = torch.empty((n, 1), device="cuda")
    loss = [None]

    def forward():
        v.ScatterKernel(K, n, [0])
        loss[0] = torch.sum((rho - rho_t) ** 2)
        v.GatherKernel(K, n, [0], out=out)

    def adjoint():
        v.GatherDensityBackward(K, n, [0], ones, grad_chans=[2], grad_pos=gp_g)  # d(sum gathered)/d rho
        grad.add_(2.0 * (rho - rho_t))
        v.ScatterDensityBackward(K, n, [2], weight=1.0, grad_pos=gp_s, grad_weight=gw, grad_attr=ga)

    def timed(f):
        for _ in range(max(3, warmup)):
            f()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            f()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    clocks = Clocks(0)
    clocks.start()
    ms_f = timed(forward)
    ms_b = timed(adjoint)
    clk = clocks.stop()
    res = {"workload": "differentiable splat: 1,000,000 shell points (r 96-100) and a 1,000,000-point target "
                       "(r 90-104), tent r=1, loss = sum (rho - rho_t)^2 + sum gathered",
           "value": n / ((ms_f + ms_b) / 1e3), "unit": "points/s", "forward_ms": ms_f, "adjoint_ms": ms_b,
           "adjoint_over_forward": ms_b / ms_f, "bricks": int(v.info().atlas_slots), "steps": steps,
           "clocks": clk, "loss": float(loss[0].item())}
    v.close()
    return res


def run_adjoint(a):
    line = {"metric": METRIC}
    line.update(measure_adjoint(a.steps, a.warmup))
    line.update({"n_gpus": 1, "data": "synthetic", "dtype": "f32"})
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# large sparse scene: 67M-point Gaussian mixture on 32^3 bricks
# ----------------------------------------------------------------------------
SPARSE_WORKLOAD = ("large sparse scene: 67,108,864-pt 32-component Gaussian mixture (sigma 8-64, means in 4096^3), "
                   "Configure(3,3,3,4,5), cubic B-spline r=2, density+3 vel channels, full rebuild every step, "
                   "forward + adjoint")


def run_sparse(a):
    """Each step: advect p += 0.1 v -> full RebuildTopology(N, 2) ->
    UpdateAtlas -> scatter of mass and momentum (4 channels) -> UpdateApron
    -> gather of the 3 velocity channels; then the adjoint of
    L = sum(out * g) + sum over voxels of rho^2 for a fixed random g: the
    gather adjoint (dL/dG into 3 channels, dL/dpos) and the scatter adjoint
    (dL/dpos, dL/dweight, dL/dattr).  Per-kernel device times come from one
    profiled step after the timed region; GB/s per kernel is algorithmic
    bytes over that time."""
    import torch
    import gvdb2
    import gvdb2.workloads as wl
    from torch.profiler import ProfilerActivity, profile
    K = gvdb2.KERNEL_CUBIC2
    n = a.points if a.points else 67_108_864
    pos_h, vel_h = wl.gaussian_mixture(n=n)
    pos = torch.from_numpy(pos_h).cuda()
    vel = torch.from_numpy(vel_h).cuda()
    del pos_h, vel_h
    g_out = torch.randn((n, 3), device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    out = torch.empty((n, 3), device="cuda")
    gp_g = torch.empty((n, 3), device="cuda")
    gp_s = torch.empty((n, 3), device="cuda")
    gw = torch.empty((n,), device="cuda")
    ga = torch.empty((n, 4), device="cuda")
    v = gvdb2.VolumeGVDB(0)
    v.Configure(3, 3, 3, 4, 5)
    for c in range(8):
        v.AddChannel(c, gvdb2.T_FLOAT, 1)
    v.SetPoints(pos)
    attrs = [None, (vel, 0), (vel, 1), (vel, 2)]

    def rec(events, name):
        if events is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            events.append((name, e))

    def step(events=None):
        rec(events, "start")
        pos.add_(vel, alpha=DT)
        v.SetPoints(pos)
        v.RequestFullRebuild(True)
        v.RebuildTopology(n, RADIUS)
        v.UpdateAtlas()
        rec(events, "topology")
        v.ScatterKernel(K, n, [0, 1, 2, 3], weight=1.0, attrs=attrs)
        rec(events, "scatter")
        for c in range(4):
            v.UpdateApron(c, 0.0)
        rec(events, "apron")
        v.GatherKernel(K, n, [1, 2, 3], out=out)
        rec(events, "gather")
        v.GatherDensityBackward(K, n, [1, 2, 3], g_out, grad_chans=[5, 6, 7], grad_pos=gp_g)
        rec(events, "gather_adjoint")
        rho, g_rho = v.atlas_tensor(0), v.atlas_tensor(4)
        torch.mul(rho, 2.0, out=g_rho)
        v.ScatterDensityBackward(K, n, [4, 5, 6, 7], weight=1.0, attrs=attrs, grad_pos=gp_s, grad_weight=gw,
                                 grad_attr=ga)
        rec(events, "scatter_adjoint")

    for _ in range(max(3, a.warmup)):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / a.steps
    if a.quick:  # timed steps only
        print(json.dumps({"metric": METRIC, "workload": SPARSE_WORKLOAD, "value": n / (ms / 1e3),
                          "unit": "points/s", "ms_per_step": ms, "n_points": n, "clocks": clk}), flush=True)
        return 0
    # per-stage device time (event pairs), median over 3 steps
    per = {}
    for _ in range(3):
        ev = []
        step(ev)
        torch.cuda.synchronize()
        for (_, x), (nm, y) in zip(ev, ev[1:]):
            per.setdefault(nm, []).append(x.elapsed_time(y))
    stage = {k: statistics.median(t) for k, t in per.items()}
    # per-kernel device time from one profiled step
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step()
        torch.cuda.synchronize()
    kt = {}
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA:
            nm = e.name.replace("(anonymous namespace)::", "").replace("gvdb2::", "").replace("void ", "")
            nm = nm.split("(")[0]
            d = kt.setdefault(nm, [0, 0.0])
            d[0] += 1
            d[1] += e.device_time / 1e3
    inf = v.info()
    slots = int(inf.atlas_slots)
    ncell = slots * 64
    T3, R3 = int(inf.tile_res) ** 3, 32 ** 3
    alg = {"k_apron": slots * (T3 - R3) * 4 * 2}
    total_ms = sum(d[1] for d in kt.values())
    kernels = []
    for nm, (cnt, t) in sorted(kt.items(), key=lambda x: -x[1][1]):
        row = {"kernel": nm, "launches": cnt, "ms": round(t, 3), "share": round(t / total_ms, 4)}
        b = alg.get(nm)
        if b is not None:
            one = t / cnt  # ms per launch
            row["alg_gb_per_launch"] = round(b / 1e9, 3)
            row["gbs"] = round(b / (one / 1e3) / 1e9, 1)
        kernels.append(row)
    peak, src = peaks()
    line = {"metric": METRIC, "workload": SPARSE_WORKLOAD, "value": n / (ms / 1e3), "unit": "points/s",
            "ms_per_step": ms, "stage_ms": stage, "bricks": slots, "cells": ncell, "n_points": n, "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "data": "synthetic", "dtype": "f32",
            "hbm_peak_gbs": peak, "peak_source": src, "kernels": kernels[:16], "clocks": clk,
            "device_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 2)}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.leg:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_leg(a.leg, a.warmup, a.workload)), flush=True)
        return 0
    if a.impl == "reference":
        if a.workload not in WORKLOADS:
            print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the dam-block step"}))
            return 0
        return run_reference(a)
    if a.workload == "batched":
        return run_batched(a)
    if a.workload == "adjoint":
        return run_adjoint(a)
    if a.workload == "sparse67m":
        return run_sparse(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
