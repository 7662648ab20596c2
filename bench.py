#!/usr/bin/env python
"""bench.py — SAH BVH build throughput (Mtri/s) on B200.

Workload: the noisy level-8 icosphere (1,310,720 f32 triangles, 655,362
shared vertices, 3-octave value noise of amplitude 0.05, seeded), leaf size
MIN = MAX = 1, max_depth 32, the reference's split profile (32 bins above
32 objects, adaptive sweep at or below). One step = one full BVH build.

  value  builds timed with CUDA events on the build stream, inputs already
         in HBM; L2 flushed (256 MiB write) before every step, outside the
         timed interval; max over ranks; Mtri/s = triangles / time.
  e2e    the same build through the C ABI's host-pointer entry point
         (mgbvh_build_indexed): pinned host inputs copied in, nodes, lens and
         permutation copied out, every step.
  cpu_baseline / --impl reference: the oracle port (faithful mode: the
         reference's algorithmic form, bvh/src/lib.rs) on host cores, one
         single-threaded build per process like the reference's sample
         collector (bvh_sample_collector/src/main.rs:41-44), on the same
         1,310,720-triangle mesh (a step: one build per core, concurrently).

With torchrun (N > 1) every rank builds its own replica (the path does not
shard within a mesh); value = all ranks' triangles / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BVH build Mtri/s"
UNIT = "Mtri/s"
SAMPLE_TRIS = 131072
# dram__bytes_read.sum + dram__bytes_write.sum of one small_kernel launch on
# this workload (24 warps per SM), from an ncu capture (cold cache):
# 52.85 MB + 58.80 MB
SMALL_KERNEL_TRAFFIC = 111650048
# smsp__inst_executed.sum of the same launch (warp instructions, spill loads
# and stores included); the issue ceiling is one warp instruction per SM
# sub-partition per cycle
SMALL_KERNEL_INST = 464942099
SM_SUBPARTITIONS = 4
WORKLOAD = ("noisy icosphere L8 (1,310,720 tris, 655,362 verts), leaf 1, max_depth 32, "
            "reference split profile")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="icosphere",
                   choices=["icosphere", "mixed", "batched", "learned"],
                   help="icosphere: the headline build; mixed: 16.8M-triangle scene + 8M rays")
    p.add_argument("--mixed-scale", type=int, default=1,
                   help="divide the mixed scene and its ray count by this factor")
    p.add_argument("--batch-mode", default="both", choices=["levels", "queue", "both"],
                   help="batched workload: level passes, the persistent queue launch, or both (the faster leads)")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-pointer (e2e) leg")
    p.add_argument("--profile-steps", type=int, default=None, help=argparse.SUPPRESS)
    return p.parse_args()


def max_over_ranks(x: float, device="cuda") -> float:
    """The largest of every rank's x (the slowest rank's time); x itself when
    no process group is running."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(per_rank_units: int, world: int, ms_per_step: float) -> float:
    """Millions of units per second over all ranks: every rank's units of one
    step / the slowest rank's step time."""
    return world * per_rank_units / (ms_per_step * 1e-3) / 1e6


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def workload():
    from marigold_b200 import synth
    v, t = synth.config2_mesh()
    return v, t, synth.mesh_bounds(v)


def workload_triangles() -> int:
    return 20 * 4 ** 8  # icosphere level 8


# ---------------------------------------------------------------- CPU leg

_cpu_mesh = None


def _cpu_init():
    global _cpu_mesh
    v, t, b = workload()
    _cpu_mesh = {"full": (v, t, b), "warm": (v, np.ascontiguousarray(t[:SAMPLE_TRIS]), None)}


def _cpu_build(which):
    from oracle import oracle
    v, t, b = _cpu_mesh[which]
    t0 = time.perf_counter()
    r = oracle.build(v, t, root_bounds=b, faithful=True)
    dt = time.perf_counter() - t0
    assert r["status"] == 0
    return dt


def cpu_measure(steps: int, warmup: int):
    """Faithful oracle builds of the whole workload mesh (1,310,720 triangles,
    the same build the GPU times), one single-threaded build per process on
    every host core, as the reference's sample collector runs its builds.
    A step ends when the last core's build ends: Mtri/s = cores * triangles /
    step time. Warm-up steps build the first SAMPLE_TRIS triangles only (they
    are untimed and need not be long)."""
    cores = max(1, min(os.cpu_count() or 1, 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_cpu_init) as pool:
        for _ in range(warmup):
            pool.map(_cpu_build, ["warm"] * cores)
        walls = []
        for _ in range(steps):
            t0 = time.perf_counter()
            pool.map(_cpu_build, ["full"] * cores)
            walls.append(time.perf_counter() - t0)
    wall = sum(walls) / len(walls)
    n = workload_triangles()
    value = cores * n / wall / 1e6
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"the whole workload mesh ({n} triangles), one single-threaded faithful-oracle "
                      f"build per core, {cores} concurrent, mean of {steps} steps",
            "same_config": True, "ms_per_step": wall * 1e3}


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit and bit != 0x1:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.nv:
            self.t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


# ---------------------------------------------------------------- GPU leg

def algorithmic_bytes(n, n_verts, internal_len_sum, node_count):
    """Bytes a build must move at minimum (per object per level of the
    partition: read + write of a 24-byte AABB and a 4-byte index)."""
    return (n * (12 + 3 * 32) + n * 24 + internal_len_sum * 56 + node_count * 32)


def issue_roofline(inst, launch_ms, clk, sms=None):
    """The instruction-issue ceiling of a kernel: `inst` warp instructions
    (smsp__inst_executed.sum from an ncu capture of the launch) at one per
    sub-partition per cycle on every SM (`sms`, else the current device's
    count), at the median SM clock sampled during the timed steps. frac is
    the ceiling's time over the measured one, i.e. the fraction of issue
    slots the launch used."""
    if sms is None:
        import torch
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz")
    if not mhz or launch_ms <= 0:
        return None
    peak = sms * SM_SUBPARTITIONS * mhz * 1e6  # warp instructions per second
    achieved = inst / (launch_ms * 1e-3)
    return {"bound": "issue", "inst_per_launch": int(inst), "achieved": round(achieved / 1e9, 1),
            "peak": round(peak / 1e9, 1), "unit": "Ginst/s", "frac": round(achieved / peak, 4),
            "sm_mhz": mhz, "sms": sms,
            "inst_source": "smsp__inst_executed.sum, one ncu capture of the launch"}


def learned_leg(ctx, build_dev, c_args, c_count, d_nodes, d_lens, n, plain_sah, flush, stream, steps):
    """The learned form on the headline mesh (committed proposer, refine gate
    on): device-timed build Mtri/s as the plain build is timed, and its tree's
    total SAH against the plain tree's."""
    import torch
    from marigold_b200 import learned
    from marigold_b200.bvh import NODE_DTYPE, sah_cost
    weights = torch.from_numpy(learned.load_weights().view(np.int16)).cuda()
    ctx.set_split_proposer(weights, True)
    ctx.set_proposer_gate(*learned.RECOMMENDED_GATE)
    try:
        for _ in range(3):
            flush.fill_(1)
            ctx.check(build_dev(*c_args))
        torch.cuda.synchronize()
        ms = []
        for k in range(steps):
            flush.fill_(k & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(build_dev(*c_args))
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        count = c_count.value
        sah = sah_cost(d_nodes[: count * 8].cpu().numpy().view(NODE_DTYPE),
                       d_lens[:count].cpu().numpy().view(np.uint32))
    finally:
        ctx.set_split_proposer(None)
        ctx.set_proposer_gate(0.0, 0)
    bms = float(np.mean(ms))
    thr, min_n = learned.RECOMMENDED_GATE
    return {"value": round(n / (bms * 1e-3) / 1e6, 3), "unit": UNIT, "ms_per_step": round(bms, 4),
            "sah": round(sah, 4), "plain_sah": round(plain_sah, 4),
            "sah_delta_vs_plain_pct": round(100.0 * (sah / plain_sah - 1.0), 4),
            "proposer": f"marigold_b200/proposer_weights.bin, refine gate on (logit > {thr}), "
                        f"network on nodes of >= {min_n} objects"}


def trace_leg(steps, flush, scale=4):
    """Closest-hit Mrays/s on the mixed scene at 1/scale of its size (blobs,
    ground grid and thin triangles each divided by scale; rays likewise):
    plain build, then device-timed traces of every ray (L2 flushed before each);
    the first 4,096 rays' hits compared with GPU brute force."""
    import ctypes
    import torch
    from marigold_b200 import BvhSettings, _lib, build_device, synth
    v, t = synth.mixed_scene(n_blob=8388608 // scale, grid=(2048, 1024 // scale), n_thin=4194304 // scale)
    n = t.shape[0]
    rays = synth.rays_in_box(8388608 // scale, v[:, :3].min(0), v[:, :3].max(0))
    m = rays.shape[0]
    ctx = _lib.Context(0)
    ctx.set_tuning(1024)
    tr = _lib.Tracer(0)
    stream = torch.cuda.current_stream()
    try:
        dv = torch.from_numpy(v).cuda()
        dt = torch.from_numpy(t.view(np.int32)).cuda()
        dr = torch.from_numpy(rays).cuda()
        d_nodes = torch.empty((2 * n - 1) * 8, dtype=torch.int32, device="cuda")
        d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
        count, rc, _ = build_device(ctx, BvhSettings(max_depth=32), d_nodes, d_perm, vertices=dv,
                                    triangles=dt, stream=stream)
        torch.cuda.synchronize()
        mrays, hits, mism = _trace_rate(tr, d_nodes, count, dv, dt, d_perm, n, dr, m, stream, flush, steps)
    finally:
        tr.close()
        ctx.close()
    return {"value": round(mrays, 3), "unit": "Mrays/s", "rays": m, "triangles": n, "hit_rays": hits,
            "mismatches_vs_gpu_bruteforce_4096": mism,
            "scene": f"mixed scene at 1/{scale} size: 64 Gaussian blobs, 2048 x {1024 // scale}-quad ground grid, "
                     f"thin 1:200 triangles; rays uniform in the scene box grown by 10%, uniform directions"}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from marigold_b200 import BvhSettings, _lib
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    v, t, bounds = workload()
    n = t.shape[0]
    settings = BvhSettings(name="bench", bounds=bounds, max_depth=32)
    ctx = _lib.Context(local)
    from marigold_b200 import autotune
    tuned = autotune.apply(ctx, "icosphere_l8")  # switch-over and block size: speed only, same tree
    dv = torch.from_numpy(v).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    cap = 2 * n - 1
    d_nodes = torch.empty(cap * 8, dtype=torch.int32, device="cuda")
    d_lens = torch.empty(cap, dtype=torch.int32, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    # the C entry point with its arguments prepared once (the same call
    # build_device makes, without rebuilding them every step)
    import ctypes
    ctx.set_stream(stream.cuda_stream)
    c_settings = settings.to_c(1, 1)
    c_count = ctypes.c_uint32(0)
    c_stats = _lib.Stats()
    c_args = (ctx.ptr, ctypes.c_void_p(dv.data_ptr()), 4 * v.shape[1], v.shape[0],
              ctypes.c_void_p(dt.data_ptr()), n, ctypes.byref(c_settings),
              ctypes.c_void_p(d_nodes.data_ptr()), cap, ctypes.byref(c_count),
              ctypes.c_void_p(d_lens.data_ptr()), ctypes.c_void_p(d_perm.data_ptr()), ctypes.byref(c_stats))
    build_dev = ctx.L.mgbvh_build_indexed_dev

    def one():
        return ctx.check(build_dev(*c_args))

    for _ in range(max(args.warmup, 3)):
        flush.fill_(1)
        one()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = 0
    phase = np.zeros(4)
    with ClockSampler(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            ev[k][0].record(stream)
            one()
            ev[k][1].record(stream)
            st = c_stats.as_dict()
            count = c_count.value
            launches += st["kernel_launches"]
            phase += np.asarray(st["phase_seconds"])
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    ms_per_step = max_over_ranks(float(np.mean(ms)))
    value = whole_job_rate(n, world, ms_per_step)

    # tree statistics for the algorithmic byte counts (S = sum of inner lens)
    nodes_h = d_nodes.cpu().numpy().view(np.uint32).reshape(-1, 8)[:count]
    lens_h = d_lens.cpu().numpy().view(np.uint32)[:count].astype(np.int64)
    child = nodes_h[:, 7].astype(np.int64)
    inner = child != 0
    S = int(lens_h[inner].sum())
    alg = algorithmic_bytes(n, v.shape[0], S, count)
    # subtrees of <= 32 objects (the small kernel's units): nodes of len <= 32
    # whose parent holds more than 32 objects
    parent_len = np.zeros(count, dtype=np.int64)
    ci = child[inner]
    parent_len[ci] = lens_h[inner]
    parent_len[ci + 1] = lens_h[inner]
    small_root = (lens_h <= 32) & (lens_h >= 2) & (parent_len > 32)
    small_objs = int(lens_h[small_root].sum())
    small_tasks = int(small_root.sum())
    # per subtree: its 64-byte task and records read (32 B/object), nodes
    # written (32 B node + 4 B len + 1 B used each, 2*len - 1 of them) and the
    # permutation entries (4 B/object)
    small_alg = small_tasks * 64 + small_objs * (32 + 4) + (2 * small_objs - small_tasks) * 37
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = alg / (ms_per_step * 1e-3) / 1e9
    phase_ms = [x * 1e3 / args.steps for x in phase]
    small_ms = phase_ms[3]
    small_achieved = small_alg / (small_ms * 1e-3) / 1e9 if small_ms > 0 else 0.0

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(value, 3), "unit": UNIT,
                              "ms_per_step": round(ms_per_step, 4), "n_gpus": world,
                              "phase_ms": [round(x * 1e3 / args.steps, 4) for x in phase],
                              "gpu_launches": int(launches), "clocks": clocks.summary()}))
        if world > 1:
            dist.destroy_process_group()
        return

    # e2e through the host-pointer C ABI entry point, pinned host buffers
    L = ctx.L
    pin_v = torch.from_numpy(v).pin_memory()
    pin_t = torch.from_numpy(t.view(np.int32)).pin_memory()
    pin_nodes = torch.empty(cap * 8, dtype=torch.int32).pin_memory()
    pin_lens = torch.empty(cap, dtype=torch.int32).pin_memory()
    pin_perm = torch.empty(n, dtype=torch.int32).pin_memory()
    cs = settings.to_c(1, 1)
    cnt = ctypes.c_uint32(0)
    ctx.set_stream(None)

    def e2e_one():
        rc = L.mgbvh_build_indexed(ctx.ptr, ctypes.c_void_p(pin_v.data_ptr()), 32, v.shape[0],
                                   ctypes.c_void_p(pin_t.data_ptr()), n, ctypes.byref(cs),
                                   ctypes.c_void_p(pin_nodes.data_ptr()), cap, ctypes.byref(cnt),
                                   ctypes.c_void_p(pin_lens.data_ptr()),
                                   ctypes.c_void_p(pin_perm.data_ptr()), None)
        ctx.check(rc)

    for _ in range(3):
        e2e_one()
    e2e_ms = []
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_one()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = max_over_ranks(float(np.mean(e2e_ms)))
    h2d = v.nbytes + t.nbytes
    d2h = cnt.value * 32 + cnt.value * 4 + n * 4

    # the metric's other two figures, on one GPU: the learned form against the
    # plain build on this mesh, and closest-hit Mrays/s on a mixed scene
    extras = {}
    if world == 1:
        from marigold_b200.bvh import NODE_DTYPE, sah_cost
        ctx.set_stream(stream.cuda_stream)
        plain_sah = sah_cost(nodes_h.reshape(-1).view(NODE_DTYPE), lens_h.astype(np.uint32))
        with ClockSampler(local) as xclocks:
            extras["learned"] = learned_leg(ctx, build_dev, c_args, c_count, d_nodes, d_lens, n, plain_sah,
                                            flush, stream, args.steps)
            extras["trace"] = trace_leg(max(3, args.steps // 2), flush)
        extras["learned"]["clocks"] = extras["trace"]["clocks"] = xclocks.summary()

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded noisy icosphere; no public dataset is named)",
        "config": {"workload": WORKLOAD, "triangles": n, "vertices": int(v.shape[0]),
                   "min_leaf": 1, "max_leaf": 1, "max_depth": 32, "bins": 32,
                   "adaptive_max_n": 32, "parallelism": f"replicas x{world}",
                   "l2": "flushed before every step (256 MiB write, outside the timed interval)",
                   "tuning": tuned},
        "e2e": {"value": round(whole_job_rate(n, world, e2e_step), 3), "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": round(e2e_step, 4)},
        "roofline": {"bound": "hbm", "kernel": "small_kernel (subtrees of <= 32 objects)",
                     "achieved": round(small_achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(small_achieved / hbm, 4), "peak_source": peak_src,
                     "traffic": SMALL_KERNEL_TRAFFIC,
                     "algorithmic_bytes_per_launch": int(small_alg),
                     "launch_ms": round(small_ms, 4), "subtrees": small_tasks,
                     "issue": issue_roofline(SMALL_KERNEL_INST, small_ms, clocks.summary()),
                     "note": "issue-bound: the adaptive sweep's O(n^2) threshold evaluation"},
        "roofline_build": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                           "unit": "GB/s", "frac": round(achieved / hbm, 4),
                           "algorithmic_bytes_per_build": int(alg), "inner_len_sum": S},
        "phase_ms": [round(x, 4) for x in phase_ms],
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "nodes": int(count),
        **extras,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_measure(steps=1, warmup=0)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cb = cpu_measure(steps=args.steps, warmup=args.warmup)
    out = {
        "impl": "reference", "metric": METRIC, "value": round(cb["value"], 4), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(cb["ms_per_step"], 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded noisy icosphere)",
        "config": {"workload": WORKLOAD, "triangles": workload_triangles(), "same_config": True,
                   "min_leaf": 1, "max_leaf": 1, "max_depth": 32, "parallelism": "host cores"},
        "cpu_baseline": cb,
        "e2e": {"value": round(cb["value"], 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_mixed(args):
    """The large mixed scene: 16,777,216 triangles (8,388,608 in 64 Gaussian
    blobs, a 2048 x 1024-quad ground grid, 4,194,304 thin 1:200 triangles),
    built twice, plain (the reference profile) and learned (the committed
    split proposer with the recommended gate), then 8,388,608 closest-hit rays with
    origins uniform in the scene box grown by 10% and uniform directions on
    each tree. Each traversal is checked hit for hit against GPU brute force
    on a 65,536-ray subset (the brute-force kernel is itself checked against
    the CPU oracle by the test suite)."""
    import ctypes
    import torch
    from marigold_b200 import BvhSettings, _lib, build_device, learned, synth
    from marigold_b200.bvh import NODE_DTYPE, sah_cost
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    sc = max(1, args.mixed_scale)

    def log(msg):
        print(f"[mixed {time.perf_counter() - t0:8.1f}s] {msg}", file=sys.stderr, flush=True)

    v, t = synth.mixed_scene(n_blob=8388608 // sc, grid=(2048, 1024 // sc), n_thin=4194304 // sc)
    n = t.shape[0]
    rays = synth.rays_in_box(8388608 // sc, v[:, :3].min(0), v[:, :3].max(0))
    gen_s = time.perf_counter() - t0
    log(f"generated {n} triangles, {rays.shape[0]} rays")
    ctx = _lib.Context(0)
    ctx.set_tuning(1024)
    dv = torch.from_numpy(v).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    cap = 2 * n - 1
    d_nodes = torch.empty(cap * 8, dtype=torch.int32, device="cuda")
    d_lens = torch.empty(cap, dtype=torch.int32, device="cuda")
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    settings = BvhSettings(name="mixed", max_depth=32)
    weights = torch.from_numpy(learned.load_weights().view(np.int16)).cuda()
    dr = torch.from_numpy(rays).cuda()
    m = rays.shape[0]
    sub = min(65536, m)
    tr = _lib.Tracer(0)
    L = tr.L
    sp = ctypes.c_void_p(stream.cuda_stream)
    vp = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    ht = torch.empty(m, dtype=torch.float32, device="cuda")
    hp = torch.empty(m, dtype=torch.int32, device="cuda")
    bt = torch.empty(sub, dtype=torch.float32, device="cuda")
    bp = torch.empty(sub, dtype=torch.int32, device="cuda")
    forms = {}
    brute = None
    clocks = ClockSampler(0).__enter__()  # sampled through every timed build and trace below
    for form in ("plain", "learned"):
        ctx.set_split_proposer(weights if form == "learned" else None, True)
        ctx.set_proposer_gate(*(learned.RECOMMENDED_GATE if form == "learned" else (0.0, 0)))
        build_ms, count, st = [], 0, {}
        for k in range(max(args.warmup, 1) + args.steps):
            flush.fill_(k & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            count, rc, st = build_device(ctx, settings, d_nodes, d_perm, vertices=dv, triangles=dt,
                                         out_lens=d_lens, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ctx.check(rc)
            if k >= max(args.warmup, 1):
                build_ms.append(e0.elapsed_time(e1))
            log(f"{form} build {k}: {e0.elapsed_time(e1):.2f} ms, {count} nodes")
        sah = sah_cost(d_nodes[: count * 8].cpu().numpy().view(NODE_DTYPE),
                       d_lens[:count].cpu().numpy().view(np.uint32))
        tr.check(L.mgbvh_tracer_set_blas_dev(tr.ptr, vp(d_nodes), count, None, vp(dv), 4 * v.shape[1], v.shape[0],
                                             vp(dt), vp(d_perm), n, sp))
        counts = (ctypes.c_uint64 * 3)()
        secs = ctypes.c_double(0)
        trace_ms = []
        for k in range(max(args.warmup, 1) + args.steps):
            flush.fill_(k & 0xFF)
            tr.check(L.mgbvh_trace_closest_dev(tr.ptr, vp(dr), m, vp(ht), vp(hp), counts,
                                               ctypes.byref(secs), sp))
            if k >= max(args.warmup, 1):
                trace_ms.append(secs.value * 1e3)
            log(f"{form} trace {k}: {secs.value * 1e3:.2f} ms")
        if brute is None:  # the closest hit does not depend on the tree
            tb = time.perf_counter()
            tr.check(L.mgbvh_trace_bruteforce_dev(tr.ptr, vp(dr), sub, vp(bt), vp(bp), sp))
            torch.cuda.synchronize()
            brute = (bt.cpu().numpy(), bp.cpu().numpy().view(np.uint32), time.perf_counter() - tb)
            log(f"brute force {sub} rays: {brute[2]:.1f} s")
        gt, gp = ht[:sub].cpu().numpy(), hp[:sub].cpu().numpy().view(np.uint32)
        mism = int(((gp != brute[1]) | (gt.view(np.uint32) != brute[0].view(np.uint32))).sum())
        # the same tree collapsed to the 8-wide BVH with quantized boxes
        wcount = ctypes.c_uint32(0)
        tw = time.perf_counter()
        tr.check(L.mgbvh_tracer_build_wide(tr.ptr, sp, ctypes.byref(wcount)))
        wide_build_s = time.perf_counter() - tw
        wcounts = (ctypes.c_uint64 * 3)()
        wide_ms = []
        for k in range(max(args.warmup, 1) + args.steps):
            flush.fill_(k & 0xFF)
            tr.check(L.mgbvh_trace_closest_wide_dev(tr.ptr, vp(dr), m, vp(ht), vp(hp), wcounts,
                                                    ctypes.byref(secs), sp))
            if k >= max(args.warmup, 1):
                wide_ms.append(secs.value * 1e3)
            log(f"{form} wide trace {k}: {secs.value * 1e3:.2f} ms")
        wgt, wgp = ht[:sub].cpu().numpy(), hp[:sub].cpu().numpy().view(np.uint32)
        wmism = int(((wgp != brute[1]) | (wgt.view(np.uint32) != brute[0].view(np.uint32))).sum())
        wms = float(np.mean(wide_ms))
        bms, tms = float(np.mean(build_ms)), float(np.mean(trace_ms))
        forms[form] = {
            "build": {"value": round(n / (bms * 1e-3) / 1e6, 2), "unit": "Mtri/s", "ms": round(bms, 3),
                      "nodes": count, "height": st.get("height"), "sah": round(sah, 4),
                      "learned_splits": st.get("learned_splits"),
                      "phase_ms": [round(x * 1e3, 3) for x in st.get("phase_seconds", [])]},
            "trace": {"value": round(m / (tms * 1e-3) / 1e6, 2), "unit": "Mrays/s", "ms": round(tms, 3),
                      "hit_rays": int((hp != -1).sum().item()), "nodes_visited": counts[0],
                      "box_tests": counts[1], "triangle_tests": counts[2]},
            "check": {"subset_rays": sub, "mismatches_vs_gpu_bruteforce": mism},
            "wide_trace": {"value": round(m / (wms * 1e-3) / 1e6, 2), "unit": "Mrays/s", "ms": round(wms, 3),
                           "wide_nodes": wcount.value, "collapse_s": round(wide_build_s, 4),
                           "nodes_visited": wcounts[0], "box_tests": wcounts[1],
                           "triangle_tests": wcounts[2], "mismatches_vs_gpu_bruteforce": wmism},
        }
    clocks.__exit__()
    ctx.set_split_proposer(None)
    out = {
        "metric": "BVH build Mtri/s; closest-hit Mrays/s", "workload": "mixed scene",
        "clocks": clocks.summary(),
        "config": {"triangles": n, "rays": m, "blobs": 64, "grid_quads": [2048, 1024 // sc],
                   "thin": 4194304 // sc, "scale": sc, "max_depth": 32, "leaf": 1,
                   "profile": "reference", "learned": "committed proposer, gate on"},
        "build": forms["plain"]["build"], "trace": forms["plain"]["trace"],
        "wide_trace": forms["plain"]["wide_trace"],
        "check": dict(forms["plain"]["check"], bruteforce_s=round(brute[2], 2)),
        "learned": forms["learned"],
        "steps": args.steps, "warmup": args.warmup, "generation_s": round(gen_s, 1),
        "l2": "flushed before every build and trace",
    }
    tr.close()
    print(json.dumps(out), flush=True)


def run_batched(args):
    """The batched scene: 512 meshes with triangle counts log-uniform in
    [64, 262144] (random small triangles or a trimmed noisy icosphere, coin
    flip) plus the TLAS over 4,096 instances (random rotation, scale in
    [0.5, 2], translation in [-100, 100]^3; instance AABBs from the 8 corners
    of the mesh bounds), all 513 trees in one batched build. A step computes
    the instance boxes on the GPU from the meshes' bounds and the instances'
    f32 transforms, then builds all trees; the first build runs eagerly and
    captures a CUDA graph, timed builds replay the graph. Both batch modes are
    timed (level passes + subtree launches; one persistent launch over
    device-side task queues), their trees compared, and the faster one leads
    the line. Then closest-hit rays through the built two-level scene."""
    import torch
    from marigold_b200 import BvhSettings, _lib, autotune, build_batch_device, synth
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    meshes, bounds, inst = synth.batched_scene()
    ids, xf = synth.scene_instances(3, len(meshes), inst.shape[0])
    gen_s = time.perf_counter() - t0
    ctx = _lib.Context(0)
    tuned = autotune.apply(ctx, "batched_scene")
    medium_max, bins = tuned["medium_max"], tuned["bins"]
    ctx.check(ctx.L.mgbvh_set_graph_capture(ctx.ptr, 1))
    descs = [{"vertices": torch.from_numpy(v).cuda(), "triangles": torch.from_numpy(t.view(np.int32)).cuda(),
              "bounds": b} for (v, t), b in zip(meshes, bounds)]
    from marigold_b200.bvh import instance_aabbs_device
    d_bounds = torch.from_numpy(bounds).cuda()
    d_ids = torch.from_numpy(ids.view(np.int32)).cuda()
    d_xf = torch.from_numpy(xf).cuda()
    d_inst = torch.empty((inst.shape[0], 6), dtype=torch.float32, device="cuda")
    descs.append({"aabbs": d_inst})
    n_tris = sum(t.shape[0] for _, t in meshes)
    total = n_tris + inst.shape[0]
    slots = sum(2 * t.shape[0] - 1 for _, t in meshes) + 2 * inst.shape[0] - 1
    nodes = torch.empty(slots * 8, dtype=torch.int32, device="cuda")
    lens = torch.empty(slots, dtype=torch.int32, device="cuda")
    perm = torch.empty(total, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    settings = BvhSettings(bins=bins)
    modes = {}
    trees = {}
    for mode in (["levels", "queue"] if args.batch_mode == "both" else [args.batch_mode]):
        ctx.set_batch_mode(mode == "queue")
        times, replays, eager_ms = [], 0, None
        offs = None
        with ClockSampler(0) as clocks:
            for k in range(max(args.warmup, 2) + args.steps):
                flush.fill_(k & 0xFF)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.set_stream(stream.cuda_stream)
                instance_aabbs_device(ctx, d_bounds, d_ids, d_xf, d_inst)
                offs, rc, st = build_batch_device(ctx, settings, descs, nodes, perm, out_lens=lens,
                                                  stream=stream)
                e1.record(stream)
                stream.synchronize()
                if k == 0:
                    eager_ms = e0.elapsed_time(e1)
                if k >= max(args.warmup, 2):
                    times.append(e0.elapsed_time(e1))
                    replays += st["graph_replay"]
        mms = float(np.mean(times))
        modes[mode] = {"value": round(total / (mms * 1e-3) / 1e6, 2), "unit": "Mtri/s", "ms_per_step": round(mms, 3),
                       "eager_first_build_ms": round(eager_ms, 3), "graph_replays": replays,
                       "kernel_launches": st["kernel_launches"], "clocks": clocks.summary()}
        trees[mode] = (offs, nodes.cpu().numpy().copy(), lens.cpu().numpy().copy(), perm.cpu().numpy().copy())
    if len(trees) == 2:
        a, b = trees["levels"], trees["queue"]
        modes["same_trees"] = bool(a[0] == b[0] and all(np.array_equal(x, y) for x, y in zip(a[1:], b[1:])))
    best = min((m for m in modes if m in ("levels", "queue")), key=lambda m: modes[m]["ms_per_step"])
    times = [modes[best]["ms_per_step"]]
    replays, eager_ms = modes[best]["graph_replays"], modes[best]["eager_first_build_ms"]
    clocks_best = modes[best]["clocks"]
    from marigold_b200.bvh import NODE_DTYPE, sah_cost
    nh = nodes.cpu().numpy().view(NODE_DTYPE)
    lh = lens.cpu().numpy().view(np.uint32)
    sah_blas = sum(sah_cost(nh[offs[i]:offs[i + 1]], lh[offs[i]:offs[i + 1]]) for i in range(len(meshes)))
    sah_tlas = sah_cost(nh[offs[-2]:offs[-1]], lh[offs[-2]:offs[-1]])
    ms = float(np.mean(times))
    # closest hits through the built scene: TLAS -> instance -> BLAS
    from marigold_b200.bvh import Scene, trace_scene_device
    scene = Scene.from_batch([(d["vertices"], d["triangles"]) for d in descs[:-1]], offs, nodes, None, perm,
                             d_ids, d_xf)
    tr = _lib.Tracer(0)
    scene.bind(tr, stream)
    n_rays = 4194304
    rays = torch.from_numpy(synth.rays_in_box(n_rays, inst[:, :3].min(0), inst[:, 3:].max(0), seed=7)).cuda()
    trace_ms, counts = [], None
    with ClockSampler(0) as tclocks:
        for k in range(max(args.warmup, 1) + args.steps):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            _, _, hp, counts, secs = trace_scene_device(tr, rays, stream=stream)
            if k >= max(args.warmup, 1):
                trace_ms.append(secs * 1e3)
    hits = int((hp != -1).sum().item())
    sub = 1024
    got = trace_scene_device(tr, rays[:sub].contiguous(), stream=stream)
    want = trace_scene_device(tr, rays[:sub].contiguous(), stream=stream, bruteforce=True, cull=True)
    mism = int(((got[1] != want[1]) | (got[2] != want[2]) |
                (got[0].view(torch.int32) != want[0].view(torch.int32))).sum().item())
    tr.close()
    tms = float(np.mean(trace_ms))
    out = {
        "metric": "BVH build Mtri/s (batched: 512 BLAS + TLAS)", "workload": "batched scene",
        "trace": {"value": round(n_rays / (tms * 1e-3) / 1e6, 2), "unit": "Mrays/s", "ms": round(tms, 3),
                  "rays": n_rays, "hit_rays": hits, "nodes_visited": counts[0], "box_tests": counts[1],
                  "triangle_tests": counts[2], "clocks": tclocks.summary(),
                  "check": {"rays": sub, "mismatches_vs_gpu_bruteforce": mism,
                            "bruteforce": "every instance whose mesh box (grown by 1e-4) the mesh-space ray "
                                          "meets, every triangle of its mesh"},
                  "rays_from": "origins uniform in the instances' world box grown by 10%, uniform directions",
                  "traversal": "two-level: TLAS with the world ray, each instance's BLAS in mesh space "
                               "(scene.slang:91-220); one thread per ray, rays sorted"},
        "value": round(total / (ms * 1e-3) / 1e6, 2), "unit": "Mtri/s", "ms_per_step": round(ms, 3),
        "clocks": clocks_best, "batch_mode": best, "modes": modes,
        "eager_first_build_ms": round(eager_ms, 3), "graph_replays": replays, "steps": args.steps,
        "config": {"meshes": len(meshes), "triangles": n_tris, "instances": int(inst.shape[0]),
                   "trees": len(meshes) + 1, "nodes": int(offs[-1]), "medium_max": medium_max,
                   "bins": bins or "reference (32)", "tuning": dict(tuned, table="marigold_b200/tuning.json")},
        "sah": {"blas_sum": round(sah_blas, 3), "tlas": round(sah_tlas, 3)},
        "instance_boxes": "computed on the GPU in every step (mgbvh_instance_aabbs_dev); equal to the "
                          "host restatement: " + str(bool(np.array_equal(d_inst.cpu().numpy().view(np.uint32),
                                                                        inst.view(np.uint32)))),
        "generation_s": round(gen_s, 1), "l2": "flushed before every build",
    }
    print(json.dumps(out), flush=True)


def _trace_rate(tr, d_nodes, count, dv, dt, d_perm, n, dr, m, stream, flush, reps, check=4096):
    """Closest-hit Mrays/s of one built tree (median of reps traces, L2
    flushed before each), the number of rays that hit, and the number of the
    first `check` rays whose hit differs from GPU brute force."""
    import ctypes
    import torch
    L = tr.L
    sp = ctypes.c_void_p(stream.cuda_stream)
    vp = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    tr.check(L.mgbvh_tracer_set_blas_dev(tr.ptr, vp(d_nodes), count, None, vp(dv), 4 * dv.shape[1],
                                         dv.shape[0], vp(dt), vp(d_perm), n, sp))
    ht = torch.empty(m, dtype=torch.float32, device="cuda")
    hp = torch.empty(m, dtype=torch.int32, device="cuda")
    counts = (ctypes.c_uint64 * 3)()
    secs = ctypes.c_double(0)
    ms = []
    for k in range(reps + 1):
        flush.fill_(k & 0xFF)
        tr.check(L.mgbvh_trace_closest_dev(tr.ptr, vp(dr), m, vp(ht), vp(hp), counts,
                                           ctypes.byref(secs), sp))
        if k:
            ms.append(secs.value * 1e3)
    hits = int((hp != -1).sum().item())
    c = min(check, m)
    bt = torch.empty(c, dtype=torch.float32, device="cuda")
    bp = torch.empty(c, dtype=torch.int32, device="cuda")
    tr.check(L.mgbvh_trace_bruteforce_dev(tr.ptr, vp(dr), c, vp(bt), vp(bp), sp))
    torch.cuda.synchronize()
    mism = int(((hp[:c] != bp) | (ht[:c].view(torch.int32) != bt.view(torch.int32))).sum().item())
    return m / (statistics.median(ms) * 1e-3) / 1e6, hits, mism


def run_learned(args):
    """The learned split proposer against the plain builder on held-out seeds
    of its training generators (65,536 random small triangles; the level-8
    noisy icosphere) and on the large mixed scene at 1/4 and full size
    (16,777,216 triangles). Per mesh and build form: device-timed build
    Mtri/s (L2 flushed before every build), total SAH cost, and closest-hit
    Mrays/s of 1,048,576 rays (origins uniform in the mesh box grown by 10%,
    uniform directions) on the built tree. The full-sweep SAH of each mesh
    comes from tests/golden/full_sweep_sah.json (written by the script beside
    it). Forms: plain (the reference's tree), learned (trained network with
    the recommended gate: refine logit > 0, network on nodes of >= 2,048
    objects), learned-ungated (every binned node of 33 or more objects scores
    the network's proposals)."""
    import torch
    from marigold_b200 import BvhSettings, _lib, build_device, learned, synth
    from marigold_b200.bvh import NODE_DTYPE, sah_cost
    torch.cuda.set_device(0)
    with open(os.path.join(ROOT, "tests", "golden", "full_sweep_sah.json")) as f:
        golden = json.load(f)
    weights = torch.from_numpy(learned.load_weights().view(np.int16)).cuda()
    ctx = _lib.Context(0)
    ctx.set_tuning(1024)
    tr = _lib.Tracer(0)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    rows = []
    clocks = ClockSampler(0).__enter__()  # sampled through every timed build and trace below
    for name, kind, size, seed in learned.EVAL_MESHES + learned.EVAL_SCENES:
        v, t = learned.eval_mesh(kind, size, seed)
        n = t.shape[0]
        dv = torch.from_numpy(v).cuda()
        dt = torch.from_numpy(t.view(np.int32)).cuda()
        cap = 2 * n - 1
        d_nodes = torch.empty(cap * 8, dtype=torch.int32, device="cuda")
        d_lens = torch.empty(cap, dtype=torch.int32, device="cuda")
        d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
        rays = synth.rays_in_box(1048576, v[:, :3].min(0), v[:, :3].max(0), seed=seed + 1)
        dr = torch.from_numpy(rays).cuda()
        full = golden[name]["full_sweep"]
        row = {"mesh": name, "triangles": n, "full_sweep_sah": round(full, 4)}
        plain_sah = None
        for form, w, gate in (("plain", None, False), ("learned", weights, True),
                              ("learned_ungated", weights, False)):
            ctx.set_split_proposer(w, gate)
            ctx.set_proposer_gate(*(learned.RECOMMENDED_GATE if gate else (0.0, 0)))
            ms = []
            for k in range(max(args.warmup, 3) + args.steps):
                flush.fill_(k & 0xFF)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                count, rc, st = build_device(ctx, BvhSettings(), d_nodes, d_perm, vertices=dv,
                                             triangles=dt, out_lens=d_lens, stream=stream)
                e1.record(stream)
                torch.cuda.synchronize()
                ctx.check(rc)
                if k >= max(args.warmup, 3):
                    ms.append(e0.elapsed_time(e1))
            nh = d_nodes[: count * 8].cpu().numpy().view(NODE_DTYPE)
            sah = sah_cost(nh, d_lens[:count].cpu().numpy().view(np.uint32))
            mrays, hits, mism = _trace_rate(tr, d_nodes, count, dv, dt, d_perm, n, dr, rays.shape[0],
                                            stream, flush, 5)
            bms = statistics.median(ms)
            row[form] = {"build_mtris": round(n / (bms * 1e-3) / 1e6, 2), "build_ms": round(bms, 3),
                         "sah": round(sah, 4), "vs_full_sweep_pct": round(100 * (sah / full - 1), 4),
                         "learned_splits": st["learned_splits"], "mrays": round(mrays, 2),
                         "hit_rays": hits, "trace_mismatches_vs_bruteforce_4096": mism}
            if form == "plain":
                plain_sah = sah
            else:
                row[form]["gap_closed_pct"] = round(100 * (plain_sah - sah) / (plain_sah - full), 2)
        ctx.set_split_proposer(None)
        rows.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    clocks.__exit__()
    tr.close()
    rec = learned.load_record()
    out = {
        "metric": "learned split proposer: SAH vs plain binned and full sweep; build Mtri/s; Mrays/s",
        "workload": "learned split proposer, held-out meshes", "dtype": "f32 (network bf16/fp32)",
        "clocks": clocks.summary(),
        "steps": args.steps, "warmup": args.warmup, "results": rows,
        "network": {"samples": rec.get("samples"), "steps": rec.get("steps"),
                    "heldout_accuracy": rec.get("heldout_accuracy")},
        "config": {"medium_max": 1024, "leaf": 1, "max_depth": 32, "profile": "reference",
                   "rays": 1048576, "l2": "flushed before every build and trace",
                   "gate": {"refine_logit_above": learned.RECOMMENDED_GATE[0],
                            "min_objects": learned.RECOMMENDED_GATE[1]}},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse_args()
    if args.workload == "learned":
        run_learned(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "mixed":
        run_mixed(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
