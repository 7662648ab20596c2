"""Autotuner of the builder's per-workload choices; writes tuning.json.

Knobs tuned per workload:
  * medium_max — the size at which nodes leave the level passes for the
    per-subtree kernels (33..1024): the level-to-subtree switch-over.
  * small_threads — the block size of the kernel that builds subtrees of
    <= 32 objects, one warp each (64, 128 or 256 threads per CTA).
  * small_warps — that kernel's resident warps per SM (24 with an 80-register
    budget, or 16 with 126 registers and fewer spills).
  * batch_mode and queue_ctas_per_sm (batched workloads) — level passes and
    subtree launches, or one persistent launch over device-side task queues
    with a given number of resident CTAs per SM.
  * bins — the binned-sweep bin count. The reference profile (bins = 0,
    32 bins) is what the crate builds; other counts change the tree. A
    non-reference count is chosen only for workloads that allow it, and only
    when its total SAH cost is within 1% of the reference profile's.
Every knob but bins changes speed only, never the tree (each phase and
mode computes the same split decisions): the fastest value is taken, the
knobs one after another (switch-over, block size, small-subtree occupancy,
batch mode, persistent CTAs per SM, bins), each at the best values found
before it.

Each candidate is timed on a fresh context as the median of several builds
(CUDA events on the build stream, inputs resident on the device, L2 flushed
before each build): a single mesh through the single-build device entry
point, batched workloads as replays of a captured CUDA graph, the forms the
bench runs.
When a knob's two fastest values are within 5% of each other, they are timed
in turn three more times each and the lower mean wins.
Run on a GPU:  python -m marigold_b200.autotune [--workloads ...]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")

MEDIUM_MAX = (64, 128, 256, 512, 1024)
SMALL_THREADS = (64, 128, 256)
SMALL_WARPS = (16, 24)
QUEUE_CTAS = (1, 2, 3)
BINS = (0, 8, 16, 24)
# repeats of one candidate spread by up to about 3% on the batched scene: the
# two fastest values of a knob within CLOSE of each other are re-timed in turn
CLOSE = 1.05
CONFIRM = 3
DEFAULTS = {"medium_max": 1024, "small_threads": 256, "small_warps": 24, "batch_mode": "levels",
            "queue_ctas_per_sm": 0, "bins": 0}


def load_table() -> dict:
    try:
        with open(TABLE) as f:
            return json.load(f)
    except FileNotFoundError:
        return {}


def choice(workload: str, key: str, default=None):
    d = DEFAULTS.get(key) if default is None else default
    return load_table().get(workload, {}).get("choice", {}).get(key, d)


def apply(ctx, workload: str) -> dict:
    """Sets the speed knobs tuning.json holds for `workload` on a context;
    returns the choices (bins included, which the caller passes in its
    settings)."""
    c = {k: choice(workload, k) for k in DEFAULTS}
    ctx.set_tuning(int(c["medium_max"]))
    ctx.set_launch_shape(int(c["small_threads"]), int(c["queue_ctas_per_sm"]))
    ctx.set_small_occupancy(int(c["small_warps"]))
    ctx.set_batch_mode(c["batch_mode"] == "queue")
    return c


def _workloads():
    from . import synth

    def icosphere():
        v, t = synth.config2_mesh()
        return [{"v": v, "t": t, "bounds": synth.mesh_bounds(v)}], False, False

    def batched():
        meshes, bounds, inst = synth.batched_scene()
        ms = [{"v": v, "t": t, "bounds": b} for (v, t), b in zip(meshes, bounds)]
        ms.append({"aabbs": inst})
        return ms, True, True

    def mixed():
        v, t = synth.mixed_scene()
        return [{"v": v, "t": t, "bounds": None}], False, False

    return {"icosphere_l8": icosphere, "batched_scene": batched, "mixed_scene": mixed}


def _measure(meshes, knobs, batched, reps=5):
    """Median build time (ms) and SAH of one candidate, on a fresh context
    (nothing carried over from the previous candidate): a single mesh through
    the single-build device entry point, batches through the batched one with
    graph capture (replays of the captured graph, the form they run in)."""
    import torch
    from . import BvhSettings, _lib, build_batch_device, build_device
    ctx = _lib.Context(0)
    try:
        ctx.set_tuning(knobs["medium_max"])
        ctx.set_launch_shape(knobs["small_threads"], knobs["queue_ctas_per_sm"])
        ctx.set_small_occupancy(knobs["small_warps"])
        ctx.set_batch_mode(knobs["batch_mode"] == "queue")
        ctx.set_graph_capture(batched)
        total = sum(m["n"] for m in meshes)
        slots = sum(2 * m["n"] - 1 for m in meshes if m["n"])
        nodes = torch.empty(slots * 8, dtype=torch.int32, device="cuda")
        lens = torch.empty(slots, dtype=torch.int32, device="cuda")
        perm = torch.empty(total, dtype=torch.int32, device="cuda")
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        # a stream of its own: graphs cannot be captured on the legacy default
        # stream, where a batched build would run eagerly instead
        stream = torch.cuda.Stream()
        single = not batched and len(meshes) == 1 and "aabbs" not in meshes[0]
        descs = []
        for m in meshes:
            if "aabbs" in m:
                descs.append({"aabbs": m["dev_aabbs"]})
            else:
                descs.append({"vertices": m["dev_v"], "triangles": m["dev_t"], "bounds": m["bounds"]})
        times = []
        offs = [0, slots]
        for k in range(reps + 1):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()  # the flush (on torch's stream) is done before the timed build
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if single:
                m = meshes[0]
                build_device(ctx, BvhSettings(bins=knobs["bins"], bounds=m["bounds"]), nodes, perm,
                             vertices=m["dev_v"], triangles=m["dev_t"], out_lens=lens, stream=stream)
            else:
                offs, rc, st = build_batch_device(ctx, BvhSettings(bins=knobs["bins"]), descs, nodes, perm,
                                                  out_lens=lens, stream=stream)
            e1.record(stream)
            stream.synchronize()
            if k:
                times.append(e0.elapsed_time(e1))
        from .bvh import NODE_DTYPE, sah_cost
        nh = nodes.cpu().numpy().view(NODE_DTYPE)
        lh = lens.cpu().numpy().view(np.uint32)
        sah = sum(sah_cost(nh[offs[i]:offs[i + 1]], lh[offs[i]:offs[i + 1]])
                  for i in range(len(offs) - 1) if offs[i + 1] > offs[i])
        return float(np.median(times)), sah
    finally:
        ctx.close()


def pick_knob(trial, best, key, values):
    """Times each value of one knob with trial(**{key: value}) (which returns
    a row with "ms") and sets best[key] to the fastest. When the two fastest
    are within CLOSE of each other, they are timed in turn CONFIRM more times
    each and the lower mean wins (its first row is returned)."""
    cands = [trial(**{key: v}) for v in values]
    order = sorted(cands, key=lambda r: r["ms"])
    top = order[0]
    if len(order) > 1 and order[1]["ms"] <= CLOSE * top["ms"]:
        a, b = top[key], order[1][key]
        ta, tb = [top["ms"]], [order[1]["ms"]]
        for _ in range(CONFIRM):
            ta.append(trial(**{key: a})["ms"])
            tb.append(trial(**{key: b})["ms"])
        top = order[0] if np.mean(ta) <= np.mean(tb) else order[1]
    best[key] = top[key]
    return top


def tune(names):
    import torch
    table = load_table()
    for name in names:
        meshes, bins_free, batched = _workloads()[name]()
        for m in meshes:
            if "aabbs" in m:
                m["dev_aabbs"] = torch.from_numpy(m["aabbs"]).cuda()
                m["n"] = m["aabbs"].shape[0]
            else:
                m["dev_v"] = torch.from_numpy(m["v"]).cuda()
                m["dev_t"] = torch.from_numpy(m["t"].view(np.int32)).cuda()
                m["n"] = m["t"].shape[0]
        rows = []
        best = dict(DEFAULTS)

        def trial(**change):
            k = dict(best, **change)
            ms, sah = _measure(meshes, k, batched)
            rows.append(dict(k, ms=round(ms, 4), sah=sah))
            print(name, rows[-1], file=sys.stderr, flush=True)
            return rows[-1]

        def pick(key, values):
            return pick_knob(trial, best, key, values)

        pick("medium_max", MEDIUM_MAX)
        pick("small_threads", SMALL_THREADS)
        pick("small_warps", SMALL_WARPS)
        if batched:
            pick("batch_mode", ("levels", "queue"))
            if best["batch_mode"] == "queue":
                pick("queue_ctas_per_sm", QUEUE_CTAS + (0,))
        ref = min((r for r in rows if r["bins"] == 0), key=lambda r: r["ms"])
        ref_sah = ref["sah"]
        chosen_ms = ref["ms"]
        if bins_free:
            for b in BINS[1:]:
                r = trial(bins=b)
                if r["sah"] <= 1.01 * ref_sah and r["ms"] < chosen_ms:
                    best["bins"] = b
                    chosen_ms = r["ms"]
        table[name] = {
            "choice": dict(best),
            "reference_profile_sah": ref_sah,
            "candidates": rows,
            "rule": ("knobs that leave the tree unchanged (medium_max, small_threads, small_warps, "
                     "batch_mode, queue_ctas_per_sm): the fastest, one knob after another; bins other than the "
                     "reference profile only where allowed and within 1% of its SAH")
                    + ("" if bins_free else "; bins fixed to the reference profile"),
            "measured": time.strftime("%Y-%m-%d"),
        }
        with open(TABLE, "w") as f:
            json.dump(table, f, indent=1)
    return table


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", nargs="*", default=["icosphere_l8", "batched_scene"])
    a = ap.parse_args()
    tune(a.workloads)
    print(json.dumps(load_table(), indent=1))
