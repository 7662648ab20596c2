"""The learned split proposer: sample generation, training and evaluation.

Everything runs on the GPU through libmgbvh.so:
  * samples: builds of synthetic meshes (random small triangles, noisy
    icospheres and small mixed scenes, fresh seeds) in sample mode, where the
    builder writes, for every binned node of 33..8192 objects, its 24
    features and the exact full-sweep SAH optimum (axis, 1/16 position
    bucket) plus whether that optimum beats the plain binned split
    (mgbvh_set_sample_output);
  * training: the project's own forward/backward kernels (BF16 weights,
    FP32 accumulation) and Adam on FP32 master weights;
  * use: mgbvh_set_split_proposer, after which builds score the network's
    proposals exactly and keep the plain split unless a proposal is cheaper.

The trained parameters are kept in proposer_weights.bin (8,945 BF16 values)
with their training record in proposer_weights.json.

Run on a GPU:  python -m marigold_b200.learned --samples 20000000 --steps 80000
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "proposer_weights.bin")
RECORD = os.path.join(HERE, "proposer_weights.json")
NPARAM = 8945
SAMPLE_WIDTH = 30


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


TRAINING_KINDS = ("random", "icosphere", "mixed")


def training_mesh(k: int, seed: int, kinds=TRAINING_KINDS):
    """Mesh k of a training stream, cycling through `kinds`, each mesh with
    its own seed: random small triangles (65,536 / 262,144 / 1,048,576),
    noisy icospheres (levels 6 / 7 / 8), and small mixed scenes (Gaussian
    blobs, a ground grid and long thin triangles, about 0.23M / 0.92M / 1.8M
    triangles: the large mixed scene's generator at reduced sizes)."""
    from . import synth
    s = seed + 7919 * k
    kind = kinds[k % len(kinds)]
    size = (k // len(kinds)) % 3
    if kind == "random":
        return synth.random_triangles([65536, 262144, 1048576][size], seed=s)
    if kind == "icosphere":
        return synth.noisy_icosphere([6, 7, 8][size], seed=s)
    blob, grid, thin = [(131072, (128, 128), 65536), (524288, (256, 256), 262144),
                        (1048576, (512, 256), 524288)][size]
    return synth.mixed_scene(seed=s, n_blob=blob, grid=grid, n_thin=thin)


# held-out evaluation meshes (seeds never drawn by training_mesh's streams):
# the 65,536-triangle random mesh and the level-8 noisy icosphere generators
EVAL_MESHES = (("random65536_s9001", "random", 65536, 9001),
               ("icosphere8_s9002", "icosphere", 8, 9002))


# the large mixed scene's generator (its seed, 5) at 1/4 size and at full size
# (16,777,216 triangles): the learned form's evaluation on scenes unlike
# single meshes; size is the divisor of the scene's parts
EVAL_SCENES = (("mixed_quarter_s5", "mixed", 4, 5), ("mixed_full_s5", "mixed", 1, 5))

# The gate the library's users should set with mgbvh_set_proposer_gate for
# the committed network: proposals are scored where the refine logit is above
# 0, and the network runs only on nodes of 2,048 objects or more (above every
# subtree CTA's size, so the subtree kernels run their plain form): on the
# level-8 icosphere 0.81x the plain build's speed for 35% of the SAH gap to
# a full sweep (1,025 objects: 0.80x for 43%). The library's own default
# (0, 0) runs the network at every binned node.
RECOMMENDED_GATE = (0.0, 2048)


def eval_mesh(kind: str, size: int, seed: int):
    from . import synth
    if kind == "random":
        return synth.random_triangles(size, seed=seed)
    if kind == "mixed":
        return synth.mixed_scene(seed=seed, n_blob=8388608 // size, grid=(2048, 1024 // size),
                                 n_thin=4194304 // size)
    return synth.noisy_icosphere(size, seed=seed)


def generate_samples(n_target: int, seed: int = 424242, ctx=None, log=print, workers: int = 0):
    """GPU-built training samples: float32 [K, 30] (torch, on the device).

    Meshes are generated on host processes (a spawn pool) while the GPU
    builds the previous ones."""
    import concurrent.futures as cf
    import multiprocessing as mp

    import torch
    from . import BvhSettings, _lib, build_device, synth
    own = ctx is None
    ctx = ctx or _lib.Context(0)
    workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
    chunks = []
    total = 0
    with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as pool:
        k = 0
        pending = []
        while total < n_target:
            while len(pending) < 2 * workers:
                pending.append(pool.submit(training_mesh, k, seed))
                k += 1
            v, t = pending.pop(0).result()
            n = t.shape[0]
            dv = torch.from_numpy(v).cuda()
            dt = torch.from_numpy(t.view(np.int32)).cuda()
            cap = max(n // 4, 1024)
            out = torch.empty(cap * SAMPLE_WIDTH, dtype=torch.float32, device="cuda")
            cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
            ctx.set_sample_output(out, cap, cnt)
            nodes = torch.empty((2 * n - 1) * 8, dtype=torch.int32, device="cuda")
            perm = torch.empty(n, dtype=torch.int32, device="cuda")
            _, rc, _ = build_device(ctx, BvhSettings(bounds=synth.mesh_bounds(v)), nodes, perm,
                                    vertices=dv, triangles=dt)
            ctx.check(rc)
            torch.cuda.synchronize()
            got = min(int(cnt.item()), cap)
            chunks.append(out[: got * SAMPLE_WIDTH].view(got, SAMPLE_WIDTH).clone())
            total += got
            log(f"samples: +{got} from {n} triangles (total {total})")
        for f in pending:
            f.cancel()
    ctx.set_sample_output(None)
    if own:
        ctx.close()
    return torch.cat(chunks)[:n_target]


def init_params(seed: int = 7) -> np.ndarray:
    """FP32 initial parameters: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in))."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    for off, rows, cols in ((0, 64, 24), (1600, 64, 64), (5760, 49, 64)):
        lim = 1.0 / np.sqrt(cols)
        p[off:off + rows * cols] = rng.uniform(-lim, lim, rows * cols)
        p[off + rows * cols:off + rows * cols + rows] = rng.uniform(-lim, lim, rows)
    return p


def to_bf16_bits(p: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(p, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def train(samples, steps: int = 4000, batch: int = 4096, lr: float = 2e-3, seed: int = 7,
          log=print):
    """Train on GPU samples (torch [K, 30]); returns (bf16 bits, record)."""
    import torch
    from . import _lib
    L = _lib.load()
    K = samples.shape[0]
    x = samples[:, :24].contiguous()
    lab = samples[:, 24].contiguous().view(torch.int32)
    gain = samples[:, 25].contiguous()
    master = torch.from_numpy(init_params(seed)).cuda()
    w = torch.from_numpy(to_bf16_bits(master.cpu().numpy()).view(np.int16)).cuda()
    m = torch.zeros(NPARAM, dtype=torch.float32, device="cuda")
    v = torch.zeros(NPARAM, dtype=torch.float32, device="cuda")
    grad = torch.zeros(NPARAM, dtype=torch.float32, device="cuda")
    loss = torch.zeros(2, dtype=torch.float32, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    stream = torch.cuda.current_stream().cuda_stream
    curve = []
    t0 = time.perf_counter()
    for step in range(1, steps + 1):
        idx = torch.randint(0, K, (batch,), device="cuda", generator=g)
        bx, bl, bg = x[idx].contiguous(), lab[idx].contiguous(), gain[idx].contiguous()
        grad.zero_()
        loss.zero_()
        rc = L.mgbvh_mlp_train_step_dev(_vp(bx), _vp(bl), _vp(bg), batch, _vp(w), _vp(grad),
                                        _vp(loss), ctypes.c_void_p(stream))
        if rc:
            raise RuntimeError(f"train step failed: {rc}")
        lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * step / steps))  # cosine decay
        rc = L.mgbvh_mlp_adam_dev(_vp(master), _vp(w), _vp(grad), _vp(m), _vp(v), step, lr_t, 0.9,
                                  0.999, 1e-8, ctypes.c_void_p(stream))
        if rc:
            raise RuntimeError(f"adam step failed: {rc}")
        if step % 200 == 0 or step == 1:
            ce, bce = (loss / batch).tolist()
            curve.append({"step": step, "ce": round(ce, 4), "bce": round(bce, 4)})
            log(f"step {step}: ce {ce:.4f} bce {bce:.4f}")
    torch.cuda.synchronize()
    bits = w.cpu().numpy().view(np.uint16).copy()
    record = {"samples": int(K), "steps": steps, "batch": batch, "lr": lr, "seed": seed,
              "train_seconds": round(time.perf_counter() - t0, 2), "loss_curve": curve}
    return bits, record


def accuracy(samples, bits):
    """Top-1 / top-2 position accuracy and refine accuracy of a network."""
    import torch
    from . import _lib
    L = _lib.load()
    x = samples[:, :24].contiguous()
    out = torch.empty(samples.shape[0] * 49, dtype=torch.float32, device="cuda")
    w = torch.from_numpy(bits.view(np.int16)).cuda()
    rc = L.mgbvh_mlp_forward_dev(_vp(x), samples.shape[0], _vp(w), _vp(out),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc:
        raise RuntimeError(f"forward failed: {rc}")
    out = out.view(-1, 49)
    lab = samples[:, 24].contiguous().view(torch.int32).long()
    ok = lab >= 0
    top2 = out[:, :48].topk(2, dim=1).indices
    t1 = (top2[:, 0] == lab)[ok].float().mean().item()
    t2 = ((top2[:, 0] == lab) | (top2[:, 1] == lab))[ok].float().mean().item()
    ref = ((out[:, 48] > 0).float() == samples[:, 25]).float().mean().item()
    return {"top1": round(t1, 4), "top2": round(t2, 4), "refine": round(ref, 4)}


def load_weights() -> np.ndarray:
    """The committed trained parameters (8,945 BF16 values as uint16)."""
    w = np.fromfile(WEIGHTS, dtype=np.uint16)
    if w.shape[0] != NPARAM:
        raise ValueError(f"{WEIGHTS}: {w.shape[0]} values, expected {NPARAM}")
    return w


def load_record() -> dict:
    with open(RECORD) as f:
        return json.load(f)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=5_000_000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args()
    log = lambda s: print(s, file=sys.stderr, flush=True)  # noqa: E731
    t0 = time.perf_counter()
    train_set = generate_samples(a.samples, seed=424242, log=log)
    gen_s = time.perf_counter() - t0
    held = generate_samples(200_000, seed=977, log=log)
    bits, rec = train(train_set, steps=a.steps, batch=a.batch, log=log)
    rec["generation_seconds"] = round(gen_s, 1)
    rec["train_accuracy"] = accuracy(train_set[:200_000], bits)
    rec["heldout_accuracy"] = accuracy(held, bits)
    rec["heldout_refine_rate"] = round(float(held[:, 25].mean().item()), 4)
    bits.tofile(a.out)
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
