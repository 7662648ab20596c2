"""Writes full_sweep_sah.json: SAH cost (mgbvh_sah_cost) of the oracle's
plain and full-sweep trees of the learned proposer's held-out evaluation
meshes and scenes (marigold_b200.learned.EVAL_MESHES, EVAL_SCENES). The full sweep takes every
centroid as a threshold on every axis at every node; it is the quality
yardstick the learned form is measured against.

Run from the repository root:  python tests/golden/make_full_sweep_sah.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from marigold_b200 import learned  # noqa: E402
from marigold_b200.bvh import NODE_DTYPE, sah_cost  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    oracle.build_library()
    out = {}
    for name, kind, size, seed in learned.EVAL_MESHES + learned.EVAL_SCENES:
        v, t = learned.eval_mesh(kind, size, seed)
        row = {"triangles": int(t.shape[0])}
        for key, kw in (("plain", {}), ("full_sweep", {"full_sweep": True})):
            r = oracle.build(v, t, vertex_stride_bytes=4 * v.shape[1], **kw)
            assert r["status"] == 0
            row[key] = sah_cost(r["nodes"].view(NODE_DTYPE).reshape(-1), r["lens"])
        out[name] = row
        print(name, row, flush=True)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "full_sweep_sah.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
