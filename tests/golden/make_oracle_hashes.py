"""Writes oracle_hashes.json: sha256 of the oracle's output (node words,
per-node object counts, permutation) for the two single-mesh workloads at
their fixed seeds, in both knob profiles each:

  config1  65,536 random triangles (seed 1), root bounds = mesh bounds
           reference profile; 16 bins with the adaptive sweep off
  config2  noisy icosphere level 8, 1,310,720 triangles (seed 2), root
           bounds = mesh bounds; reference profile; 16 adaptive thresholds

The CPU tests check the oracle still produces these bytes; the GPU tests
check the CUDA builder produces them too, without running the oracle.
Also recorded: the oracle's tie events and order-dependent nodes (splits
picked by list order among equal-cost splits over different sets).

Run from the repository root:  python tests/golden/make_oracle_hashes.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from marigold_b200 import synth  # noqa: E402
from oracle import oracle  # noqa: E402

CASES = {
    "config1_reference": ("config1", {}),
    "config1_bins16_adaptive_off": ("config1", {"bins": 16, "adaptive_max_n": 0}),
    "config2_reference": ("config2", {}),
    "config2_adaptive_steps16": ("config2", {"adaptive_steps": 16}),
}


def mesh(name):
    return synth.config1_mesh() if name == "config1" else synth.config2_mesh()


def digest(nodes, lens, perm):
    """sha256 over the little-endian u32 words of nodes, then lens, then perm."""
    h = hashlib.sha256()
    for a in (nodes, lens, perm):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


def main():
    oracle.build_library()
    out = {}
    for key, (name, kw) in CASES.items():
        v, t = mesh(name)
        r = oracle.build(v, t, root_bounds=synth.mesh_bounds(v), **kw)
        assert r["status"] == 0
        out[key] = {"mesh": name, "knobs": kw, "nodes": int(r["nodes"].shape[0]),
                    "sha256": digest(r["nodes"], r["lens"], r["perm"]),
                    "tie_events": int(r["tie_events"]), "order_dependent": int(r["order_dependent"])}
        print(key, out[key], flush=True)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_hashes.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
