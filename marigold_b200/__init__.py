"""marigold_b200 — B200-native SAH BVH builder, a drop-in for marigold's `bvh` crate.

The builder itself is CUDA (csrc/, compiled to libmgbvh.so with the C ABI of
include/mgbvh.h); this package holds its Python binding and host-side mirror
of the crate's interface, plus seeded synthetic workloads.
"""
from ._lib import Context, MgbvhError  # noqa: F401
from .bvh import (  # noqa: F401
    NODE_DTYPE,
    BoundingVolume,
    BoundingVolumeHierarchy,
    BvhSettings,
    build_batch_device,
    build_device,
    encode_gpu_bytes,
    sah_cost,
)
