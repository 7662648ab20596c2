"""ctypes binding of ``libmgbvh.so`` (the C ABI in include/mgbvh.h).

The library is the only compute path: there is no CPU fallback. Loading
fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgbvh.so")

OK = 0
WARN_EMPTY = 1
WARN_INFEASIBLE = 2
ERR_INVALID_ARG = -1
ERR_CAPACITY = -2
ERR_CUDA = -3
ERR_TIMEOUT = -4
ERR_ASSERT = -5
ERR_UNSUPPORTED = -6
ERR_NO_DEVICE = -7
ERR_TOO_LARGE = -8
NOALLOC_MAX_OBJECTS = 1024

# every entry point declared in include/mgbvh.h
EXPORTED = (
    "mgbvh_default_settings", "mgbvh_create", "mgbvh_destroy", "mgbvh_set_stream",
    "mgbvh_last_error", "mgbvh_status_string", "mgbvh_build_indexed", "mgbvh_build_aabbs",
    "mgbvh_build_indexed_dev", "mgbvh_build_aabbs_dev", "mgbvh_encode_gpu_bytes",
    "mgbvh_sah_cost", "mgbvh_build_aabbs_noalloc", "mgbvh_tracer_create", "mgbvh_tracer_destroy",
    "mgbvh_tracer_set_blas_dev", "mgbvh_trace_closest_dev", "mgbvh_trace_bruteforce_dev",
    "mgbvh_build_batch_dev", "mgbvh_set_tuning", "mgbvh_set_graph_capture",
    "mgbvh_mlp_train_step_dev", "mgbvh_mlp_forward_dev", "mgbvh_mlp_adam_dev",
    "mgbvh_set_split_proposer", "mgbvh_set_sample_output", "mgbvh_instance_aabbs_dev",
    "mgbvh_tracer_build_wide", "mgbvh_tracer_wide_nodes", "mgbvh_trace_closest_wide_dev",
    "mgbvh_tracer_set_scene_dev", "mgbvh_trace_scene_dev", "mgbvh_trace_scene_bruteforce_dev",
    "mgbvh_set_batch_mode", "mgbvh_set_queue_limits", "mgbvh_set_launch_shape", "mgbvh_set_proposer_gate",
    "mgbvh_set_small_occupancy",
)
BATCH_LEVELS = 0
BATCH_QUEUE = 1


class Node(ctypes.Structure):
    """mgbvh_node: 32 bytes, AsGpuBytes layout for MAX_LEAF_OBJECTS == 1."""

    _fields_ = [("min", ctypes.c_float * 3), ("start_index", ctypes.c_uint32),
                ("max", ctypes.c_float * 3), ("child_node", ctypes.c_uint32)]


class Settings(ctypes.Structure):
    _fields_ = [
        ("min_leaf_objects", ctypes.c_uint32),
        ("max_leaf_objects", ctypes.c_uint32),
        ("max_depth", ctypes.c_uint32),
        ("has_bounds", ctypes.c_uint32),
        ("bounds", ctypes.c_float * 6),
        ("bins", ctypes.c_uint32),
        ("adaptive_max_n", ctypes.c_uint32),
        ("adaptive_steps", ctypes.c_uint32),
        ("profiling_info", ctypes.c_uint32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("construction_time", ctypes.c_double),
        ("node_count", ctypes.c_uint32),
        ("leaf_node_count", ctypes.c_uint32),
        ("min_leaf_object_count", ctypes.c_uint32),
        ("max_leaf_object_count", ctypes.c_uint32),
        ("avg_leaf_object_count", ctypes.c_double),
        ("stddev_leaf_object_count", ctypes.c_double),
        ("total_object_count", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("max_depth", ctypes.c_uint32),
        ("median_splits", ctypes.c_uint32),
        ("depth_capped_leaves", ctypes.c_uint32),
        ("feasible", ctypes.c_uint32),
        ("kernel_launches", ctypes.c_uint32),
        ("levels", ctypes.c_uint32),
        ("phase_seconds", ctypes.c_double * 4),
        ("graph_replay", ctypes.c_uint32),
        ("learned_splits", ctypes.c_uint32),
    ]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["phase_seconds"] = list(self.phase_seconds)
        return d


class MeshDesc(ctypes.Structure):
    """mgbvh_mesh_desc: one mesh of a batched build (device pointers)."""

    _fields_ = [
        ("vertices", ctypes.c_void_p),
        ("vertex_stride_bytes", ctypes.c_uint32),
        ("vertex_count", ctypes.c_uint32),
        ("triangles", ctypes.c_void_p),
        ("aabbs", ctypes.c_void_p),
        ("count", ctypes.c_uint32),
        ("has_bounds", ctypes.c_uint32),
        ("bounds", ctypes.c_float * 6),
    ]


class MgbvhError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"mgbvh status {status}: {message}")
        self.status = status


_lock = threading.Lock()
_lib = None


def load():
    """Load libmgbvh.so and declare its prototypes."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m marigold_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        u32 = ctypes.c_uint32
        pu32 = ctypes.POINTER(u32)
        L.mgbvh_default_settings.argtypes = [ctypes.POINTER(Settings)]
        L.mgbvh_default_settings.restype = None
        L.mgbvh_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
        L.mgbvh_create.restype = ctypes.c_int
        L.mgbvh_destroy.argtypes = [P]
        L.mgbvh_destroy.restype = None
        L.mgbvh_set_stream.argtypes = [P, P]
        L.mgbvh_set_stream.restype = ctypes.c_int
        L.mgbvh_last_error.argtypes = [P]
        L.mgbvh_last_error.restype = ctypes.c_char_p
        L.mgbvh_status_string.argtypes = [ctypes.c_int]
        L.mgbvh_status_string.restype = ctypes.c_char_p
        build_args = [P, P, u32, u32, P, u32, ctypes.POINTER(Settings), P, u32, pu32, P, P,
                      ctypes.POINTER(Stats)]
        L.mgbvh_build_indexed.argtypes = build_args
        L.mgbvh_build_indexed.restype = ctypes.c_int
        L.mgbvh_build_indexed_dev.argtypes = build_args
        L.mgbvh_build_indexed_dev.restype = ctypes.c_int
        aabb_args = [P, P, u32, ctypes.POINTER(Settings), P, u32, pu32, P, P, ctypes.POINTER(Stats)]
        L.mgbvh_build_aabbs.argtypes = aabb_args
        L.mgbvh_build_aabbs.restype = ctypes.c_int
        L.mgbvh_build_aabbs_dev.argtypes = aabb_args
        L.mgbvh_build_aabbs_dev.restype = ctypes.c_int
        L.mgbvh_encode_gpu_bytes.argtypes = [P, P, u32, u32, P]
        L.mgbvh_encode_gpu_bytes.restype = ctypes.c_int
        L.mgbvh_build_aabbs_noalloc.argtypes = [P, u32, ctypes.POINTER(Settings), P, u32, pu32, P,
                                                P, P]
        L.mgbvh_build_aabbs_noalloc.restype = ctypes.c_int
        L.mgbvh_tracer_create.argtypes = [ctypes.c_int, ctypes.POINTER(P)]
        L.mgbvh_tracer_create.restype = ctypes.c_int
        L.mgbvh_tracer_destroy.argtypes = [P]
        L.mgbvh_tracer_destroy.restype = None
        L.mgbvh_tracer_set_blas_dev.argtypes = [P, P, u32, P, P, u32, u32, P, P, u32, P]
        L.mgbvh_tracer_set_blas_dev.restype = ctypes.c_int
        L.mgbvh_trace_closest_dev.argtypes = [P, P, u32, P, P, ctypes.POINTER(ctypes.c_uint64),
                                              ctypes.POINTER(ctypes.c_double), P]
        L.mgbvh_trace_closest_dev.restype = ctypes.c_int
        L.mgbvh_tracer_build_wide.argtypes = [P, P, pu32]
        L.mgbvh_tracer_build_wide.restype = ctypes.c_int
        L.mgbvh_tracer_wide_nodes.argtypes = [P, ctypes.POINTER(P), pu32]
        L.mgbvh_tracer_wide_nodes.restype = ctypes.c_int
        L.mgbvh_trace_closest_wide_dev.argtypes = [P, P, u32, P, P, ctypes.POINTER(ctypes.c_uint64),
                                                   ctypes.POINTER(ctypes.c_double), P]
        L.mgbvh_trace_closest_wide_dev.restype = ctypes.c_int
        L.mgbvh_trace_bruteforce_dev.argtypes = [P, P, u32, P, P, P]
        L.mgbvh_trace_bruteforce_dev.restype = ctypes.c_int
        L.mgbvh_tracer_set_scene_dev.argtypes = [P, P, u32, P, P, u32, P, u32, P, u32, P, P, u32, u32, P, u32,
                                                 P]
        L.mgbvh_tracer_set_scene_dev.restype = ctypes.c_int
        L.mgbvh_trace_scene_dev.argtypes = [P, P, u32, P, P, P, ctypes.POINTER(ctypes.c_uint64),
                                            ctypes.POINTER(ctypes.c_double), P]
        L.mgbvh_trace_scene_dev.restype = ctypes.c_int
        L.mgbvh_trace_scene_bruteforce_dev.argtypes = [P, P, u32, P, P, P, ctypes.c_int, P]
        L.mgbvh_trace_scene_bruteforce_dev.restype = ctypes.c_int
        L.mgbvh_build_batch_dev.argtypes = [P, ctypes.POINTER(MeshDesc), u32, ctypes.POINTER(Settings),
                                            P, u32, P, P, pu32, ctypes.POINTER(Stats)]
        L.mgbvh_build_batch_dev.restype = ctypes.c_int
        L.mgbvh_mlp_train_step_dev.argtypes = [P, P, P, u32, P, P, P, P]
        L.mgbvh_mlp_train_step_dev.restype = ctypes.c_int
        L.mgbvh_mlp_forward_dev.argtypes = [P, u32, P, P, P]
        L.mgbvh_mlp_forward_dev.restype = ctypes.c_int
        f32 = ctypes.c_float
        L.mgbvh_mlp_adam_dev.argtypes = [P, P, P, P, P, u32, f32, f32, f32, f32, P]
        L.mgbvh_mlp_adam_dev.restype = ctypes.c_int
        L.mgbvh_set_split_proposer.argtypes = [P, P, ctypes.c_int]
        L.mgbvh_set_split_proposer.restype = ctypes.c_int
        L.mgbvh_set_sample_output.argtypes = [P, P, u32, P]
        L.mgbvh_set_sample_output.restype = ctypes.c_int
        L.mgbvh_set_graph_capture.argtypes = [P, ctypes.c_int]
        L.mgbvh_set_graph_capture.restype = ctypes.c_int
        L.mgbvh_instance_aabbs_dev.argtypes = [P, P, u32, P, P, u32, P]
        L.mgbvh_instance_aabbs_dev.restype = ctypes.c_int
        L.mgbvh_set_tuning.argtypes = [P, u32]
        L.mgbvh_set_tuning.restype = ctypes.c_int
        L.mgbvh_set_batch_mode.argtypes = [P, ctypes.c_int]
        L.mgbvh_set_batch_mode.restype = ctypes.c_int
        L.mgbvh_set_queue_limits.argtypes = [P, u32, u32]
        L.mgbvh_set_queue_limits.restype = ctypes.c_int
        L.mgbvh_set_launch_shape.argtypes = [P, u32, u32]
        L.mgbvh_set_launch_shape.restype = ctypes.c_int
        L.mgbvh_set_small_occupancy.argtypes = [P, u32]
        L.mgbvh_set_small_occupancy.restype = ctypes.c_int
        L.mgbvh_set_proposer_gate.argtypes = [P, ctypes.c_float, u32]
        L.mgbvh_set_proposer_gate.restype = ctypes.c_int
        L.mgbvh_sah_cost.argtypes = [P, P, u32]
        L.mgbvh_sah_cost.restype = ctypes.c_double
        _lib = L
    return _lib


def status_string(status: int) -> str:
    return load().mgbvh_status_string(status).decode()


class Context:
    """An mgbvh_ctx: one CUDA device, its stream and scratch buffers."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.ptr = ctypes.c_void_p()
        rc = self.L.mgbvh_create(device, ctypes.byref(self.ptr))
        if rc != OK:
            raise MgbvhError(rc, status_string(rc))

    def last_error(self) -> str:
        return self.L.mgbvh_last_error(self.ptr).decode()

    def check(self, rc: int) -> int:
        if rc < 0:
            raise MgbvhError(rc, f"{status_string(rc)}: {self.last_error()}")
        return rc

    def set_stream(self, stream_handle: int | None):
        self.check(self.L.mgbvh_set_stream(self.ptr, ctypes.c_void_p(stream_handle or 0)))

    def set_tuning(self, medium_max: int):
        self.check(self.L.mgbvh_set_tuning(self.ptr, medium_max))

    def set_batch_mode(self, queue: bool):
        """Batched builds by one persistent launch over device-side task
        queues (True) or by level passes and subtree launches (False)."""
        self.check(self.L.mgbvh_set_batch_mode(self.ptr, BATCH_QUEUE if queue else BATCH_LEVELS))

    def set_queue_limits(self, wait_us: int = 0, held_tasks: int = 0):
        self.check(self.L.mgbvh_set_queue_limits(self.ptr, wait_us, held_tasks))

    def set_launch_shape(self, small_threads: int = 0, queue_ctas_per_sm: int = 0):
        self.check(self.L.mgbvh_set_launch_shape(self.ptr, small_threads, queue_ctas_per_sm))

    def set_small_occupancy(self, warps_per_sm: int = 0):
        """Resident warps per SM of the small-subtree kernel: 24 (0) or 16."""
        self.check(self.L.mgbvh_set_small_occupancy(self.ptr, warps_per_sm))

    def set_proposer_gate(self, refine_threshold: float = 0.0, min_objects: int = 0):
        """The learned form's cost knobs (see include/mgbvh.h)."""
        self.check(self.L.mgbvh_set_proposer_gate(self.ptr, refine_threshold, min_objects))

    def set_graph_capture(self, on: bool):
        self.check(self.L.mgbvh_set_graph_capture(self.ptr, 1 if on else 0))

    def set_split_proposer(self, weights_bf16=None, gate: bool = True):
        """Device BF16 parameter tensor (8,945 values; the library keeps its
        own copy) or None to build with the plain binned split only."""
        p = ctypes.c_void_p(weights_bf16.data_ptr()) if weights_bf16 is not None else None
        self.check(self.L.mgbvh_set_split_proposer(self.ptr, p, 1 if gate else 0))

    def set_sample_output(self, samples=None, capacity: int = 0, count=None):
        """Device float32 buffer of capacity x 30 values and a uint32/int32
        counter (both kept alive by the caller), or None to stop sampling."""
        if samples is None:
            self.check(self.L.mgbvh_set_sample_output(self.ptr, None, 0, None))
            return
        self.check(self.L.mgbvh_set_sample_output(self.ptr, ctypes.c_void_p(samples.data_ptr()),
                                                  capacity, ctypes.c_void_p(count.data_ptr())))

    def close(self):
        if self.ptr:
            self.L.mgbvh_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tracer:
    """An mgbvh_tracer: closest-hit traversal of one built BLAS on one device."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.ptr = ctypes.c_void_p()
        rc = self.L.mgbvh_tracer_create(device, ctypes.byref(self.ptr))
        if rc != OK:
            raise MgbvhError(rc, status_string(rc))

    def check(self, rc: int) -> int:
        if rc < 0:
            raise MgbvhError(rc, status_string(rc))
        return rc

    def close(self):
        if self.ptr:
            self.L.mgbvh_tracer_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
