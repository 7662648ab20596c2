/*
 * mgbvh.h — C ABI of the B200-native SAH BVH builder.
 *
 * This is the drop-in boundary for marigold's `bvh` crate. Each entry point
 * replaces one piece of the crate's public interface (paths are relative to
 * the marigold repository):
 *
 *   BoundingVolumeHierarchy::<MIN,MAX>::new(list, source, settings)
 *       bvh/src/lib.rs:698-878
 *       -> mgbvh_build_indexed   (T = MeshTriangle, S = MeshVertex;
 *                                 mesh_interface/src/lib.rs:19-30)
 *       -> mgbvh_build_aabbs     (any T: AsBoundingVolume, e.g. the TLAS over
 *                                 UploadedMesh, mesh_interface/src/lib.rs:87-91)
 *   BoundingVolumeHierarchy::nodes / into_nodes   bvh/src/lib.rs:880-886
 *       -> the out_nodes / out_lens arrays
 *   the in-place permutation of `list`            bvh/src/lib.rs:597-612
 *       -> out_perm (out_perm[i] = original index of the object now at i)
 *   AsGpuBytes for BvhNode                        bvh/src/lib.rs:157-212
 *       -> mgbvh_node (exact bytes when MAX_LEAF_OBJECTS == 1)
 *       -> mgbvh_encode_gpu_bytes (the packed form for MAX_LEAF_OBJECTS > 1)
 *   BvhProfilingInfo                              bvh/src/lib.rs:676-689, 767-875
 *       -> mgbvh_stats
 *
 * The builder runs on one CUDA device. There is no CPU fallback: without a
 * usable device every build returns MGBVH_ERR_NO_DEVICE.
 *
 * Threading: one mgbvh_ctx per calling thread. Calls on distinct contexts may
 * run concurrently (the crate is called from rayon workers, one mesh each,
 * marigold/src/app/data/scene/model.rs:77-95). A context is not thread-safe.
 *
 * Errors: no exceptions cross this ABI. Negative status = error, nothing
 * valid written; positive status = warning, outputs valid.
 */
#ifndef MGBVH_H
#define MGBVH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGBVH_ABI_VERSION 1

#if defined(__GNUC__)
#define MGBVH_API __attribute__((visibility("default")))
#else
#define MGBVH_API
#endif

typedef enum mgbvh_status {
    MGBVH_OK = 0,
    /* Empty object list: zero nodes written. The crate logs a warning and
       returns an empty hierarchy (bvh/src/lib.rs:703-708). */
    MGBVH_WARN_EMPTY = 1,
    /* MIN/MAX leaf bounds cannot all be met for this object count; the tree is
       built and follows the max rule first (bvh/src/lib.rs:710-726). */
    MGBVH_WARN_INFEASIBLE = 2,
    MGBVH_ERR_INVALID_ARG = -1,
    MGBVH_ERR_CAPACITY = -2,   /* node_capacity too small for the result */
    MGBVH_ERR_CUDA = -3,       /* a CUDA runtime call failed */
    MGBVH_ERR_TIMEOUT = -4,    /* a bounded device-side wait gave up */
    /* One of the crate's release-mode assertions would have panicked
       (bvh/src/lib.rs:588, 618-646): child counts or centroid containment. */
    MGBVH_ERR_ASSERT = -5,
    MGBVH_ERR_UNSUPPORTED = -6, /* a knob or size outside this build's limits */
    MGBVH_ERR_NO_DEVICE = -7,
    MGBVH_ERR_TOO_LARGE = -8    /* above MGBVH_NOALLOC_MAX_OBJECTS (allocation-free build) */
} mgbvh_status;

/* Largest object count mgbvh_build_aabbs_noalloc accepts. */
#define MGBVH_NOALLOC_MAX_OBJECTS 1024

/* One node, 32 bytes. For MAX_LEAF_OBJECTS == 1 these are exactly the bytes
   AsGpuBytes writes (bvh/src/lib.rs:163-169) and scene.slang's BvhNode reads.
   child_node == 0 marks a leaf (the root, index 0, is nobody's child); the
   children of an inner node are child_node (gt side) and child_node + 1
   (lt side), bvh/src/lib.rs:650-653. */
typedef struct mgbvh_node {
    float min[3];
    uint32_t start_index;
    float max[3];
    uint32_t child_node;
} mgbvh_node;

/* BvhSettings (bvh/src/lib.rs:668-674) plus the const generics and the split
   knobs. Fill with mgbvh_default_settings(), which sets the reference profile:
   32 bins above 32 objects, adaptive sweep at or below 32 objects with
   len.clamp(8,32) steps, exact centroid thresholds below 8 objects. */
typedef struct mgbvh_settings {
    uint32_t min_leaf_objects; /* MIN_LEAF_OBJECTS (>= 1) */
    uint32_t max_leaf_objects; /* MAX_LEAF_OBJECTS (>= 1) */
    uint32_t max_depth;        /* BvhSettings::max_depth */
    uint32_t has_bounds;       /* BvhSettings::bounds is Some(..) */
    float bounds[6];           /* min xyz, max xyz when has_bounds */
    /* Split knobs. The reference has none of these (its values are
       hard-wired at bvh/src/lib.rs:343, 399, 430, 518); defaults reproduce it. */
    uint32_t bins;           /* 0: len.clamp(16,32); else a fixed count 2..32 */
    uint32_t adaptive_max_n; /* nodes with len <= this use the adaptive sweep
                                (reference 32, max 32); 0 turns it off */
    uint32_t adaptive_steps; /* 0: len.clamp(8,32) thresholds for len >= 8;
                                else a fixed count 1..32 */
    uint32_t profiling_info; /* fill mgbvh_stats leaf statistics */
} mgbvh_settings;

/* BvhProfilingInfo field set (bvh/src/lib.rs:676-689), plus counters that
   the reference does not keep. construction_time is device time in seconds
   from the first build kernel to the last. */
typedef struct mgbvh_stats {
    double construction_time;
    uint32_t node_count;
    uint32_t leaf_node_count;
    uint32_t min_leaf_object_count;
    uint32_t max_leaf_object_count;
    double avg_leaf_object_count;
    double stddev_leaf_object_count;
    uint32_t total_object_count;
    uint32_t height;
    uint32_t max_depth;
    uint32_t median_splits;       /* forced median splits taken */
    uint32_t depth_capped_leaves; /* leaves made by depth == max_depth with len > 1 */
    uint32_t feasible;            /* the crate's feasibility flag */
    uint32_t kernel_launches;     /* builder kernels launched by this build */
    uint32_t levels;              /* level-synchronous passes over the largest nodes */
    /* device seconds per phase: [0] object records + root, [1] level passes,
       [2] subtrees of 33..1024 objects, [3] subtrees of <= 32 objects */
    double phase_seconds[4];
    uint32_t graph_replay;        /* 1: a batched build replayed its captured CUDA graph */
    uint32_t learned_splits;      /* nodes where a split-network proposal replaced the binned split */
} mgbvh_stats;

typedef struct mgbvh_ctx mgbvh_ctx;

/* Fills *s with the reference profile and max_depth 32
   (marigold/src/app/data/scene/mod.rs:28-29), MIN = MAX = 1, no bounds. */
MGBVH_API void mgbvh_default_settings(mgbvh_settings* s);

/* Device context: owns scratch buffers (grown on demand), a stream and events. */
MGBVH_API int mgbvh_create(int device, mgbvh_ctx** out_ctx);
MGBVH_API void mgbvh_destroy(mgbvh_ctx* ctx);
/* Run subsequent builds on a caller stream (cudaStream_t); NULL = own stream. */
MGBVH_API int mgbvh_set_stream(mgbvh_ctx* ctx, void* cuda_stream);
/* Text of the last error recorded on this context. */
MGBVH_API const char* mgbvh_last_error(const mgbvh_ctx* ctx);
MGBVH_API const char* mgbvh_status_string(int status);

/*
 * BLAS build over MeshTriangle / MeshVertex. Replaces
 * BoundingVolumeHierarchy::<MIN,MAX>::new(&mut triangles, &vertices, settings)
 * (bvh/src/lib.rs:698), as called at marigold/src/app/data/scene/model.rs:93.
 *
 * vertices: vertex_count records of vertex_stride_bytes bytes whose first 12
 *   bytes are the f32 position (MeshVertex is 32 bytes,
 *   mesh_interface/src/lib.rs:6-12).
 * triangles: triangle_count * 3 vertex indices (MeshTriangle).
 * out_nodes: node_capacity >= 2 * triangle_count - 1 is always enough.
 * out_lens: per-node object count (BvhNode::len), may be NULL.
 * out_perm: triangle_count entries; apply it to the triangle list to obtain
 *   the crate's in-place permutation.
 * out_stats: may be NULL.
 * All pointers are host pointers. Returns mgbvh_status.
 * When out_nodes (and out_lens, if given) are page-locked host memory
 * (cudaMallocHost, cudaHostAlloc, cudaHostRegister), node_capacity >=
 * 2 * triangle_count - 1 and leaves hold one object, finished chunks of the
 * node array are copied to the caller while the build's last kernels still
 * run; the result is the same as with pageable arrays, which are filled after
 * the build.
 */
MGBVH_API int mgbvh_build_indexed(mgbvh_ctx* ctx, const float* vertices, uint32_t vertex_stride_bytes,
                        uint32_t vertex_count, const uint32_t* triangles, uint32_t triangle_count,
                        const mgbvh_settings* settings, mgbvh_node* out_nodes,
                        uint32_t node_capacity, uint32_t* out_node_count, uint32_t* out_lens,
                        uint32_t* out_perm, mgbvh_stats* out_stats);

/*
 * Build over precomputed object AABBs (min xyz, max xyz per object, 24 bytes):
 * the AsBoundingVolume path, e.g. the TLAS over UploadedMesh built by
 * marigold/src/app/data/scene/geometry/mod.rs:175-199. Same outputs.
 */
MGBVH_API int mgbvh_build_aabbs(mgbvh_ctx* ctx, const float* aabbs, uint32_t count,
                      const mgbvh_settings* settings, mgbvh_node* out_nodes,
                      uint32_t node_capacity, uint32_t* out_node_count, uint32_t* out_lens,
                      uint32_t* out_perm, mgbvh_stats* out_stats);

/* Device-pointer forms of the two builds: every array argument is device
   memory; out_node_count and out_stats stay host pointers. The call returns
   after the build has finished on the context's stream. */
MGBVH_API int mgbvh_build_indexed_dev(mgbvh_ctx* ctx, const float* d_vertices, uint32_t vertex_stride_bytes,
                            uint32_t vertex_count, const uint32_t* d_triangles,
                            uint32_t triangle_count, const mgbvh_settings* settings,
                            mgbvh_node* d_out_nodes, uint32_t node_capacity,
                            uint32_t* out_node_count, uint32_t* d_out_lens, uint32_t* d_out_perm,
                            mgbvh_stats* out_stats);
MGBVH_API int mgbvh_build_aabbs_dev(mgbvh_ctx* ctx, const float* d_aabbs, uint32_t count,
                          const mgbvh_settings* settings, mgbvh_node* d_out_nodes,
                          uint32_t node_capacity, uint32_t* out_node_count, uint32_t* d_out_lens,
                          uint32_t* d_out_perm, mgbvh_stats* out_stats);

/*
 * Batched build: one BVH per mesh, every mesh in one pass of the pipeline.
 * The BLAS loop of marigold/src/app/data/scene/model.rs:77-95 (one
 * BoundingVolumeHierarchy::new per mesh, rayon across meshes) plus the TLAS
 * of marigold/src/app/data/scene/geometry/mod.rs:175-199 become one call:
 * give the TLAS as one more mesh whose objects are the instance AABBs.
 *
 * Each mesh's result is exactly what mgbvh_build_indexed / _aabbs returns for
 * it alone: its nodes sit at d_out_nodes[out_node_offsets[m] ..
 * out_node_offsets[m+1]) with child links relative to that range (as the
 * crate's per-mesh node arrays), and its permutation at d_out_perm[first ..
 * first + count) with first = the sum of the earlier meshes' counts.
 * node_capacity >= sum over meshes of (2 count - 1) is always enough.
 * All array pointers are device pointers; `meshes` and out_node_offsets
 * (mesh_count + 1 entries) are host arrays. The settings' bounds field is
 * ignored (each mesh carries its own).
 */
typedef struct mgbvh_mesh_desc {
    const float* vertices;      /* device; NULL when the objects are AABBs */
    uint32_t vertex_stride_bytes;
    uint32_t vertex_count;
    const uint32_t* triangles;  /* device, count x 3 (when vertices != NULL) */
    const float* aabbs;         /* device, count x 6 (when vertices == NULL) */
    uint32_t count;             /* objects of this mesh */
    uint32_t has_bounds;        /* BvhSettings::bounds is Some(..) for this mesh */
    float bounds[6];
} mgbvh_mesh_desc;

MGBVH_API int mgbvh_build_batch_dev(mgbvh_ctx* ctx, const mgbvh_mesh_desc* meshes,
                                    uint32_t mesh_count, const mgbvh_settings* settings,
                                    mgbvh_node* d_out_nodes, uint32_t node_capacity,
                                    uint32_t* d_out_lens, uint32_t* d_out_perm,
                                    uint32_t* out_node_offsets, mgbvh_stats* out_stats);

/* Batched builds on this context capture their launch sequence in a CUDA
   graph and replay it when the same mesh set (pointers, counts, settings,
   outputs, stream) is built again; a tree deeper than the captured one falls
   back to a regular build. Off by default. */
MGBVH_API int mgbvh_set_graph_capture(mgbvh_ctx* ctx, int enable);

/* Speed knob of a context, no effect on the trees: nodes with more than
   medium_max objects (33..1024, default 1024) go through the level passes,
   smaller ones to the per-subtree kernels. */
MGBVH_API int mgbvh_set_tuning(mgbvh_ctx* ctx, uint32_t medium_max);

/* How mgbvh_build_batch_dev builds (no counterpart in the reference, whose
   marigold/src/app/data/scene/model.rs:77-95 builds one BLAS per rayon
   worker and then the TLAS; the trees are the same either way):
     MGBVH_BATCH_LEVELS  level passes over every mesh's nodes above
                         medium_max, then one launch for the subtrees of
                         33..medium_max objects and one for those of <= 32
                         (the default);
     MGBVH_BATCH_QUEUE   one persistent launch: resident CTAs take node
                         tasks of every mesh and the TLAS from device-side
                         queues (one CTA splits a node above medium_max or
                         builds a subtree of 33..medium_max objects; its
                         warps build subtrees of <= 32) and push the
                         children. Plain builds of meshes up to 4,194,304
                         objects; others take the level passes. Forced medians
                         of nodes above medium_max run after the launch.
   Every wait of the persistent launch is bounded (2 s by default): when one
   runs out the launch ends and the build returns MGBVH_ERR_TIMEOUT. */
#define MGBVH_BATCH_LEVELS 0
#define MGBVH_BATCH_QUEUE 1
MGBVH_API int mgbvh_set_batch_mode(mgbvh_ctx* ctx, int mode);
/* The persistent launch's wait bound in microseconds (0: 2 s), and, for
   tests of that bound, a number of tasks counted as pending that never
   arrive (0 in normal use): with held_tasks > 0 every wait runs out and the
   build returns MGBVH_ERR_TIMEOUT. */
MGBVH_API int mgbvh_set_queue_limits(mgbvh_ctx* ctx, uint32_t wait_microseconds, uint32_t held_tasks);
/* Launch shapes of a context, speed only (the trees do not change): threads
   per CTA of the kernel that builds subtrees of <= 32 objects, one warp each
   (64, 128 or 256; 0: 256), and persistent CTAs per SM of the
   MGBVH_BATCH_QUEUE launch (0: as many as fit). The autotuner
   (marigold_b200/autotune.py) picks them per workload. */
MGBVH_API int mgbvh_set_launch_shape(mgbvh_ctx* ctx, uint32_t small_threads, uint32_t queue_ctas_per_sm);
/* Occupancy of the kernel that builds subtrees of <= 32 objects, speed only
   (the trees do not change): the resident warps per SM its register budget
   allows, 24 (80 registers a thread; 0 selects it) or 16 (126 registers,
   fewer spills); any other value gives MGBVH_ERR_UNSUPPORTED. The autotuner
   picks it per workload. */
MGBVH_API int mgbvh_set_small_occupancy(mgbvh_ctx* ctx, uint32_t warps_per_sm);

/* World AABBs of instances for the TLAS, computed on the GPU as marigold's
   scene upload computes them on the host (marigold/src/app/data/scene/
   model.rs:191-234): the 8 corners of each instance's mesh bounds through its
   column-major 4x4 f32 transform (glam's Mat4 * Vec4 order), min/max over the
   corners. d_mesh_bounds: mesh_count x 6 floats (min xyz, max xyz);
   d_instance_mesh: instance_count mesh indices; d_transforms: instance_count x
   16 floats; d_out_aabbs: instance_count x 6 floats, the input of
   mgbvh_build_aabbs_dev or of a batched build's TLAS. Runs on the context's
   stream and returns when done; an index >= mesh_count gives
   MGBVH_ERR_INVALID_ARG. The uploaded record's inverse transform is not
   computed here. */
MGBVH_API int mgbvh_instance_aabbs_dev(mgbvh_ctx* ctx, const float* d_mesh_bounds, uint32_t mesh_count,
                                       const uint32_t* d_instance_mesh, const float* d_transforms,
                                       uint32_t instance_count, float* d_out_aabbs);

/*
 * Allocation-free build over device-resident AABBs. This entry point has no
 * counterpart in the reference. It exists for callers that must not allocate
 * while they build: a render loop that rebuilds its TLAS every frame (as
 * marigold does over its instances) cannot afford cudaMalloc/cudaFree there,
 * because those calls can synchronize the whole device and stall the frame,
 * and a host engine that hands all device memory out through its own pool
 * may not allocate behind its back. mgbvh_build_aabbs_dev needs an mgbvh_ctx,
 * whose creation and growth allocate; this call needs no context.
 *
 * Limits: count <= MGBVH_NOALLOC_MAX_OBJECTS (1024), else
 * MGBVH_ERR_TOO_LARGE. Scratch is one fixed array inside the library (about
 * 140 KB of device memory on every device that loads the library, held until
 * the process exits), shared by all calls: calls whose work overlaps on the
 * GPU (several host threads, or several streams) race on it and must be
 * serialized by the caller. Every call sets up on the current device: it
 * looks up the array's device address there (cudaGetSymbolAddress, which
 * allocates nothing) and sets a kernel attribute; nothing is cached between
 * calls, so a call after a device reset uses the new context's array. The
 * first call on a device also loads the library's device code there (CUDA
 * loads modules lazily), so make that first call before any stream capture.
 *
 * Same tree, permutation and status codes as mgbvh_build_aabbs_dev.
 * d_aabbs, d_out_nodes, d_out_lens (nullable) and d_out_perm are device
 * pointers on the current device; out_node_count is a host pointer. Runs on
 * cuda_stream (cudaStream_t, NULL = legacy default stream) and returns after
 * the build has finished. Calls no allocating routine of CUDA or any library.
 */
MGBVH_API int mgbvh_build_aabbs_noalloc(const float* d_aabbs, uint32_t count,
                                        const mgbvh_settings* settings, mgbvh_node* d_out_nodes,
                                        uint32_t node_capacity, uint32_t* out_node_count,
                                        uint32_t* d_out_lens, uint32_t* d_out_perm,
                                        void* cuda_stream);

/*
 * Closest-hit traversal of a built BVH over triangles, restating the BLAS
 * traversal math of marigold/assets/shaders/slang/lib/scene.slang:19-89
 * (Moller-Trumbore, |det| < 1e-6 and t < 1e-6 reject), :143-220 (stack
 * traversal, nearer child first) and :296-310 (slab test), as CUDA over device
 * buffers (the shader itself needs a graphics stack). One mgbvh_tracer per
 * calling thread.
 *
 * Rays: n_rays records of 8 floats (origin xyz, unused, direction xyz,
 * unused). Results: hit distance in ray units (-1 for a miss) and the
 * original triangle index (0xFFFFFFFF for a miss); equal distances resolve to
 * the lowest triangle index. out_counts (host, nullable) receives the
 * shader's traversal counters summed over all rays: nodes visited, box tests,
 * triangle tests (scene.slang:108, 121, 208).
 */
typedef struct mgbvh_tracer mgbvh_tracer;
MGBVH_API int mgbvh_tracer_create(int device, mgbvh_tracer** out);
MGBVH_API void mgbvh_tracer_destroy(mgbvh_tracer* tracer);
/* Binds a built BLAS: device nodes (and lens for leaves of several objects,
   NULL = one object per leaf), the vertices/triangles it was built from and
   the build's permutation. Gathers the triangles into leaf order; keeps the
   node/len pointers, which must stay valid while tracing. */
MGBVH_API int mgbvh_tracer_set_blas_dev(mgbvh_tracer* tracer, const mgbvh_node* d_nodes,
                                        uint32_t node_count, const uint32_t* d_lens,
                                        const float* d_vertices, uint32_t vertex_stride_bytes,
                                        uint32_t vertex_count, const uint32_t* d_triangles,
                                        const uint32_t* d_perm, uint32_t triangle_count,
                                        void* cuda_stream);
/* Closest hit of every ray through the BVH. The call first sorts the rays
   (by origin cell of the root box, then direction bin) and traces them in
   that order, so that rays that start near one another in similar directions
   share warps; every ray's hit is still written at its own index, and the
   order changes no result. The sort buffers (about 16 bytes per ray) are
   kept by the tracer and grown on a call with more rays than before.
   out_seconds (host, nullable): device time of the sort and the traversal. */
MGBVH_API int mgbvh_trace_closest_dev(mgbvh_tracer* tracer, const float* d_rays, uint32_t n_rays,
                                      float* d_hit_t, uint32_t* d_hit_prim, uint64_t* out_counts,
                                      double* out_seconds, void* cuda_stream);
/* Wide BVH (no counterpart in the reference, which names compressed wide
   BVHs as its next step): collapses the bound binary tree into an 8-wide BVH
   whose child boxes are quantized to 8-bit steps on a per-node power-of-two
   grid, widened outward so that every stored box contains its exact box.
   112-byte nodes: origin xyz (f32), per-axis step exponents (u8, step =
   2^(e - 127)), child count (u8), child box steps lo x/y/z[8], hi x/y/z[8]
   (u8), child refs[8] (u32: wide node index, or first triangle | 0x80000000
   for a leaf), leaf triangle counts[8] (u8), 8 bytes of padding; node 0 is
   the root. Runs on cuda_stream and returns when done. */
MGBVH_API int mgbvh_tracer_build_wide(mgbvh_tracer* tracer, void* cuda_stream, uint32_t* out_wide_count);
/* The wide nodes of the last mgbvh_tracer_build_wide (device pointer, owned by the tracer). */
MGBVH_API int mgbvh_tracer_wide_nodes(mgbvh_tracer* tracer, const void** out_d_wide_nodes,
                                      uint32_t* out_wide_count);
/* Closest hit of every ray through the wide BVH, rays in the same sorted
   order as mgbvh_trace_closest_dev: same results as
   mgbvh_trace_closest_dev (same triangle test and tie rule; conservative
   boxes). out_counts: wide nodes visited, child boxes tested, triangle tests. */
MGBVH_API int mgbvh_trace_closest_wide_dev(mgbvh_tracer* tracer, const float* d_rays, uint32_t n_rays,
                                           float* d_hit_t, uint32_t* d_hit_prim, uint64_t* out_counts,
                                           double* out_seconds, void* cuda_stream);
/* Closest hit of every ray against every triangle of the bound BLAS, with
   the same triangle test: the check for mgbvh_trace_closest_dev. */
MGBVH_API int mgbvh_trace_bruteforce_dev(mgbvh_tracer* tracer, const float* d_rays,
                                         uint32_t n_rays, float* d_hit_t, uint32_t* d_hit_prim,
                                         void* cuda_stream);

/*
 * Two-level scenes: the TLAS over instances, each instance a mesh with its
 * own BLAS, walked as marigold's scene shader walks them
 * (marigold/assets/shaders/slang/lib/scene.slang:91-141 raytraceTlas,
 * :143-220 raytraceBlas). The records are the ones marigold uploads for the
 * shader (marigold/src/app/data/scene/model.rs:167-234 and
 * geometry/mod.rs:175-199; the shader's Mesh: inverseTransform, blasRoot,
 * vertexOffset, triangleOffset).
 */
typedef struct mgbvh_scene_mesh {
    uint32_t blas_root;       /* its BLAS's root in the BLAS node array; child links are relative to it */
    uint32_t triangle_offset; /* its first triangle in the scene triangle array */
    uint32_t triangle_count;
    uint32_t vertex_offset;   /* added to its triangles' vertex indices */
} mgbvh_scene_mesh;

typedef struct mgbvh_scene_instance {
    float inverse_transform[16]; /* column-major, world space -> mesh space */
    uint32_t mesh;               /* index into the mesh table */
    uint32_t pad[3];
} mgbvh_scene_instance;

/* Binds a scene (device pointers, which must stay valid while tracing; the
   mesh table is copied). The TLAS's leaves index d_instances, which are in
   the TLAS build's permuted order (as the crate leaves the instance list);
   each mesh's BLAS leaves index its triangles, which sit in the scene
   triangle array in that BLAS build's permuted order, as vertex index
   triples relative to the mesh's vertex_offset. Lens arrays (NULL = one
   object per leaf) are node-aligned with their node arrays. Gathers the
   triangles with their vertices. */
MGBVH_API int mgbvh_tracer_set_scene_dev(mgbvh_tracer* tracer, const mgbvh_node* d_tlas_nodes,
                                         uint32_t tlas_node_count, const uint32_t* d_tlas_lens,
                                         const mgbvh_scene_instance* d_instances, uint32_t instance_count,
                                         const mgbvh_scene_mesh* d_meshes, uint32_t mesh_count,
                                         const mgbvh_node* d_blas_nodes, uint32_t blas_node_count,
                                         const uint32_t* d_blas_lens, const float* d_vertices,
                                         uint32_t vertex_stride_bytes, uint32_t vertex_count,
                                         const uint32_t* d_triangles, uint32_t triangle_count,
                                         void* cuda_stream);
/* Closest hit of every world-space ray through the scene: the TLAS with the
   world ray, each reached instance's BLAS with the ray moved into mesh space
   by its inverse transform. Hit distances are the world ray's parameter in
   every instance (the shader's rescaling by the mesh-space direction length,
   scene.slang:168-169, is wrong for scaled instances and is not copied).
   Results per ray: distance (-1 for a miss), the instance (position in
   d_instances) and the triangle (position in the scene triangle array), both
   0xFFFFFFFF for a miss; equal distances resolve to the lowest (instance,
   triangle). Rays are sorted by origin cell of the TLAS root box and
   direction bin first, as in mgbvh_trace_closest_dev. out_counts: nodes
   visited (both levels), box tests, triangle tests. */
MGBVH_API int mgbvh_trace_scene_dev(mgbvh_tracer* tracer, const float* d_rays, uint32_t n_rays,
                                    float* d_hit_t, uint32_t* d_hit_instance, uint32_t* d_hit_triangle,
                                    uint64_t* out_counts, double* out_seconds, void* cuda_stream);
/* The check for mgbvh_trace_scene_dev: every ray against every triangle of
   every instance, in mesh space, same test and tie rule. cull_by_mesh_bounds
   != 0 skips instances whose mesh-space ray misses the mesh's BLAS root box
   grown by a relative 1e-4 (for large scenes). */
MGBVH_API int mgbvh_trace_scene_bruteforce_dev(mgbvh_tracer* tracer, const float* d_rays, uint32_t n_rays,
                                               float* d_hit_t, uint32_t* d_hit_instance,
                                               uint32_t* d_hit_triangle, int cull_by_mesh_bounds,
                                               void* cuda_stream);

/*
 * Learned split proposer (no counterpart in the reference). A small MLP,
 * 24 -> 64 -> 64 -> 49 with GELU, BF16 parameters and FP32 accumulation,
 * proposes two (axis, 1/16 position bucket) candidates at every binned node
 * of 33 or more objects; the builder scores 16 thresholds inside each
 * candidate exactly with the reference's cost formula and keeps the plain
 * split unless one costs strictly less (mgbvh_set_split_proposer). Parameters:
 * MGBVH_MLP_PARAMS values, W1[64x24] b1[64] W2[64x64] b2[64] W3[49x64] b3[49].
 * Training on the GPU: the caller zeroes d_grad and d_loss, calls
 * mgbvh_mlp_train_step_dev over a batch (features B x 24 f32, labels B u32 =
 * axis * 16 + position bucket or 0xFFFFFFFF, gains B f32 in {0, 1}), which
 * adds the gradient of the mean loss (softmax cross-entropy of the 48
 * position logits + binary cross-entropy of the refine logit) and the summed
 * losses [ce, bce]; then mgbvh_mlp_adam_dev updates the FP32 master weights
 * and rewrites the BF16 copy. All pointers are device pointers.
 */
#define MGBVH_MLP_PARAMS 8945
MGBVH_API int mgbvh_mlp_train_step_dev(const float* d_features, const uint32_t* d_labels,
                                       const float* d_gains, uint32_t batch,
                                       const void* d_weights_bf16, float* d_grad, float* d_loss,
                                       void* cuda_stream);
MGBVH_API int mgbvh_mlp_forward_dev(const float* d_features, uint32_t batch,
                                    const void* d_weights_bf16, float* d_out, void* cuda_stream);
MGBVH_API int mgbvh_mlp_adam_dev(float* d_master, void* d_weights_bf16, const float* d_grad,
                                 float* d_m, float* d_v, uint32_t step, float lr, float beta1,
                                 float beta2, float eps, void* cuda_stream);

/* Builds on this context use the learned split proposer at every binned node
   of 33 or more objects (d_weights_bf16: MGBVH_MLP_PARAMS BF16 values on the
   device, copied by this call, which returns once the copy is done; NULL
   turns the proposer off). gate != 0: only where the network's refine logit
   is positive. The trees then differ from the reference's (the plain split
   is replaced only by an exactly cheaper one). No reference counterpart. */
MGBVH_API int mgbvh_set_split_proposer(mgbvh_ctx* ctx, const void* d_weights_bf16, int gate);
/* The learned form's cost knobs (no reference counterpart): with the gate on,
   proposals are scored only where the refine logit exceeds refine_threshold
   (default 0); nodes of fewer than min_objects objects (default 0) take the
   plain split without running the network. Higher values build faster and
   close less of the gap to the full sweep. */
MGBVH_API int mgbvh_set_proposer_gate(mgbvh_ctx* ctx, float refine_threshold, uint32_t min_objects);
/* Builds on this context also write one training sample (30 floats: 24
   features, label bits, gain, n, plain cost, full-sweep cost, node start) per
   binned node of 33..8192 objects to d_samples (device, capacity samples) and
   count them in *d_count (device; the caller zeroes it). The label is the
   exact full sweep's optimum (every centroid a threshold on every axis),
   computed by the builder. NULL turns it off. */
MGBVH_API int mgbvh_set_sample_output(mgbvh_ctx* ctx, float* d_samples, uint32_t capacity,
                                      uint32_t* d_count);

/*
 * AsGpuBytes for BvhNode (bvh/src/lib.rs:157-212), host side: 8 u32 words per
 * node. For MAX_LEAF_OBJECTS == 1 this copies the node. For larger MAX the
 * last word packs len into the top ilog2(MAX.next_power_of_two()) bits and
 * keeps child_node & !len_mask in the rest, exactly as the crate writes it.
 * Returns MGBVH_ERR_ASSERT where the crate's assert (leaf len < 2^len_bits)
 * would panic.
 */
MGBVH_API int mgbvh_encode_gpu_bytes(const mgbvh_node* nodes, const uint32_t* lens, uint32_t count,
                           uint32_t max_leaf_objects, uint32_t* out_words);

/* Total SAH cost of a built tree, normalised by the root's surface area, with
   the crate's DEPTH_COST = 1 and OBJECT_COST = 8 (bvh/src/lib.rs:217-218):
   sum over inner nodes of SA(n)/SA(root) + sum over leaves of
   8 * len * SA(n)/SA(root). Host computation in f64. */
MGBVH_API double mgbvh_sah_cost(const mgbvh_node* nodes, const uint32_t* lens, uint32_t count);

#ifdef __cplusplus
}
#endif

#endif /* MGBVH_H */
