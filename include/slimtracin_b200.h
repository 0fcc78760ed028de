/*
 * slimtracin_b200.h — C ABI of libslimtracin_b200, the B200 (sm_100a) tracing path of SlimTracin.
 *
 * The library replaces the reference's per-frame render and its BVH updates:
 *   renderScene        render/raytracer.h:302   -> st_render_scene / st_render_ex
 *   updateSceneBVH     acceleration_structures/builder_top_down.h:366 -> st_update_scene_bvh
 *   updateMeshBVH      acceleration_structures/builder_top_down.h:272 -> st_update_mesh_bvh
 *   allocateDeviceScene, upload*   core/init.h:36-126 -> st_allocate_device_scene, st_upload_*
 *
 * Conventions (they differ from the reference on purpose, see each function):
 *   - every entry point returns an int status, ST_OK == 0; nothing calls exit();
 *   - the library owns all device memory; host structs are read-only inputs unless a function says
 *     it writes them; output buffers are caller-allocated;
 *   - one st_ctx is used by one host thread at a time.
 */
#ifndef SLIMTRACIN_B200_H
#define SLIMTRACIN_B200_H

#include "slimtracin_types.h"
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define ST_API __attribute__((visibility("default")))
#else
#define ST_API
#endif

typedef struct st_ctx st_ctx;

enum st_status {
    ST_OK = 0,
    ST_ERR_INVALID_ARG = 1,     /* a null pointer, a bad slot, a size outside the stated limits */
    ST_ERR_NO_DEVICE = 2,       /* no CUDA device, or the device is not sm_100 */
    ST_ERR_CUDA = 3,            /* a CUDA runtime call failed; st_last_cuda_error() has the text */
    ST_ERR_OUT_OF_MEMORY = 4,   /* cudaMalloc failed */
    ST_ERR_BUDGET = 5,          /* the request would exceed the context's device-memory budget */
    ST_ERR_STACK_OVERFLOW = 6,  /* a traversal stack overflowed (the kernel stops that ray) */
    ST_ERR_TIMEOUT = 7,         /* a bounded device-side wait gave up */
    ST_ERR_NOT_RESIDENT = 8,    /* the scene slot holds no uploaded scene */
    ST_ERR_BAD_SCENE = 9,       /* the scene data is inconsistent (e.g. a leaf id out of range) */
    ST_ERR_QUEUE_FULL = 10,     /* the serving queue has no free slot */
    ST_ERR_NOT_READY = 11,      /* st_poll: the request is still running */
    ST_ERR_CANCELLED = 12,      /* st_poll: the request was cancelled before it ran */
    ST_ERR_IO = 13              /* a file could not be opened, or was shorter than its header says */
};

/* TLAS/BLAS build modes for st_update_scene_bvh / st_update_mesh_bvh. */
enum st_bvh_mode {
    ST_BVH_LBVH30 = 1,      /* 30-bit Morton LBVH: device radix sort, Karras topology, leaf collapse */
    ST_BVH_BINNED_SAH = 2,  /* breadth-first binned SAH (32 bins) on the device */
    ST_BVH_REFIT = 3,       /* keep the resident topology, recompute every AABB bottom-up */
    ST_BVH_REF_SAH = 4      /* the reference's own full-sweep SAH (buildBVH, builder_top_down.h:204), node
                               for node; for TLASes, whose topology decides which occluder a shadow ray
                               meets first (st_update_scene_bvh, st_build_bvh; not for BLASes) */
};

typedef struct st_config {
    int device;                 /* CUDA device ordinal */
    uint64_t memory_budget;     /* bytes of device memory the context may hold; 0 -> 120 GB */
    int max_scenes;             /* resident scene slots; 0 -> 16 */
    uint32_t flags;             /* reserved, 0 */
} st_config;

/* Outputs and knobs of one render, beyond what the reference's Viewport carries.
 * All output pointers are optional.  When `device_outputs` is non-zero they are device pointers and
 * no host copy happens inside the call. */
typedef struct st_render_options {
    void *stream;               /* cudaStream_t to launch on; NULL -> the context's stream */
    int device_outputs;         /* 1: the out_* pointers below are device pointers */
    FloatPixel *out_float;      /* (W+1)x(H+1) QCAA grid; NULL -> viewport->frame_buffer->float_pixels */
    Pixel *out_u8;              /* W x H resolved BGRA; NULL -> viewport->frame_buffer->pixels */
    uint32_t *out_prim_id;      /* (W+1)x(H+1) primary-hit primitive id, 0xFFFFFFFF on a miss */
    int skip_float_copy;        /* 1: do not copy the float grid to the host (u8 only) */
    int count_work;             /* 1: fill `counters` (a slower instrumented kernel) */
    uint64_t counters[16];      /* out: see enum st_counter */
    float trace_ms;             /* out: CUDA-event time of the trace kernel on the launch stream */
    float total_ms;             /* out: CUDA-event time of the whole render on the launch stream */
    int overlays;               /* ST_OVERLAY_* bits: debug overlays drawn over the traced grid, before
                                   the resolve */
} st_render_options;

/* The debug overlays of render/raytracer.h:46 (drawBVH: TLAS node boxes, leaf primitives' boxes,
 * mesh instances' BLAS nodes of depth <= 5) and render/SSB.h:175 (drawSSB: each visible primitive's
 * screen-space bounds), drawn on the device in the reference's order with its anti-aliased line
 * rasteriser (shapes/line.h:46) and blending (setPixel, core/types.h:422), using
 * viewport->projection_matrix (set by beginDrawing) and the clipping distances of
 * viewport->settings.  drawBVH walks every TLAS node (the reference's u8 node counter never
 * terminates at 256 nodes or more). */
enum st_overlay {
    ST_OVERLAY_BVH = 1,
    ST_OVERLAY_SSB = 2
};

enum st_counter {
    ST_CNT_PRIMARY_RAYS = 0,
    ST_CNT_SHADOW_RAYS = 1,     /* point-light shadow rays (any-hit TLAS walks) */
    ST_CNT_BOUNCE_RAYS = 2,     /* reflection/refraction rays (closest-hit TLAS walks) */
    ST_CNT_AABB_TESTS = 3,      /* TLAS + BLAS node AABB tests */
    ST_CNT_TRIANGLE_TESTS = 4,
    ST_CNT_PRIMITIVE_TESTS = 5, /* implicit-primitive intersection tests */
    ST_CNT_LEAF_ID_READS = 6,
    ST_CNT_SHADED_HITS = 7,
    ST_CNT_TEXEL_FETCHES = 8,
    ST_CNT_MESH_ENTRIES = 9,    /* BLAS traversals started */
    ST_CNT_TEXEL_MIP_FETCHES = 10, /* the texel fetches of ST_CNT_TEXEL_FETCHES from a mip level above 0 */
    ST_CNT_COUNT = 11
};

/* ---- context ---------------------------------------------------------------------------------- */
ST_API int  st_init(st_ctx **ctx, const st_config *cfg);
ST_API void st_shutdown(st_ctx *ctx);
ST_API const char *st_strerror(int status);
ST_API const char *st_last_cuda_error(st_ctx *ctx);
ST_API void *st_get_stream(st_ctx *ctx);                       /* the context's cudaStream_t */
ST_API uint64_t st_device_bytes_in_use(st_ctx *ctx);
/* Size of a contract struct ("Primitive") or offset of a field ("Primitive.rotation") as this
 * library was compiled; -1 if the name is not in include/slimtracin_layout.h. */
ST_API long st_layout_query(const char *name);

/* ---- residency: core/init.h:36-126 -------------------------------------------------------------- */
/* allocateDeviceScene (core/init.h:36): reserve device arenas for `scene` in `slot`. */
ST_API int st_allocate_device_scene(st_ctx *ctx, int slot, const Scene *scene);
/* uploadScene (core/init.h:85): lights, primitives, materials, textures (+ mip chains). */
ST_API int st_upload_scene(st_ctx *ctx, int slot, const Scene *scene);
/* uploadPrimitives (core/init.h:74). */
ST_API int st_upload_primitives(st_ctx *ctx, int slot, const Scene *scene);
/* uploadMaterials (core/init.h:77). */
ST_API int st_upload_materials(st_ctx *ctx, int slot, const Scene *scene);
/* uploadLights (core/init.h:80). */
ST_API int st_upload_lights(st_ctx *ctx, int slot, const Scene *scene);
/* uploadSceneBVH (core/init.h:106): the host-built TLAS (scene->bvh) as-is. */
ST_API int st_upload_scene_bvh(st_ctx *ctx, int slot, const Scene *scene);
/* uploadMeshBVHs (core/init.h:111): every mesh's BLAS nodes and BVH-ordered Triangles as-is. */
ST_API int st_upload_mesh_bvhs(st_ctx *ctx, int slot, const Scene *scene);
/* Primitives whose transform changed since the last upload: primitives[k] replaces primitive
 * ids[k]; the ids must be distinct and below the scene's primitive count (else ST_ERR_INVALID_ARG,
 * nothing changed).  Only those records cross to the device, in one copy; the TLAS is then stale
 * until st_update_scene_bvh (the reference re-uploads the whole array, core/init.h:74). */
ST_API int st_update_primitives(st_ctx *ctx, int slot, const Primitive *primitives,
                         const uint32_t *ids, uint32_t count);
ST_API int st_free_scene(st_ctx *ctx, int slot);

/* ---- BVH builds: render/acceleration_structures/builder_top_down.h ---------------------------- */
/* updateSceneBVH (builder_top_down.h:366): build the TLAS of the resident primitives on the device.
 * mode: ST_BVH_LBVH30 | ST_BVH_BINNED_SAH | ST_BVH_REFIT.  When scene->bvh.nodes and
 * scene->bvh.leaf_ids are non-null the result is also copied there (node_count, height set). */
ST_API int st_update_scene_bvh(st_ctx *ctx, int slot, Scene *scene, int mode);
/* updateMeshBVH (builder_top_down.h:272): build the BLAS of `mesh` on the device and write the
 * reference's outputs into the caller's arrays: mesh->bvh.nodes (capacity 2*triangle_count),
 * mesh->bvh.leaf_ids, mesh->bvh.node_count/height and the BVH-ordered mesh->triangles. */
ST_API int st_update_mesh_bvh(st_ctx *ctx, Mesh *mesh, int mode);

/* The device builders of st_update_scene_bvh (mode ST_BVH_LBVH30 or ST_BVH_BINNED_SAH) over any `n`
 * caller boxes (host array, 6 floats each: min.xyz, max.xyz) with leaves of at most `max_leaf`
 * items.  Outputs (host): codes[n] the Morton code of each item (LBVH30 only, optional),
 * order[n] the items in leaf order, nodes[2n] in the reference's BVHNode layout, info =
 * {node_count, height}.  No reference counterpart: it exposes the builders behind updateSceneBVH's
 * replacement to callers with their own boxes. */
ST_API int st_build_bvh(st_ctx *ctx, int mode, const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *codes,
                        uint32_t *order, BVHNode *nodes, uint32_t info[2]);

/* Validate a BVH in the reference's layout the way the uploads do (st_upload_scene_bvh,
 * st_upload_mesh_bvhs), on the host, with no context: every children pair reached from the root
 * lies inside `nodes[node_count]` and is reached once, every leaf range lies inside `items`, and
 * both `height` and the depth the walk reaches leave room in the 64-entry traversal stacks (depth
 * + 2 <= 64).  ST_OK, ST_ERR_BAD_SCENE, or ST_ERR_INVALID_ARG for a null array.  No reference
 * counterpart: a host can check a loaded .mesh or .scene BVH before it uploads it. */
ST_API int st_validate_bvh(const BVHNode *nodes, uint32_t node_count, uint32_t items, uint32_t height);

/* ---- render: render/raytracer.h:302 ------------------------------------------------------------ */
/* renderScene (raytracer.h:302) + the QCAA resolve of drawViewportToWindowContent (viewport.h:12).
 * Renders the scene resident in `slot` from viewport->camera into viewport->frame_buffer:
 * float_pixels ((W+1)x(H+1), as renderScene leaves them after beginDrawing) and, when
 * frame_buffer->pixels is non-null, the resolved W x H BGRA pixels.  `scene` supplies the per-frame
 * values the reference passes by value to its kernel (counts, ambient light); the arrays come from
 * the device copy.  viewport->trace.depth is the bounce count.  Page-locked host buffers (pinned
 * or registered) are filled while the frame is traced: it is traced in column strips, and each
 * strip's float_pixels are copied and its pixels resolved into them as soon as the strip is done;
 * pageable ones receive a copy once the whole frame is done.  viewport->settings.show_BVH / show_SSB draw the drawBVH / drawSSB overlays
 * into the frame before the resolve (a host that binds renderScene here drops its own drawBVH and
 * drawSSB calls). */
ST_API int st_render_scene(st_ctx *ctx, int slot, const Scene *scene, Viewport *viewport);
/* st_render_scene with explicit outputs, stream, counters and timings. */
ST_API int st_render_ex(st_ctx *ctx, int slot, const Scene *scene, const Viewport *viewport,
                 st_render_options *options);

/* ---- batched views: many views of resident scenes in one call ------------------------------------ */
/* How a batch's views are launched (st_batch_options.launch_mode, st_serve_config.launch_mode). */
enum st_launch_mode {
    ST_LAUNCH_AUTOTUNED = -1,   /* st_render_batch only: timed per scene class and cached */
    ST_LAUNCH_PER_VIEW = 0,     /* one trace kernel per view, the views on concurrent streams */
    ST_LAUNCH_PERSISTENT = 1    /* one persistent kernel over a shared tile queue */
};

typedef struct st_view {
    int slot;                   /* resident scene */
    const Scene *scene;         /* per-frame values (ambient light); NULL -> the uploaded ones */
    const Viewport *viewport;   /* camera, projection plane (set by the caller), dims, mode, trace.depth */
    FloatPixel *out_float;      /* optional (W+1)x(H+1) grid, host or device per device_outputs */
    Pixel *out_u8;              /* optional W x H resolved BGRA */
} st_view;

typedef struct st_batch_options {
    void *stream;               /* cudaStream_t; NULL -> the context's stream */
    int device_outputs;         /* 1: out_* are device pointers */
    int tile_shape;             /* -1: autotuned; 0: 8x4, 1: 16x2, 2: 32x1, 3: 4x8 grid points per warp */
    int chunk;                  /* groups of four tiles a block takes per queue fetch (a tile per warp); 0: autotuned */
    int use_graph;              /* 1: launch through a CUDA graph: the batch's launches are captured and an
                                   instantiated graph of the same topology is updated in place */
    float batch_ms;             /* out: CUDA-event time of the batch on the launch stream */
    uint64_t rays;              /* out: primary rays traced */
    int tile_shape_used, chunk_used, graph_replayed;   /* out; graph_replayed: an existing graph was updated */
    int stack_placement;        /* -1: autotuned; 0: traversal stacks in local memory; 1: their first 16
                                   entries in shared memory (the traversal is the same either way) */
    int stack_placement_used;   /* out */
    int launch_mode;            /* st_launch_mode: ST_LAUNCH_AUTOTUNED (-1), ST_LAUNCH_PER_VIEW (0) or
                                   ST_LAUNCH_PERSISTENT (1); tile_shape, chunk and stack_placement apply to
                                   the persistent kernel */
    int launch_mode_used;       /* out (per view: tile_shape_used and stack_placement_used are -1) */
    int compaction_threshold;   /* persistent kernel, warp-vote ray compaction: at a bounce, a warp whose
                                   lanes still tracing number fewer than this parks their paths in a queue
                                   that a second persistent pass traces to the end (outputs unchanged);
                                   -1: autotuned, 0: off, 1..32 */
    int compaction_threshold_used;   /* out */
    uint64_t parked_rays;       /* out: paths parked by the compaction and traced by the second pass */
} st_batch_options;

/* Render `view_count` views (different sizes, scenes, render modes and bounce counts) in one call:
 * one persistent kernel over a shared tile queue, or one trace kernel per view on concurrent
 * streams (launch_mode; the views' set-up and resolves are one launch each per 64 views).  No
 * reference counterpart: the reference renders one viewport per renderScene call (raytracer.h:302);
 * each view's output equals st_render_ex's. */
ST_API int st_render_batch(st_ctx *ctx, const st_view *views, int view_count, st_batch_options *options);

/* LBVH30 over device-resident boxes with no allocation.  No counterpart in the reference.
 * Same inputs and outputs as st_build_bvh (ST_BVH_LBVH30), but every pointer is DEVICE memory:
 * aabbs (6 floats per item), codes (n, may be null), order (n), nodes (2n BVHNodes); info[2] is
 * host memory.  The scratch is a static device array sized for ST_NOALLOC_LBVH_MAX_ITEMS items
 * (about 4.8 MB, held by every GPU that loads the library until the process exits), so the call
 * makes no cudaMalloc/cudaFree and grows no pool: for hosts that must not allocate while other
 * streams are busy or whose budget is reserved up front.  n > ST_NOALLOC_LBVH_MAX_ITEMS returns
 * ST_ERR_INVALID_ARG before any work.  Every call looks up the array's device address
 * (cudaGetSymbolAddress); the first call on a device may also load the module, so make it once at
 * set-up, before any stream capture.  Calls on one device share the array: overlapping calls
 * (threads, streams or contexts of one process) race and must be serialised by the caller.
 * Returns after `stream` (null: the context's stream) has finished the build. */
#define ST_NOALLOC_LBVH_MAX_ITEMS 65536u
ST_API int st_build_lbvh_noalloc(st_ctx *ctx, const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *codes,
                                 uint32_t *order, BVHNode *nodes, uint32_t info[2], void *stream);

/* The object a click at pixel (x, y) of `viewport` selects, as manipulateSelection computes it
 * (viewport/manipulation.h:55-123): the picking ray of setRayFromCoords (shaders/common.h:170),
 * hitPrimitives over the resident primitives with the screen-space visibility cull at (x, y), then
 * the glow sphere of every light.  viewport->projection_plane must be current (beginDrawing or
 * setViewportProjectionPlane).  The host-side selection bookkeeping (pointers, offsets) stays with
 * the caller. */
typedef struct st_pick_result {
    int found;                  /* 1 when a primitive or a light was hit */
    int object_type;            /* PrimitiveType_* of the hit; PrimitiveType_Light for a light */
    uint32_t object_id;         /* primitive index, or light index */
    float position[3];          /* world-space hit position */
    float distance;             /* along the picking ray */
    float object_distance;      /* camera-space z of the hit (selection->object_distance) */
} st_pick_result;
ST_API int st_pick(st_ctx *ctx, int slot, const Scene *scene, const Viewport *viewport, int x, int y,
                   st_pick_result *result);

/* ---- serving: continuous batching of render requests ---------------------------------------------
 * A worker thread inside the library takes submitted requests in order, admits them while the
 * device-memory budget for in-flight frame/ray buffers allows, applies their transform updates,
 * refits (few moved primitives) or rebuilds (many) the TLAS of exactly the scenes that changed,
 * and launches each batch (one trace kernel per view on the batch's own streams, or the persistent
 * multi-view kernel) from one of `max_in_flight` streams, so requests that arrive while other
 * batches run are launched beside them.  An update to a scene
 * that batches in flight still read goes to a new copy of the scene's primitive and TLAS arrays
 * (a scene version; at most one per batch in flight, counted against the context's budget), so it
 * never waits for them.  A request never shares a batch with a request that changes its scene
 * after it, so every result equals the result of the same request rendered alone after the same
 * sequence of updates.
 * While serving, only st_submit / st_poll / st_wait / st_serve_stop may be called on the context
 * (from any one host thread); the scenes must already be resident.  No reference counterpart. */
typedef struct st_serve_config {
    int max_in_flight;          /* batches on the device at once; 0 -> 3 */
    int max_views_per_batch;    /* 0 -> 64 */
    uint64_t frame_budget;      /* device bytes for in-flight frame/ray buffers; 0 -> budget - resident scenes */
    int tile_shape, chunk;      /* -1 / 0: the autotuned choice for the scene class, else 8x4 and 1 */
    double refit_fraction;      /* primitives moved since the scene's last full TLAS build, as a fraction of
                                   all, below which the TLAS is refit, else rebuilt (LBVH30); 0 -> 0.25 */
    int launch_mode;            /* st_launch_mode: ST_LAUNCH_PER_VIEW (0) or ST_LAUNCH_PERSISTENT (1; tile_shape
                                   and chunk apply) */
} st_serve_config;

typedef struct st_request {
    st_view view;               /* host outputs; they must stay valid until the request completes */
    const Primitive *moved;     /* transform updates applied before this view renders (copied at submit) */
    const uint32_t *moved_ids;
    uint32_t moved_count;
    double arrival_time;        /* carried to the result; use st_clock() for the library's clock */
} st_request;

typedef struct st_result {
    int status;                 /* ST_OK, or the error that failed the request */
    double arrival_time, launch_time, completion_time;   /* st_clock() seconds */
    uint64_t rays;
    int batch_size;             /* requests in the batch that rendered it */
} st_result;

typedef uint64_t st_ticket;

ST_API int st_serve_start(st_ctx *ctx, const st_serve_config *config);
ST_API int st_submit(st_ctx *ctx, const st_request *request, st_ticket *ticket);
/* ST_OK with *result filled once the request has completed (the ticket is then released),
 * ST_ERR_NOT_READY before that, ST_ERR_INVALID_ARG for an unknown ticket. */
ST_API int st_poll(st_ctx *ctx, st_ticket ticket, st_result *result);
ST_API int st_wait(st_ctx *ctx, st_ticket ticket, st_result *result, double timeout_s);
/* Finish every submitted request, then stop the worker. */
ST_API int st_serve_stop(st_ctx *ctx);
/* The library's steady clock, in seconds. */
ST_API double st_clock(void);

/* ---- ingestion: textures and the reference's file formats ----------------------------------- */
/* loadTexture (bmp2texture.c:324) on the device: an 8-bit image (`components`, row-major RGB, or
 * RGBX when bit_count == 32) -> the reference's texture: wrap/mipmap flags, the mip chain (halving
 * while both sides exceed 4 when mipmap is set), each mip a (w+1)x(h+1) TexelQuad grid with the
 * reference's edge replication, byte-identical to the reference's baker.  `memory` (host,
 * st_texture_bytes bytes) receives the TextureMip table and the quads; texture->mips points into it.
 * width and height must be at least 2. */
ST_API uint64_t st_texture_bytes(uint16_t width, uint16_t height, int mipmap);
ST_API int st_bake_texture(st_ctx *ctx, const uint8_t *components, uint16_t width, uint16_t height, int bit_count,
                           int wrap, int mipmap, Texture *texture, void *memory, uint64_t memory_bytes);

/* .mesh files (scene/io.h:62-175): st_mesh_file_bytes = the host memory st_read_mesh_file needs
 * (getMeshMemorySize), or -1 when the header cannot be read; st_read_mesh_file = loadMeshFromFile
 * into `memory` (mesh's arrays point into it; bvh.nodes has room for 2 * triangle_count nodes);
 * st_write_mesh_file = saveMeshToFile. */
ST_API int64_t st_mesh_file_bytes(const char *path);
ST_API int st_read_mesh_file(const char *path, Mesh *mesh, void *memory, uint64_t memory_bytes);
ST_API int st_write_mesh_file(const char *path, const Mesh *mesh);
/* .texture files (scene/io.h:6-59; written by bmp2texture.c:367-385): sizes from the file's own mip
 * table, so a file whose mip count differs from getTextureMemorySize's estimate still fits. */
ST_API int64_t st_texture_file_bytes(const char *path);
ST_API int st_read_texture_file(const char *path, Texture *texture, void *memory, uint64_t memory_bytes);
ST_API int st_write_texture_file(const char *path, const Texture *texture);
/* .scene files (scene/io.h:178-213): SceneSettings, cameras, primitives.  Reading takes the counts
 * from the file, refuses (ST_ERR_BUDGET) more cameras or primitives than the capacities of
 * scene->cameras / scene->primitives, keeps the caller's file-name strings (the file holds the
 * writer's pointers) and re-points each camera's direction pointers at its own matrix. */
ST_API int st_read_scene_file(const char *path, Scene *scene, uint32_t camera_capacity, uint32_t primitive_capacity);
ST_API int st_write_scene_file(const char *path, const Scene *scene);
/* obj2mesh (obj2mesh.c:25): a Wavefront OBJ with faces "f v/t/n v/t/n v/t/n" -> a Mesh ready for
 * st_write_mesh_file or upload: positions, uvs, normals and their 1-based face indices read as the
 * reference reads them (the same sscanf formats, lines of at most 1023 characters), winding
 * optionally inverted, the AABB over the vertices and the origin with the vertices centred on its
 * middle, the unique edges in first-appearance order (found on the device), and the BLAS with the
 * Triangle records built on the device by `mode` (ST_BVH_LBVH30 or ST_BVH_BINNED_SAH; the reference
 * uses its full-sweep SAH).  Arrays are carved from `memory` (st_obj_mesh_bytes bytes, -1 when the
 * file cannot be read).  Other face layouts give ST_ERR_BAD_SCENE (the reference's updateMeshBVH
 * reads vertex normals for every triangle). */
ST_API int64_t st_obj_mesh_bytes(const char *obj_path);
ST_API int st_obj_to_mesh(st_ctx *ctx, const char *obj_path, int invert_winding_order, int mode, Mesh *mesh,
                          void *memory, uint64_t memory_bytes);

#ifdef __cplusplus
}
#endif

#endif /* SLIMTRACIN_B200_H */
