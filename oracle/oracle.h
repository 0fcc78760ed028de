/*
 * oracle.h — TEST INFRASTRUCTURE: the CPU restatement of SlimTracin's tracing path.
 * Only tests, the smoke check and bench.py's CPU-baseline arm load liboracle.so.
 */
#ifndef ST_ORACLE_H
#define ST_ORACLE_H
#include "slimtracin_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Event counters of one render, same indices as the library's enum st_counter. */
enum {
    ORC_PRIMARY_RAYS = 0, ORC_SHADOW_RAYS = 1, ORC_BOUNCE_RAYS = 2, ORC_AABB_TESTS = 3,
    ORC_TRIANGLE_TESTS = 4, ORC_PRIMITIVE_TESTS = 5, ORC_LEAF_ID_READS = 6, ORC_SHADED_HITS = 7,
    ORC_TEXEL_FETCHES = 8, ORC_MESH_ENTRIES = 9, ORC_TEXEL_MIP_FETCHES = 10,
    ORC_COUNTERS = 16
};

/* Render the whole QCAA grid of viewport->frame_buffer (clear, trace every ray, resolve to
 * frame_buffer->pixels when non-null) with `threads` threads.  The caller fills
 * viewport->projection_plane.  Primitive screen bounds/visibility are taken from `scene` as given
 * (call orc_update_scene_ssb first).  prim_ids (optional, grid-sized) receives the primary-hit
 * primitive id or 0xFFFFFFFF; counters (optional) receives ORC_COUNTERS u64s. */
int orc_render_frame(const Scene *scene, Viewport *viewport, int threads, uint32_t *prim_ids,
                     uint64_t *counters);

/* updateSceneSSB (render/SSB.h:168) restated; writes screen_bounds and IS_VISIBLE. */
void orc_update_scene_ssb(Scene *scene, const Viewport *viewport);

/* updateSceneBVH (builder_top_down.h:366) and updateMeshBVH (:272) restated. */
void orc_update_scene_bvh(Scene *scene);
void orc_update_mesh_bvh(Mesh *mesh);

/* World AABBs of the scene's primitives as updateSceneBVH computes them: out[6*i .. 6*i+5] =
 * min.xyz, max.xyz. */
void orc_primitive_aabbs(const Scene *scene, float *out);

/* The 30-bit Morton LBVH over `n` AABBs (aabbs: 6 floats each) with leaves of at most
 * `max_leaf` items.  Outputs: codes[n] (Morton code of item i), order[n] (items sorted by
 * (code, index)), nodes[2n] in the reference's BVHNode layout, and info[2] = {node_count,
 * height}.  Returns 0. */
int orc_lbvh30(const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *codes, uint32_t *order,
               BVHNode *nodes, uint32_t *leaf_ids, uint32_t *info);

/* Binned SAH over `n` AABBs (32 bins, breadth-first, the project's specification; see oracle.c).
 * Outputs order[n] (leaf order), nodes[2n] in the reference's BVHNode layout, info = {node_count,
 * height}.  Returns 0. */
int orc_binned_sah(const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *order, BVHNode *nodes,
                   uint32_t *info);

/* updateMeshBVH (builder_top_down.h:272) with the binned-SAH topology of orc_binned_sah: fills
 * mesh->bvh (nodes, leaf_ids as source triangle -> slot, node_count, height) and mesh->triangles
 * in leaf order, like the library's st_update_mesh_bvh(ST_BVH_BINNED_SAH).  Returns 0. */
int orc_update_mesh_bvh_binned(Mesh *mesh);

/* The object a click at pixel (x, y) selects (manipulateSelection, viewport/manipulation.h:55):
 * found, PrimitiveType (PrimitiveType_Light for a light's glow sphere), index, world position,
 * distance along the picking ray and camera-space z. */
typedef struct OrcPick {
    int found, object_type;
    uint32_t object_id;
    vec3 position;
    float distance, object_distance;
} OrcPick;
int orc_pick(const Scene *scene, const Viewport *viewport, int x, int y, OrcPick *out);

/* The debug overlays drawBVH (render/raytracer.h:46) and drawSSB (render/SSB.h:175), drawn into
 * viewport->frame_buffer->float_pixels with viewport->projection_matrix (set by beginDrawing) and
 * the unit box of initBox.  drawSSB reads the primitives' screen_bounds and IS_VISIBLE (call
 * orc_update_scene_ssb first).  drawBVH walks all scene->bvh.node_count nodes (the reference's u8
 * node counter only terminates below 256 nodes). */
enum { ORC_OVERLAY_BVH = 1, ORC_OVERLAY_SSB = 2 };
void orc_draw_overlays(const Scene *scene, const Viewport *viewport, int what);

#ifdef __cplusplus
}
#endif
#endif
