// st_kernels.h — host-visible kernel launchers and the per-view parameter block.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "st_device.cuh"

namespace st {

// One view: what rayTrace / renderSceneOnCPU read from the Viewport and its Camera
// (raytracer.h:136-170) and what computeSSB reads from the frame buffer's Dimensions (SSB.h:5).
constexpr int kSegment = 8;        // grid points per stored row-segment start (row_segments_kernel)

struct ViewDev {
    v3 cam_pos;
    q4 cam_rot_inv;                 // camera->transform.rotation_inverted
    float cam_rot_matrix_inv[9];    // camera->transform.rotation_matrix_inverted (SSB.h:143)
    float focal_length;
    v3 pp_start, pp_right, pp_down; // viewport->projection_plane
    float cone_angle;
    u32t grid_w, grid_h;            // QCAA grid (W+1)x(H+1)
    float f_width, f_height, h_width, h_height, width_over_height, height_over_width;
    int mode;                       // enum RenderMode
    u32t depth;                     // trace.depth (bounces)
    int primary_tlas;               // 1: primary rays walk the TLAS (with the SSB cull); 0: brute force
};

// One view of a batch: the scene it renders, the view, its per-view scratch and outputs, and where
// its tiles start in the batch's tile numbering.
struct BatchView {
    SceneDev scene;
    ViewDev view;
    const int4 *ssb;
    const float *dirs;             // row-segment starts (row_segments_kernel)
    FloatPixel *out;
    u32t *prim_ids;
    uint32_t *out_u8;              // resolved frame (device), or null
    u32t tile_begin;               // first tile slot (4 per group of warp tiles)
    u32t groups_y;                 // groups of warp tiles per column of groups
};
// Warp tiles across one group of four: groups cover about 8x16 grid points (four 8x4 tiles
// stacked, 2x2 tiles of 4x8, four 16x2 or 32x1 tiles stacked).
__host__ __device__ constexpr u32t group_tiles_w(int tile_w) { return tile_w >= 8 ? 1u : 2u; }
// A batch's views as a kernel parameter of its set-up and resolve kernels: one launch group takes at
// most kTableViews views.  (The trace kernel reads the same views from device memory: indexed by a
// tile's view, kernel-parameter memory measured slower there than an L1-cached table.)
constexpr int kTableViews = 64;
struct BatchTable {
    BatchView v[kTableViews];
};
static_assert(sizeof(BatchTable) + 64 <= 32764, "kernel parameters are limited to 32764 bytes");
enum TileShape { TILE_8x4 = 0, TILE_16x2 = 1, TILE_32x1 = 2, TILE_4x8 = 3, TILE_SHAPES = 4 };
// A batch kernel variant: tile shape + TILE_SHAPES * stack placement (0: traversal stacks in local
// memory; 1: their first kSharedStackEntries entries in shared memory).
constexpr int kSharedStackEntries = 16;
constexpr int STACK_PLACEMENTS = 2;
constexpr int BATCH_VARIANTS = TILE_SHAPES * STACK_PLACEMENTS;
inline int variant_tile(int variant) { return variant % TILE_SHAPES; }
inline int variant_stack(int variant) { return variant / TILE_SHAPES; }
// The other launch mode of a batch: one per-frame trace kernel per view, views spread over
// kAuxStreams streams (16 streams measured the same as 8 on the 64-view mix and the served stream).
constexpr int kPerViewVariant = BATCH_VARIANTS;
#ifndef ST_AUX_STREAMS
#define ST_AUX_STREAMS 8
#endif
constexpr int kAuxStreams = ST_AUX_STREAMS;

// A grid point of a batch parked at a bounce: the persistent kernel's warp-vote compaction moves the
// bounce rays of a warp that few lanes still trace into a queue, and drain_kernel traces them to the
// end.  The record holds the whole path state carried across shadeSurface's bounce loop
// (surface.h:180-239): the bounce ray, colour, throughput, the ray-cone footprints, the glow limit,
// the bounces left and the primary hit's distance and depth.
struct __align__(16) ParkedRay {
    float4 origin_r;               // bounce ray origin xyz, colour r
    float4 direction_g;            // bounce ray direction xyz, colour g
    float4 throughput_b;           // throughput xyz, colour b
    float4 carry;                  // du, dv, max_distance, closest_distance
    uint4 where;                   // x, y, view in the launch group (kEmptySlot: nothing parked there),
                                   // bounces << 2 | lights_shaded << 1 | hit_found
    float4 depth;                  // z, unused x3
};
constexpr u32t kEmptySlot = 0xFFFFFFFFu;
// The queue of one launch group: `threshold` is the warp-vote limit (a warp whose lanes still tracing
// at a bounce number fewer than it parks them; 0: never), `reserved` counts slots handed out (parks
// beyond `capacity` are refused and traced in place), `taken` the slots drained.
struct ParkQueue {
    ParkedRay *rays = nullptr;
    u32t *reserved = nullptr, *taken = nullptr;
    u32t *drained = nullptr;       // the batch's total of parked paths traced by the drain (all groups)
    u32t capacity = 0, threshold = 0;
};
constexpr u32t kParkCapacity = 1u << 20;   // parked rays per launch group at most (96 MB)

void launch_ssb(const SceneDev &S, const ViewDev &v, int4 *ssb, cudaStream_t st);
int launch_batch(const BatchView *views, u32t n_views, u32t total_tiles, int variant, u32t chunk, u32t grid_blocks,
                 u32t *tile_counter, unsigned *status, unsigned long long *counters, bool count, cudaStream_t st,
                 const ParkQueue &park);
// The parked rays of a launch group, traced to the end (a persistent grid of grid_blocks blocks).
int launch_drain(const BatchView *views, const ParkQueue &park, int variant, u32t grid_blocks, unsigned *status,
                 unsigned long long *counters, bool count, cudaStream_t st);
void tile_dims(int variant, u32t &tw, u32t &th);
int batch_blocks_per_sm(int variant);
// Row-segment starts of the view's ray directions: ceil(grid_w / kSegment) x grid_h float3,
// segment-major.
void launch_ray_rows(const ViewDev &v, float *dirs, cudaStream_t st);
inline size_t ray_rows_floats(const ViewDev &v) { return (size_t)v.grid_h * ((v.grid_w + kSegment - 1) / kSegment) * 3; }
// Block columns [bx_first, bx_first + bx_count) of the grid (8 grid points wide each; bx_count 0:
// to the last column).  overlapped: the grid is copied to the host while it is traced (the kernel
// then runs with fewer blocks per SM).
void launch_trace(const SceneDev &S, const ViewDev &v, const int4 *ssb, const float *dirs, FloatPixel *out,
                  u32t *prim_ids, unsigned *status, unsigned long long *counters, bool count, cudaStream_t st,
                  u32t bx_first = 0, u32t bx_count = 0, bool overlapped = false);
// The result of a pick (layout of st_pick_result)
struct PickDev {
    int found, object_type;
    u32t object_id;
    float position[3];
    float distance, object_distance;
};
void launch_pick(const SceneDev &S, const ViewDev &v, const int4 *ssb, int x, int y, PickDev *out, cudaStream_t st);
// Pixel columns [x0, x1) of the QCAA resolve (all of them by default).
void launch_resolve(const FloatPixel *in, u32t grid_w, u32t width, u32t height, uint32_t *out, cudaStream_t st,
                    u32t x0 = 0, u32t x1 = 0xFFFFFFFFu);
// A batch's SSBs and ray-row starts (every view of the table), and its resolves (views with out_u8).
void launch_batch_setup(const BatchTable &T, u32t n_views, u32t max_prims, u32t max_rows, cudaStream_t st);
void launch_batch_resolve(const BatchTable &T, u32t n_views, u32t max_width, u32t max_height, cudaStream_t st);

// ---- BVH builds (st_bvh.cu, st_sah.cu, st_refsah.cu) ----
// The reference's full-sweep SAH (buildBVH) over n device boxes: nodes and leaf ids as the reference
// lays them out, info = {node_count, height}; synchronous on st.
cudaError_t refsah_build(const float *boxes, u32t n, u32t max_leaf, BVHNode *nodes, u32t *leaf_ids, u32t info[2],
                         cudaStream_t st);
// Device scratch the LBVH build needs for n items (allocated once per context and grown).
struct LbvhScratch {
    u32t capacity = 0;
    float *aabbs = nullptr;          // 6 floats per item (world boxes)
    unsigned *bounds = nullptr;      // 6 ordered-bit words: scene min.xyz, max.xyz
    u32t *codes = nullptr, *codes_alt = nullptr;
    u32t *order = nullptr, *order_alt = nullptr;
    u32t *hist = nullptr;            // 256 * blocks
    u32t *first = nullptr, *last = nullptr, *lchild = nullptr, *rchild = nullptr, *parent = nullptr;
    u32t *leaf_parent = nullptr, *rank = nullptr, *flags = nullptr;
    unsigned *kbox = nullptr;        // 6 ordered-bit words per internal node
    u32t *info = nullptr;            // node_count, height
};

cudaError_t lbvh_reserve(LbvhScratch &s, u32t n);
void lbvh_release(LbvhScratch &s);
// Bytes of one caller-provided block holding every LbvhScratch array except aabbs for builds of up
// to `cap` items (radix tiles of 2048 items, scan blocks of 1024 elements; arrays 256-byte aligned).
constexpr size_t lbvh_align(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t lbvh_scratch_bytes(u32t cap) {
    return lbvh_align(32) + 12 * lbvh_align(4 * (size_t)cap) + lbvh_align(24 * (size_t)cap) + lbvh_align(16) +
           lbvh_align(8 * (256 * (((size_t)cap + 2047) / 2048) + 2 * (((size_t)cap + 1023) / 1024) + 64));
}
// Point the arrays of `s` (aabbs excepted) into `base`, a 256-byte aligned block of
// lbvh_scratch_bytes(cap) bytes; s.capacity = cap.
void lbvh_carve(LbvhScratch &s, void *base, u32t cap);
// Items' world boxes -> Morton codes -> stable radix sort -> Karras tree -> leaf collapse ->
// reference-layout BVHNode array (1 + 2*kept nodes) + leaf order.  Synchronous w.r.t. `st`.
// out_nodes must hold 2n nodes; out_order n ids.  info (host) receives node_count, height.
cudaError_t lbvh_build(LbvhScratch &s, u32t n, u32t max_leaf, BVHNode *out_nodes, u32t *out_order,
                       u32t info[2], cudaStream_t st);
// The same build (n > 0) without waiting: counts[3] (page-locked host memory, filled once `st`
// reaches it) receive the words from which node_count = 1 + 2 * counts[2] and height = counts[1].
void lbvh_enqueue(LbvhScratch &s, u32t n, u32t max_leaf, BVHNode *out_nodes, u32t *out_order, u32t *counts,
                  cudaStream_t st);
// Binned SAH over n device boxes (st_sah.cu): reference-layout nodes (2n capacity) + leaf order.
// scratch (optional, sah_scratch_bytes(n) bytes): used instead of a stream-ordered allocation
cudaError_t sah_build(const float *aabbs, u32t n, u32t max_leaf, BVHNode *out_nodes, u32t *out_order, u32t info[2],
                      cudaStream_t st, void *scratch = nullptr, size_t scratch_bytes = 0);
size_t sah_scratch_bytes(u32t n);
// After lbvh_build: the Morton code of every item, by item index.
void launch_codes_by_item(const LbvhScratch &s, u32t n, u32t *out, cudaStream_t st);
// World boxes of primitives as updateSceneBVH computes them (builder_top_down.h:370-377).
void launch_prim_aabbs(const Primitive *prims, const MeshDev *meshes, u32t n, float *aabbs, cudaStream_t st);
// Triangle boxes with the reference's EPS padding (builder_top_down.h:283-318).
void launch_tri_aabbs(const vec3 *pos, const uint32_t *idx, u32t n, float *aabbs, cudaStream_t st);
// The Triangle record of updateMeshBVH (builder_top_down.h:330-363) for every leaf-ordered slot.
void launch_tri_records(const vec3 *pos, const vec3 *nrm, const vec2 *uv, const uint32_t *pidx, const uint32_t *nidx,
                        const uint32_t *uidx, int has_uvs, const u32t *order, u32t n, Triangle *out,
                        u32t *inverse, cudaStream_t st);
// Refit: recompute every node box of a reference-layout BVH whose items' boxes are `aabbs`
// (leaf ranges index `leaf_ids`), bottom-up.
cudaError_t refit_bvh(BVHNode *nodes, u32t node_count, const u32t *leaf_ids, const float *aabbs,
                      u32t *scratch_parent, u32t *scratch_flags, unsigned *scratch_box, cudaStream_t st);
// Reference-layout BVHNode array -> child-pair array (pair k = nodes 1+2k, 2+2k).
void launch_make_pairs(const BVHNode *nodes, u32t node_count, NodePair *pairs, cudaStream_t st);
// Triangle -> TriHot
void launch_make_trihot(const Triangle *tris, u32t n, TriHot *hot, cudaStream_t st);
// Primitive -> PrimDev
void launch_make_primdev(const Primitive *prims, u32t n, PrimDev *out, cudaStream_t st);
// recs[k] replaces primitive ids[k] (distinct ids): raw record and PrimDev
void launch_scatter_prims(const Primitive *recs, const u32t *ids, u32t count, Primitive *raw, PrimDev *dev,
                          cudaStream_t st);

// ---- texture baking (st_texture.cu): loadTexture bmp2texture.c:324 ----
int texture_mip_count(u32t width, u32t height, bool mipmap);
size_t texture_quad_count(u32t width, u32t height, bool mipmap);
size_t texture_scratch_bytes(u32t width, u32t height);
// dev_components: width*height texels of 3 (bit_count 24) or 4 (32) bytes; scratch:
// texture_scratch_bytes; dev_quads: texture_quad_count quads, mip after mip.
cudaError_t bake_texture(const uint8_t *dev_components, u32t width, u32t height, int bit_count, bool wrap, bool mipmap,
                         void *scratch, TexelQuad *dev_quads, cudaStream_t st);

// ---- OBJ ingestion (st_obj.cu): obj2mesh.c:25 ----
struct ObjCounts {
    uint32_t vertices = 0, normals = 0, uvs = 0, triangles = 0;
    int layout = 0;    // face layout of obj2mesh: 0 unknown, 1 positions, 2 positions/uvs, 3 positions/uvs/normals
};
// Count pass: -1 when the file cannot be read.
int obj_count(const char *path, ObjCounts &c);
// Parse pass into caller arrays sized by `expect` (the count pass): -1 unreadable or changed file,
// -2 a line that does not parse with the face layout or an index out of range.
int obj_parse(const char *path, bool invert_winding, const ObjCounts &expect, vec3 *positions, vec3 *normals, vec2 *uvs,
              uint32_t *position_ids, uint32_t *uv_ids, uint32_t *normal_ids);
// The unique undirected triangle sides in first-appearance order (obj2mesh.c:209-234); dev_edges
// holds up to 3 * n_triangles.  Synchronises `st`.
size_t unique_edges_scratch_bytes(u32t n_triangles);
cudaError_t unique_edges(const uint32_t *dev_ids, u32t n_triangles, u32t n_vertices, void *scratch,
                         EdgeVertexIndices *dev_edges, u32t *n_edges, cudaStream_t st);

// ---- shared primitives (st_bvh.cu) ----
// Exclusive scan of n u32 values (in place allowed); sums: (n/1024 + 1) words of scratch; total
// (optional, device) receives the sum.
void scan_exclusive_u32(const u32t *in, u32t *out, u32t n, u32t *sums, u32t *total, cudaStream_t st);
// Stable LSD radix sort of n (key, value) pairs on the low 8*passes bits of the keys, ping-ponging
// between (k0, v0) and (k1, v1); returns 1 when the result is in (k1, v1), 0 when in (k0, v0).
// scratch: radix_sort_scratch_bytes(n) bytes.
size_t radix_sort_scratch_bytes(u32t n);
int radix_sort_pairs(u32t *k0, u32t *v0, u32t *k1, u32t *v1, u32t n, int passes, void *scratch, cudaStream_t st);

// ---- debug overlays (st_overlay.cu): drawBVH raytracer.h:46, drawSSB SSB.h:175 ----
// One BLAS node drawMeshAccelerationStructure outlines (depth <= 5): its box and colour id
// (Magenta leaf, Green inner, Blue root).
struct OutlineBox {
    float aabb[6];
    u32t color, pad;
};
struct OverlayParams {
    const BVHNode *nodes;          // the TLAS (reference layout), node_count nodes; null: no BVH overlay
    u32t node_count;
    const u32t *leaf_ids;
    const Primitive *prims;
    u32t n_prims;
    const OutlineBox *outlines;    // every mesh's outlined nodes, in node order
    const uint2 *outline_range;    // per mesh: (first outline, count)
    u32t n_meshes;
    v3 cam_pos;
    q4 cam_rot_inv;                // camera->transform.rotation_inverted
    float proj[16];                // viewport->projection_matrix, rows X Y Z W
    float near_plane, far_plane, focal_length;
    float width_over_height, h_width, h_height, f_height;   // frame buffer Dimensions
    u32t width, height, stride;    // frame buffer width/height (the QCAA grid); stride = width
    int pos_x, pos_y;              // viewport->position
    u32t grid_pixels;              // pixels in the float grid
};
// Device scratch for one overlay pass with n_boxes boxes (0: drawSSB only).
size_t overlay_scratch_bytes(const OverlayParams &P, u32t n_boxes);
size_t overlay_fragment_bytes(u32t n_frags);
// Pass 1: boxes, edges and the number of pixels the overlays plot (synchronises `st`).
cudaError_t overlay_count(const OverlayParams &P, const int4 *ssb, u32t n_boxes, void *scratch, u32t *n_frags,
                          cudaStream_t st);
// Pass 2: plot, sort by pixel and blend into grid (and grid_host, a device view of a page-locked
// host copy, when non-null).  frag_buf: overlay_fragment_bytes(n_frags) bytes.
cudaError_t overlay_draw(const OverlayParams &P, const int4 *ssb, u32t n_boxes, void *scratch, u32t n_frags,
                         void *frag_buf, FloatPixel *grid, FloatPixel *grid_host, cudaStream_t st);

}  // namespace st
