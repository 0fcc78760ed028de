/*
 * ref_harness.c — TEST INFRASTRUCTURE, not part of the product.
 *
 * Compiles the reference's own tracing path (render/raytracer.h, the top-down SAH builder, the
 * bmp2texture texture baker and the obj2mesh converter) in place from the reference sources and
 * exposes it to the tests and to bench.py's reference arm as a shared library,
 * oracle/_ref/libslimref.so.  Nothing in the product links or loads this file.
 *
 * The reference is written for Win32, where `unsigned long` is 32 bits.  To get that layout on
 * Linux without copying or patching any reference source, the reference headers are compiled with
 * `long` defined as empty (so `unsigned long` -> `unsigned`, `signed long` -> `signed`) and `u64`
 * pinned to 64 bits with a mode(DI) attribute; the system headers are included first so that the
 * macro never reaches them.  The resulting structs are byte-identical to include/slimtracin_types.h
 * (checked by ref_layout_query against the same X-macro list the library answers from).
 *
 * Build: oracle/Makefile (gcc -O2 -DNDEBUG -ffp-contract=off, no -march, no -ffast-math).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>
#include <stdint.h>
#include <malloc.h>
#include <pthread.h>

#define long
#define u64 u64 __attribute__((mode(DI)))
#include "app.h"
#include "render/raytracer.h"
#define main st_ref_bmp2texture_main
#include "bmp2texture.c"
#undef main
#define main st_ref_obj2mesh_main
#define EndsWith st_ref_obj2mesh_EndsWith
#include "obj2mesh.c"
#undef EndsWith
#undef main
#undef long
#undef u64

#include "../include/slimtracin_layout.h"

/* app.h declares the example's initApp; the harness drives the pieces itself and never calls
 * _initApp, but the symbol must exist for the shared library to load. */
void initApp(Defaults *defaults) { (void)defaults; }

/* ---- layout ----------------------------------------------------------------------------------- */
long ref_layout_query(const char *name) {
#define ST_REF_S(T) if (!strcmp(name, #T)) return (long)sizeof(T);
#define ST_REF_F(T, F) if (!strcmp(name, #T "." #F)) return (long)offsetof(T, F);
    ST_LAYOUT_LIST(ST_REF_S, ST_REF_F)
#undef ST_REF_S
#undef ST_REF_F
    return -1;
}

/* ---- camera / viewport set-up ----------------------------------------------------------------- */
static void fixCameraPointers(Camera *camera) {
    camera->transform.right_direction   = &camera->transform.rotation_matrix.X;
    camera->transform.up_direction      = &camera->transform.rotation_matrix.Y;
    camera->transform.forward_direction = &camera->transform.rotation_matrix.Z;
}

/* beginDrawing (viewport/viewport.h:114): clear + projection matrix + projection plane. */
void ref_begin_drawing(Viewport *viewport) {
    fixCameraPointers(viewport->camera);
    beginDrawing(viewport);
}

/* updateSceneSSB (render/SSB.h:168): per-primitive screen-space bounds and IS_VISIBLE. */
void ref_update_scene_ssb(Scene *scene, Viewport *viewport) {
    updateSceneSSB(scene, viewport);
}

/* ---- render ----------------------------------------------------------------------------------- */
typedef struct {
    Scene *scene;
    Viewport *viewport;
    vec3 *row_starts;
    u32 *rows;
    u32 row_count;
    volatile u32 next_row;
    pthread_mutex_t lock;
    u32 stack_entries;
} RenderJob;

static u32 maxMeshHeight(Scene *scene) {
    u32 h = 0;
    for (u32 m = 0; m < scene->settings.meshes; m++)
        if (scene->meshes[m].bvh.height > h) h = scene->meshes[m].bvh.height;
    return h;
}

/* One thread's share of renderSceneOnCPU (raytracer.h:136): the same per-pixel steps, with a
 * private, zero-initialised Trace (as the app's zeroed arena gives) and large stacks, over whole
 * rows taken from a shared counter.  Each row starts from the projection-plane start advanced by
 * `down` y times in sequence and walks `right` pixel by pixel, exactly as the reference's loop does,
 * so the rays are bit-identical to the single-threaded render. */
static void *renderRows(void *arg) {
    RenderJob *job = (RenderJob*)arg;
    Scene *scene = job->scene;
    Viewport *viewport = job->viewport;
    PixelGrid *frame_buffer = viewport->frame_buffer;
    Dimensions *dim = &frame_buffer->dimensions;

    Trace trace;
    memset(&trace, 0, sizeof(trace));
    trace.depth = viewport->trace.depth;
    trace.closest_mesh_hit.object_type = viewport->trace.closest_mesh_hit.object_type;
    trace.mesh_stack_size = 255;
    trace.scene_stack_size = 255;
    trace.scene_stack = (u32*)calloc(job->stack_entries, sizeof(u32));
    trace.mesh_stack = (u32*)calloc(256, sizeof(u32));

    quat camera_rotation = viewport->camera->transform.rotation_inverted;
    vec3 camera_position = viewport->camera->transform.position;
    vec3 right = viewport->projection_plane.right;
    enum RenderMode mode = viewport->settings.render_mode;
    const u16 w = dim->width;
    Ray ray;
    memset(&ray, 0, sizeof(ray));

    for (;;) {
        pthread_mutex_lock(&job->lock);
        u32 index = job->next_row++;
        pthread_mutex_unlock(&job->lock);
        if (index >= job->row_count) break;
        u16 y = (u16)job->rows[index];
        vec3 current = job->row_starts[y];
        FloatPixel *pixel = frame_buffer->float_pixels + (u32)y * w;
        for (u16 x = 0; x < w; x++, pixel++) {
            ray.origin = camera_position;
            ray.direction = normVec3(current);
            ray.direction_reciprocal = oneOverVec3(ray.direction);
            trace.closest_hit.distance = trace.closest_hit.distance_squared = INFINITY;
            trace.closest_hit.cone_angle = viewport->projection_plane.cone_angle;
            trace.closest_hit.cone_width = 0;
            rayTrace(&ray, &trace, scene, mode, pixel, x, y, camera_position, camera_rotation);
            current = addVec3(current, right);
        }
    }
    free(trace.scene_stack);
    free(trace.mesh_stack);
    return NULL;
}

/* Render rows y_first, y_first+y_step, ... (y_count of them) of the QCAA grid with `threads`
 * threads.  The caller has run ref_begin_drawing (clear + projection plane) and, when wanted,
 * ref_update_scene_ssb.  Returns 0. */
int ref_render_rows(Scene *scene, Viewport *viewport, int threads, u32 y_first, u32 y_step, u32 y_count) {
    Dimensions *dim = &viewport->frame_buffer->dimensions;
    u32 h = dim->height;
    if (threads < 1) threads = 1;
    if (scene->settings.meshes) viewport->trace.closest_mesh_hit.object_type = PrimitiveType_Mesh;
    (void)maxMeshHeight;

    RenderJob job;
    job.scene = scene;
    job.viewport = viewport;
    job.row_starts = (vec3*)malloc(sizeof(vec3) * (h ? h : 1));
    vec3 start = viewport->projection_plane.start;
    for (u32 y = 0; y < h; y++) {
        job.row_starts[y] = start;
        start = addVec3(start, viewport->projection_plane.down);
    }
    job.rows = (u32*)malloc(sizeof(u32) * (y_count ? y_count : 1));
    job.row_count = 0;
    for (u32 i = 0; i < y_count; i++) {
        u32 y = y_first + i * y_step;
        if (y < h) job.rows[job.row_count++] = y;
    }
    job.next_row = 0;
    pthread_mutex_init(&job.lock, NULL);
    job.stack_entries = scene->settings.primitives * 2 + 64;

    if (threads == 1) {
        renderRows(&job);
    } else {
        pthread_t *tids = (pthread_t*)malloc(sizeof(pthread_t) * threads);
        for (int t = 0; t < threads; t++) pthread_create(&tids[t], NULL, renderRows, &job);
        for (int t = 0; t < threads; t++) pthread_join(tids[t], NULL);
        free(tids);
    }
    pthread_mutex_destroy(&job.lock);
    free(job.rows);
    free(job.row_starts);
    return 0;
}

/* The reference's per-frame sequence of an example's updateAndRender (e.g. 02_Geometry.c:80-83):
 * updateSceneSSB (optional) -> beginDrawing -> renderScene -> drawViewportToWindowContent.
 * threads == 0 calls the reference's own single-threaded renderSceneOnCPU (raytracer.h:136). */
int ref_render_frame(Scene *scene, Viewport *viewport, int threads, int update_ssb) {
    if (update_ssb) ref_update_scene_ssb(scene, viewport);
    ref_begin_drawing(viewport);
    if (threads == 0) {
        Trace saved = viewport->trace;
        u32 *scene_stack = (u32*)calloc(scene->settings.primitives * 2 + 64, sizeof(u32));
        u32 *mesh_stack = (u32*)calloc(256, sizeof(u32));
        viewport->trace.scene_stack = scene_stack;
        viewport->trace.mesh_stack = mesh_stack;
        viewport->trace.mesh_stack_size = 255;
        if (scene->settings.meshes) viewport->trace.closest_mesh_hit.object_type = PrimitiveType_Mesh;
        renderSceneOnCPU(scene, viewport);
        saved.closest_mesh_hit.object_type = viewport->trace.closest_mesh_hit.object_type;
        viewport->trace = saved;
        free(scene_stack);
        free(mesh_stack);
    } else {
        ref_render_rows(scene, viewport, threads, 0, 1, viewport->frame_buffer->dimensions.height);
    }
    if (viewport->frame_buffer->pixels) drawViewportToWindowContent(viewport);
    return 0;
}

/* drawViewportToWindowContent (viewport/viewport.h:12): the QCAA resolve alone. */
void ref_resolve(Viewport *viewport) {
    drawViewportToWindowContent(viewport);
}

/* ---- BVH builds ------------------------------------------------------------------------------- */
static void *builderArena(Scene *scene, u32 leaf_count, BVHBuilder *builder) {
    u64 size = (u64)getBVHBuilderMemorySize(scene, leaf_count) + 4096;
    void *mem = calloc(1, size);
    Memory memory;
    initMemory(&memory, (u8*)mem, size);
    builder->build_iterations = (BuildIteration*)allocateMemory(&memory, sizeof(BuildIteration) * leaf_count);
    builder->leaf_nodes       = (BVHNode*       )allocateMemory(&memory, sizeof(BVHNode)        * leaf_count);
    builder->leaf_ids         = (u32*           )allocateMemory(&memory, sizeof(u32)            * leaf_count);
    builder->sort_stack       = (i32*           )allocateMemory(&memory, sizeof(i32)            * leaf_count);
    PartitionAxis *pa = builder->partition_axis;
    for (u8 i = 0; i < 3; i++, pa++) {
        pa->sorted_leaf_ids     = (u32* )allocateMemory(&memory, sizeof(u32)  * leaf_count);
        pa->left.aabbs          = (AABB*)allocateMemory(&memory, sizeof(AABB) * leaf_count);
        pa->right.aabbs         = (AABB*)allocateMemory(&memory, sizeof(AABB) * leaf_count);
        pa->left.surface_areas  = (f32* )allocateMemory(&memory, sizeof(f32)  * leaf_count);
        pa->right.surface_areas = (f32* )allocateMemory(&memory, sizeof(f32)  * leaf_count);
    }
    return mem;
}

/* updateSceneBVH (builder_top_down.h:366).  scene->bvh.nodes must hold 2*primitives nodes and
 * scene->bvh.leaf_ids `primitives` ids (initBVH, core/init.h:503). */
void ref_update_scene_bvh(Scene *scene) {
    BVHBuilder builder;
    u32 leaf_count = scene->settings.primitives;
    for (u32 m = 0; m < scene->settings.meshes; m++)
        if (scene->meshes[m].triangle_count > leaf_count) leaf_count = scene->meshes[m].triangle_count;
    void *mem = builderArena(scene, leaf_count ? leaf_count : 1, &builder);
    updateSceneBVH(scene, &builder);
    free(mem);
}

/* updateMeshBVH (builder_top_down.h:272).  mesh->bvh.nodes (2N), mesh->bvh.leaf_ids (N) and
 * mesh->triangles (N) are caller-allocated. */
void ref_update_mesh_bvh(Mesh *mesh) {
    BVHBuilder builder;
    Scene dummy;
    memset(&dummy, 0, sizeof(dummy));
    u32 n = mesh->triangle_count ? mesh->triangle_count : 1;
    void *mem = builderArena(&dummy, n, &builder);
    updateMeshBVH(mesh, &builder);
    free(mem);
}

/* ---- mesh / texture files --------------------------------------------------------------------- */
static void *stOpen(const char *path) { return fopen(path, "rb"); }
static bool stRead(void *out, unsigned size, void *handle) { return fread(out, 1, size, (FILE*)handle) == size; }
static void stClose(void *handle) { fclose((FILE*)handle); }

/* loadMeshFromFile (scene/io.h:95) into an arena the harness allocates; returns the arena (free it
 * with ref_free) or NULL. */
void *ref_load_mesh(const char *path, Mesh *mesh) {
    Platform platform;
    memset(&platform, 0, sizeof(platform));
    platform.openFileForReading = (CallbackForFileOpen)stOpen;
    platform.readFromFile = stRead;
    platform.closeFile = stClose;
    FILE *probe = fopen(path, "rb");
    if (!probe) return NULL;
    fclose(probe);
    Mesh sizing;
    memset(&sizing, 0, sizeof(sizing));
    u64 size = (u64)getMeshMemorySize(&sizing, (char*)path, &platform) + 4096;
    void *mem = calloc(1, size);
    Memory memory;
    initMemory(&memory, (u8*)mem, size);
    loadMeshFromFile(mesh, (char*)path, &platform, &memory);
    return mem;
}

/* loadTexture (bmp2texture.c:324): bake an RGB(A) image into the TexelQuad mip chain. */
void ref_load_texture(Texture *texture, u16 width, u16 height, int wrap, int mipmap,
                      u8 *texel_components, int bit_count) {
    loadTexture(texture, width, height, (bool)wrap, (bool)mipmap, texel_components, (u8)bit_count);
}

void ref_free_texture(Texture *texture) {
    for (u8 i = 0; i < texture->mip_count; i++) free(texture->mips[i].texel_quads);
    free(texture->mips);
    texture->mips = NULL;
}

void ref_free(void *p) { free(p); }

/* The picking ray of manipulateSelection (viewport/manipulation.h:55-123), run with the reference's
 * own functions: setViewportProjectionPlane, setRayFromCoords (shaders/common.h:170), hitPrimitives
 * over scene->bvh.leaf_ids with the visibility cull at (x, y), then every light's glow sphere
 * (hitSphereSimple, sphere.h:44).  Outputs the hit the selection would take: found, object type and
 * id, world position, distance and the camera-space z the selection keeps (object_distance). */
typedef struct { int found, object_type; u32 object_id; vec3 position; f32 distance, object_distance; } RefPick;
int ref_pick(Scene *scene, Viewport *viewport, int x, int y, RefPick *out) {
    Trace trace;
    memset(&trace, 0, sizeof(trace));
    trace.scene_stack = (u32*)calloc(scene->settings.primitives * 2 + 64, sizeof(u32));
    trace.mesh_stack = (u32*)calloc(256, sizeof(u32));
    trace.mesh_stack_size = 255;
    trace.scene_stack_size = 255;
    if (scene->settings.meshes) trace.closest_mesh_hit.object_type = PrimitiveType_Mesh;
    setViewportProjectionPlane(viewport);
    vec2i coords;
    coords.x = x;
    coords.y = y;
    Ray ray;
    setRayFromCoords(&ray, coords, viewport);
    ray.direction_reciprocal = oneOverVec3(ray.direction);
    RayHit *hit = &trace.closest_hit;
    hit->distance = hit->distance_squared = MAX_DISTANCE;
    bool found = hitPrimitives(&ray, &trace, scene, scene->bvh.leaf_ids, scene->settings.primitives, false, true,
                               (u16)x, (u16)y);
    Light *light = scene->lights;
    if (light) {
        for (u32 i = 0; i < scene->settings.lights; i++, light++) {
            f32 light_radius = light->intensity * (1.0f / (8.0f * 16.0f));
            trace.sphere_hit.furthest = hit->distance / light_radius;
            if (hitSphereSimple(ray.origin, ray.direction, light->position_or_direction, 1.0f / light_radius,
                                &trace.sphere_hit)) {
                hit->distance = trace.sphere_hit.t_near * light_radius;
                hit->position = scaleAddVec3(ray.direction, hit->distance, ray.origin);
                hit->object_type = PrimitiveType_Light;
                hit->object_id = i;
                found = true;
            }
        }
    }
    memset(out, 0, sizeof(*out));
    out->found = found;
    if (found) {
        out->object_type = hit->object_type;
        out->object_id = hit->object_id;
        out->position = hit->position;
        out->distance = hit->distance;
        out->object_distance = mulVec3Mat3(subVec3(hit->position, ray.origin),
                                           viewport->camera->transform.rotation_matrix_inverted).z;
    }
    free(trace.scene_stack);
    free(trace.mesh_stack);
    return 0;
}

/* The debug overlays with the reference's own drawBVH (render/raytracer.h:46) and drawSSB
 * (render/SSB.h:175), after initBox on the viewport's default box as initViewport does
 * (core/init.h:443).  what: 1 = BVH, 2 = SSB.  drawBVH counts nodes with a u8, so a BVH of 256 or
 * more nodes would never finish: refused with -1. */
int ref_draw_overlays(Scene *scene, Viewport *viewport, int what) {
    if ((what & 1) && scene->bvh.node_count > 255) return -1;
    initBox(&viewport->default_box);
    if (what & 1) drawBVH(scene, viewport);
    if (what & 2) drawSSB(scene, viewport);
    return 0;
}

/* ---- the reference's file formats (scene/io.h) ---------------------------------------------- */
static void *stOpenW(const char *path) { return fopen(path, "wb"); }
static bool stWrite(void *in, unsigned size, void *handle) { return fwrite(in, 1, size, (FILE*)handle) == size; }
static void fileCallbacks(Platform *platform) {
    memset(platform, 0, sizeof(*platform));
    platform->openFileForReading = (CallbackForFileOpen)stOpen;
    platform->openFileForWriting = (CallbackForFileOpen)stOpenW;
    platform->readFromFile = stRead;
    platform->writeToFile = (CallbackForFileRW)stWrite;
    platform->closeFile = stClose;
}

/* saveMeshToFile (scene/io.h:145) */
void ref_save_mesh(Mesh *mesh, const char *path) {
    Platform platform;
    fileCallbacks(&platform);
    saveMeshToFile(mesh, (char*)path, &platform);
}

/* saveSceneToFile (scene/io.h:199) and loadSceneFromFile (:178) */
void ref_save_scene(Scene *scene, const char *path) {
    Platform platform;
    fileCallbacks(&platform);
    saveSceneToFile(scene, (char*)path, &platform);
}
void ref_load_scene(Scene *scene, const char *path) {
    Platform platform;
    fileCallbacks(&platform);
    loadSceneFromFile(scene, (char*)path, &platform);
}

/* loadTextureFromFile (scene/io.h:34) into an arena the harness allocates (free with ref_free) */
void *ref_load_texture_file(Texture *texture, const char *path, u64 bytes) {
    Platform platform;
    fileCallbacks(&platform);
    void *mem = calloc(1, bytes);
    Memory memory;
    initMemory(&memory, (u8*)mem, bytes);
    loadTextureFromFile(texture, (char*)path, &platform, &memory);
    return mem;
}
