/*
 * dropin.c — TEST INFRASTRUCTURE, not part of the product.
 *
 * A SlimTracin host written the way an example is (examples/02_Geometry.c:75-83): compiled from the
 * reference's own headers, with the reference's scene, camera and viewport code, its top-down SAH
 * TLAS build and its per-frame sequence (updateSceneSSB, beginDrawing, renderScene,
 * drawViewportToWindowContent) — and the GPU seams bound to libslimtracin_b200 through the C ABI
 * (allocateDeviceScene and the upload* stubs forward to st_allocate_device_scene / st_upload_*,
 * renderScene to st_render_scene).  The test compares its GPU frames with the same host's CPU frames.
 *
 * Built by oracle/Makefile into oracle/_ref/libdropin.so (it needs the reference sources; the
 * reference's 32-bit `u32` is obtained as in ref_harness.c).
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
#undef long
#undef u64

#define SLIMTRACIN_REFERENCE_TYPES
#include "slimtracin_b200.h"

void initApp(Defaults *defaults) { (void)defaults; }

static st_ctx *g_st;

/* The seams an integrator fills (core/init.h:36-126, render/raytracer.h:302), slot 0. */
static int dropin_upload(Scene *scene) {
    if (!g_st) {
        st_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        int s = st_init(&g_st, &cfg);
        if (s != ST_OK) return s;
    }
    int s = st_allocate_device_scene(g_st, 0, scene);                 /* allocateDeviceScene */
    if (s == ST_OK) s = st_upload_scene(g_st, 0, scene);              /* uploadScene */
    if (s == ST_OK && scene->settings.meshes) s = st_upload_mesh_bvhs(g_st, 0, scene);   /* uploadMeshBVHs */
    if (s == ST_OK) s = st_upload_scene_bvh(g_st, 0, scene);          /* uploadSceneBVH, after updateSceneBVH */
    return s;
}

/* One frame of the host: the TLAS from the reference's own builder on the first frame, then the
 * reference's per-frame sequence with renderScene on the device (use_gpu) or the reference CPU. */
int dropin_frame(Scene *scene, Viewport *viewport, int use_gpu, int first_frame) {
    Camera *camera = viewport->camera;
    camera->transform.right_direction = &camera->transform.rotation_matrix.X;
    camera->transform.up_direction = &camera->transform.rotation_matrix.Y;
    camera->transform.forward_direction = &camera->transform.rotation_matrix.Z;
    if (first_frame) {
        BVHBuilder builder;
        u32 leaves = scene->settings.primitives;
        for (u32 m = 0; m < scene->settings.meshes; m++)
            if (scene->meshes[m].triangle_count > leaves) leaves = scene->meshes[m].triangle_count;
        Memory memory;
        u64 bytes = (u64)getBVHBuilderMemorySize(scene, leaves ? leaves : 1) + 4096;
        void *block = calloc(1, bytes);
        if (!block) return -1;
        initMemory(&memory, (u8*)block, bytes);
        initBVHBuilder(&builder, scene, &memory);                     /* builder_top_down.h:42 */
        updateSceneBVH(scene, &builder);                              /* builder_top_down.h:366 */
        free(block);
        if (use_gpu) {
            int s = dropin_upload(scene);
            if (s != ST_OK) return s;
        }
    }
    updateSceneSSB(scene, viewport);
    beginDrawing(viewport);
    if (use_gpu) {
        int s = st_render_scene(g_st, 0, scene, viewport);            /* renderScene */
        if (s != ST_OK) return s;
    } else {
        if (scene->settings.meshes) viewport->trace.closest_mesh_hit.object_type = PrimitiveType_Mesh;
        u32 *scene_stack = (u32*)calloc(scene->settings.primitives * 2 + 64, sizeof(u32));
        u32 *mesh_stack = (u32*)calloc(256, sizeof(u32));
        viewport->trace.scene_stack = scene_stack;
        viewport->trace.mesh_stack = mesh_stack;
        viewport->trace.mesh_stack_size = 255;
        renderSceneOnCPU(scene, viewport);
        viewport->trace.scene_stack = NULL;
        viewport->trace.mesh_stack = NULL;
        free(scene_stack);
        free(mesh_stack);
    }
    if (viewport->frame_buffer->pixels) drawViewportToWindowContent(viewport);
    return 0;
}

void dropin_shutdown(void) {
    if (g_st) st_shutdown(g_st);
    g_st = NULL;
}
