/*
 * slimtracin_layout.h — X-macro list of the data-contract structs and fields whose size and offset
 * must equal the reference's (core/types.h with 32-bit u32).  st_layout_offsetof() answers from this
 * list; a test compares it with the same list evaluated against the reference's own headers.
 *
 *   ST_LAYOUT_STRUCT(type)         one entry per struct
 *   ST_LAYOUT_FIELD(type, field)   one entry per checked field
 */
#ifndef SLIMTRACIN_LAYOUT_H
#define SLIMTRACIN_LAYOUT_H

#define ST_LAYOUT_LIST(ST_LAYOUT_STRUCT, ST_LAYOUT_FIELD) \
    ST_LAYOUT_STRUCT(Primitive) \
    ST_LAYOUT_FIELD(Primitive, screen_bounds) \
    ST_LAYOUT_FIELD(Primitive, rotation) \
    ST_LAYOUT_FIELD(Primitive, position) \
    ST_LAYOUT_FIELD(Primitive, scale) \
    ST_LAYOUT_FIELD(Primitive, id) \
    ST_LAYOUT_FIELD(Primitive, type) \
    ST_LAYOUT_FIELD(Primitive, color) \
    ST_LAYOUT_FIELD(Primitive, flags) \
    ST_LAYOUT_FIELD(Primitive, material_id) \
    ST_LAYOUT_STRUCT(Camera) \
    ST_LAYOUT_FIELD(Camera, focal_length) \
    ST_LAYOUT_FIELD(Camera, transform) \
    ST_LAYOUT_FIELD(Camera, current_velocity) \
    ST_LAYOUT_FIELD(Camera, zoom) \
    ST_LAYOUT_FIELD(Camera, dolly) \
    ST_LAYOUT_FIELD(Camera, target_distance) \
    ST_LAYOUT_STRUCT(xform3) \
    ST_LAYOUT_FIELD(xform3, matrix) \
    ST_LAYOUT_FIELD(xform3, rotation_matrix) \
    ST_LAYOUT_FIELD(xform3, rotation_matrix_inverted) \
    ST_LAYOUT_FIELD(xform3, rotation) \
    ST_LAYOUT_FIELD(xform3, rotation_inverted) \
    ST_LAYOUT_FIELD(xform3, position) \
    ST_LAYOUT_FIELD(xform3, scale) \
    ST_LAYOUT_FIELD(xform3, up_direction) \
    ST_LAYOUT_FIELD(xform3, right_direction) \
    ST_LAYOUT_FIELD(xform3, forward_direction) \
    ST_LAYOUT_STRUCT(Ray) \
    ST_LAYOUT_FIELD(Ray, origin) \
    ST_LAYOUT_FIELD(Ray, scaled_origin) \
    ST_LAYOUT_FIELD(Ray, direction) \
    ST_LAYOUT_FIELD(Ray, direction_reciprocal) \
    ST_LAYOUT_FIELD(Ray, octant) \
    ST_LAYOUT_STRUCT(RayHit) \
    ST_LAYOUT_FIELD(RayHit, position) \
    ST_LAYOUT_FIELD(RayHit, normal) \
    ST_LAYOUT_FIELD(RayHit, uv) \
    ST_LAYOUT_FIELD(RayHit, dUV) \
    ST_LAYOUT_FIELD(RayHit, distance) \
    ST_LAYOUT_FIELD(RayHit, distance_squared) \
    ST_LAYOUT_FIELD(RayHit, cone_angle) \
    ST_LAYOUT_FIELD(RayHit, cone_width) \
    ST_LAYOUT_FIELD(RayHit, NdotV) \
    ST_LAYOUT_FIELD(RayHit, area) \
    ST_LAYOUT_FIELD(RayHit, uv_area) \
    ST_LAYOUT_FIELD(RayHit, material_id) \
    ST_LAYOUT_FIELD(RayHit, object_id) \
    ST_LAYOUT_FIELD(RayHit, object_type) \
    ST_LAYOUT_FIELD(RayHit, from_behind) \
    ST_LAYOUT_STRUCT(Trace) \
    ST_LAYOUT_FIELD(Trace, sphere_hit) \
    ST_LAYOUT_FIELD(Trace, closest_hit) \
    ST_LAYOUT_FIELD(Trace, closest_mesh_hit) \
    ST_LAYOUT_FIELD(Trace, current_hit) \
    ST_LAYOUT_FIELD(Trace, quad_light_hits) \
    ST_LAYOUT_FIELD(Trace, local_space_ray) \
    ST_LAYOUT_FIELD(Trace, scene_stack) \
    ST_LAYOUT_FIELD(Trace, mesh_stack) \
    ST_LAYOUT_FIELD(Trace, depth) \
    ST_LAYOUT_FIELD(Trace, mesh_stack_size) \
    ST_LAYOUT_FIELD(Trace, scene_stack_size) \
    ST_LAYOUT_STRUCT(BVHNode) \
    ST_LAYOUT_FIELD(BVHNode, aabb) \
    ST_LAYOUT_FIELD(BVHNode, first_child_id) \
    ST_LAYOUT_FIELD(BVHNode, child_count) \
    ST_LAYOUT_FIELD(BVHNode, depth) \
    ST_LAYOUT_STRUCT(BVH) \
    ST_LAYOUT_FIELD(BVH, node_count) \
    ST_LAYOUT_FIELD(BVH, height) \
    ST_LAYOUT_FIELD(BVH, leaf_ids) \
    ST_LAYOUT_FIELD(BVH, nodes) \
    ST_LAYOUT_STRUCT(Navigation) \
    ST_LAYOUT_FIELD(Navigation, settings) \
    ST_LAYOUT_FIELD(Navigation, move) \
    ST_LAYOUT_FIELD(Navigation, turn) \
    ST_LAYOUT_FIELD(Navigation, zoomed) \
    ST_LAYOUT_FIELD(Navigation, moved) \
    ST_LAYOUT_FIELD(Navigation, turned) \
    ST_LAYOUT_STRUCT(ProjectionPlane) \
    ST_LAYOUT_FIELD(ProjectionPlane, start) \
    ST_LAYOUT_FIELD(ProjectionPlane, right) \
    ST_LAYOUT_FIELD(ProjectionPlane, down) \
    ST_LAYOUT_FIELD(ProjectionPlane, cone_angle) \
    ST_LAYOUT_STRUCT(ViewportSettings) \
    ST_LAYOUT_FIELD(ViewportSettings, background_color) \
    ST_LAYOUT_FIELD(ViewportSettings, position) \
    ST_LAYOUT_FIELD(ViewportSettings, near_clipping_plane_distance) \
    ST_LAYOUT_FIELD(ViewportSettings, far_clipping_plane_distance) \
    ST_LAYOUT_FIELD(ViewportSettings, background_opacity) \
    ST_LAYOUT_FIELD(ViewportSettings, hud_line_count) \
    ST_LAYOUT_FIELD(ViewportSettings, hud_lines) \
    ST_LAYOUT_FIELD(ViewportSettings, hud_default_color) \
    ST_LAYOUT_FIELD(ViewportSettings, render_mode) \
    ST_LAYOUT_FIELD(ViewportSettings, show_hud) \
    ST_LAYOUT_FIELD(ViewportSettings, use_GPU) \
    ST_LAYOUT_STRUCT(Viewport) \
    ST_LAYOUT_FIELD(Viewport, settings) \
    ST_LAYOUT_FIELD(Viewport, navigation) \
    ST_LAYOUT_FIELD(Viewport, projection_plane) \
    ST_LAYOUT_FIELD(Viewport, hud) \
    ST_LAYOUT_FIELD(Viewport, camera) \
    ST_LAYOUT_FIELD(Viewport, frame_buffer) \
    ST_LAYOUT_FIELD(Viewport, trace) \
    ST_LAYOUT_FIELD(Viewport, default_box) \
    ST_LAYOUT_FIELD(Viewport, position) \
    ST_LAYOUT_FIELD(Viewport, projection_matrix) \
    ST_LAYOUT_STRUCT(Triangle) \
    ST_LAYOUT_FIELD(Triangle, world_to_tangent) \
    ST_LAYOUT_FIELD(Triangle, position) \
    ST_LAYOUT_FIELD(Triangle, normal) \
    ST_LAYOUT_FIELD(Triangle, vertex_normals) \
    ST_LAYOUT_FIELD(Triangle, uvs) \
    ST_LAYOUT_FIELD(Triangle, area_of_parallelogram) \
    ST_LAYOUT_FIELD(Triangle, area_of_uv) \
    ST_LAYOUT_STRUCT(Mesh) \
    ST_LAYOUT_FIELD(Mesh, aabb) \
    ST_LAYOUT_FIELD(Mesh, triangle_count) \
    ST_LAYOUT_FIELD(Mesh, vertex_count) \
    ST_LAYOUT_FIELD(Mesh, edge_count) \
    ST_LAYOUT_FIELD(Mesh, normals_count) \
    ST_LAYOUT_FIELD(Mesh, uvs_count) \
    ST_LAYOUT_FIELD(Mesh, vertex_positions) \
    ST_LAYOUT_FIELD(Mesh, vertex_normals) \
    ST_LAYOUT_FIELD(Mesh, vertex_uvs) \
    ST_LAYOUT_FIELD(Mesh, vertex_position_indices) \
    ST_LAYOUT_FIELD(Mesh, vertex_normal_indices) \
    ST_LAYOUT_FIELD(Mesh, vertex_uvs_indices) \
    ST_LAYOUT_FIELD(Mesh, edge_vertex_indices) \
    ST_LAYOUT_FIELD(Mesh, triangles) \
    ST_LAYOUT_FIELD(Mesh, bvh) \
    ST_LAYOUT_STRUCT(Light) \
    ST_LAYOUT_FIELD(Light, attenuation) \
    ST_LAYOUT_FIELD(Light, position_or_direction) \
    ST_LAYOUT_FIELD(Light, color) \
    ST_LAYOUT_FIELD(Light, intensity) \
    ST_LAYOUT_FIELD(Light, is_directional) \
    ST_LAYOUT_STRUCT(Material) \
    ST_LAYOUT_FIELD(Material, albedo) \
    ST_LAYOUT_FIELD(Material, reflectivity) \
    ST_LAYOUT_FIELD(Material, emission) \
    ST_LAYOUT_FIELD(Material, uv_repeat) \
    ST_LAYOUT_FIELD(Material, metallic) \
    ST_LAYOUT_FIELD(Material, roughness) \
    ST_LAYOUT_FIELD(Material, n1_over_n2) \
    ST_LAYOUT_FIELD(Material, n2_over_n1) \
    ST_LAYOUT_FIELD(Material, is) \
    ST_LAYOUT_FIELD(Material, use) \
    ST_LAYOUT_FIELD(Material, texture_count) \
    ST_LAYOUT_FIELD(Material, texture_ids) \
    ST_LAYOUT_FIELD(Material, brdf) \
    ST_LAYOUT_STRUCT(SceneSettings) \
    ST_LAYOUT_FIELD(SceneSettings, cameras) \
    ST_LAYOUT_FIELD(SceneSettings, primitives) \
    ST_LAYOUT_FIELD(SceneSettings, meshes) \
    ST_LAYOUT_FIELD(SceneSettings, materials) \
    ST_LAYOUT_FIELD(SceneSettings, lights) \
    ST_LAYOUT_FIELD(SceneSettings, area_lights) \
    ST_LAYOUT_FIELD(SceneSettings, textures) \
    ST_LAYOUT_FIELD(SceneSettings, file) \
    ST_LAYOUT_FIELD(SceneSettings, mesh_files) \
    ST_LAYOUT_FIELD(SceneSettings, texture_files) \
    ST_LAYOUT_STRUCT(Scene) \
    ST_LAYOUT_FIELD(Scene, settings) \
    ST_LAYOUT_FIELD(Scene, selection) \
    ST_LAYOUT_FIELD(Scene, bvh) \
    ST_LAYOUT_FIELD(Scene, textures) \
    ST_LAYOUT_FIELD(Scene, cameras) \
    ST_LAYOUT_FIELD(Scene, ambient_light) \
    ST_LAYOUT_FIELD(Scene, lights) \
    ST_LAYOUT_FIELD(Scene, area_lights) \
    ST_LAYOUT_FIELD(Scene, materials) \
    ST_LAYOUT_FIELD(Scene, primitives) \
    ST_LAYOUT_FIELD(Scene, meshes) \
    ST_LAYOUT_FIELD(Scene, mesh_bvh_node_counts) \
    ST_LAYOUT_FIELD(Scene, mesh_triangle_counts) \
    ST_LAYOUT_FIELD(Scene, last_io_ticks) \
    ST_LAYOUT_FIELD(Scene, last_io_is_save) \
    ST_LAYOUT_STRUCT(Texture) \
    ST_LAYOUT_FIELD(Texture, width) \
    ST_LAYOUT_FIELD(Texture, height) \
    ST_LAYOUT_FIELD(Texture, mip_count) \
    ST_LAYOUT_FIELD(Texture, wrap) \
    ST_LAYOUT_FIELD(Texture, mipmap) \
    ST_LAYOUT_FIELD(Texture, mips) \
    ST_LAYOUT_STRUCT(TextureMip) \
    ST_LAYOUT_FIELD(TextureMip, width) \
    ST_LAYOUT_FIELD(TextureMip, height) \
    ST_LAYOUT_FIELD(TextureMip, texel_quads) \
    ST_LAYOUT_STRUCT(PixelGrid) \
    ST_LAYOUT_FIELD(PixelGrid, dimensions) \
    ST_LAYOUT_FIELD(PixelGrid, pixels) \
    ST_LAYOUT_FIELD(PixelGrid, float_pixels) \
    ST_LAYOUT_FIELD(PixelGrid, QCAA) \
    ST_LAYOUT_STRUCT(Dimensions) \
    ST_LAYOUT_FIELD(Dimensions, width) \
    ST_LAYOUT_FIELD(Dimensions, height) \
    ST_LAYOUT_FIELD(Dimensions, width_times_height) \
    ST_LAYOUT_FIELD(Dimensions, height_over_width) \
    ST_LAYOUT_FIELD(Dimensions, f_height) \
    ST_LAYOUT_FIELD(Dimensions, h_width) \
    ST_LAYOUT_STRUCT(HUD) \
    ST_LAYOUT_FIELD(HUD, position) \
    ST_LAYOUT_FIELD(HUD, line_count) \
    ST_LAYOUT_FIELD(HUD, line_height) \
    ST_LAYOUT_FIELD(HUD, lines) \
    ST_LAYOUT_STRUCT(FloatPixel) \
    ST_LAYOUT_FIELD(FloatPixel, color) \
    ST_LAYOUT_FIELD(FloatPixel, opacity) \
    ST_LAYOUT_FIELD(FloatPixel, depth)

#endif /* SLIMTRACIN_LAYOUT_H */
