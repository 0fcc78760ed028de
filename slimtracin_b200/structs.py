"""ctypes / numpy mirrors of the SlimTracin data contract (include/slimtracin_types.h).

Every struct here has the reference's name, field order and 32-bit-u32 layout
(core/types.h:56-374, core/base.h:193-365).  Element arrays that the tracing path reads in bulk
(Primitive, Material, Light, Triangle, BVHNode, TexelQuad, FloatPixel, Pixel) also get numpy
structured dtypes with the same byte layout, so scene generators can fill them vectorised and
hand the buffers to the C ABI without copies.
"""
import ctypes as C

import numpy as np

u8, u16, u32, i32, f32, f64, u64 = (C.c_uint8, C.c_uint16, C.c_uint32, C.c_int32, C.c_float,
                                    C.c_double, C.c_uint64)
cbool = C.c_uint8


class vec2i(C.Structure):
    _fields_ = [("x", i32), ("y", i32)]


class vec2(C.Structure):
    _fields_ = [("x", f32), ("y", f32)]


class vec3(C.Structure):
    _fields_ = [("x", f32), ("y", f32), ("z", f32)]


class vec4(C.Structure):
    _fields_ = [("x", f32), ("y", f32), ("z", f32), ("w", f32)]


class u8_3(C.Structure):
    _fields_ = [("x", u8), ("y", u8), ("z", u8)]


class mat3(C.Structure):
    _fields_ = [("X", vec3), ("Y", vec3), ("Z", vec3)]


class mat4(C.Structure):
    _fields_ = [("X", vec4), ("Y", vec4), ("Z", vec4), ("W", vec4)]


class AABB(C.Structure):
    _fields_ = [("min", vec3), ("max", vec3)]


class quat(C.Structure):
    _fields_ = [("axis", vec3), ("amount", f32)]


class Edge(C.Structure):
    _fields_ = [("from_", vec3), ("to", vec3)]


class Rect(C.Structure):
    _fields_ = [("min", vec2i), ("max", vec2i)]


class FloatPixel(C.Structure):
    _fields_ = [("color", vec3), ("opacity", f32), ("depth", f64)]


class Dimensions(C.Structure):
    _fields_ = [("width", u16), ("height", u16), ("width_times_height", u32),
                ("height_over_width", f32), ("width_over_height", f32), ("f_height", f32),
                ("f_width", f32), ("h_height", f32), ("h_width", f32)]


class PixelGrid(C.Structure):
    _fields_ = [("dimensions", Dimensions), ("pixels", C.c_void_p), ("float_pixels", C.c_void_p),
                ("QCAA", cbool)]


class String(C.Structure):
    _fields_ = [("length", u32), ("char_ptr", C.c_char_p)]


class HUD(C.Structure):
    _fields_ = [("position", vec2i), ("line_count", u32), ("line_height", f32), ("lines", C.c_void_p)]


class TextureMip(C.Structure):
    _fields_ = [("width", u16), ("height", u16), ("texel_quads", C.c_void_p)]


class Texture(C.Structure):
    _fields_ = [("width", u16), ("height", u16), ("mip_count", u8), ("wrap", cbool),
                ("mipmap", cbool), ("mips", C.POINTER(TextureMip))]


class Box(C.Structure):
    _fields_ = [("vertices", vec3 * 8), ("edges", Edge * 12)]


class Primitive(C.Structure):
    _fields_ = [("screen_bounds", Rect), ("rotation", quat), ("position", vec3), ("scale", vec3),
                ("id", u32), ("type", C.c_int), ("color", C.c_int), ("flags", u8),
                ("material_id", u8)]


class xform3(C.Structure):
    _fields_ = [("matrix", mat3), ("yaw_matrix", mat3), ("pitch_matrix", mat3),
                ("roll_matrix", mat3), ("rotation_matrix", mat3),
                ("rotation_matrix_inverted", mat3), ("rotation", quat),
                ("rotation_inverted", quat), ("position", vec3), ("scale", vec3),
                ("up_direction", C.POINTER(vec3)), ("right_direction", C.POINTER(vec3)),
                ("forward_direction", C.POINTER(vec3))]


class Camera(C.Structure):
    _fields_ = [("focal_length", f32), ("transform", xform3), ("current_velocity", vec3),
                ("zoom", f32), ("dolly", f32), ("target_distance", f32)]


class SphereHit(C.Structure):
    _fields_ = [(n, f32) for n in ("b", "c", "t_near", "t_far", "furthest",
                                   "closest_hit_distance", "closest_hit_density")]


class Ray(C.Structure):
    _fields_ = [("origin", vec3), ("scaled_origin", vec3), ("direction", vec3),
                ("direction_reciprocal", vec3), ("octant", u8_3)]


class RayHit(C.Structure):
    _fields_ = [("position", vec3), ("normal", vec3), ("uv", vec2), ("dUV", vec2),
                ("distance", f32), ("distance_squared", f32), ("cone_angle", f32),
                ("cone_width", f32), ("NdotV", f32), ("area", f32), ("uv_area", f32),
                ("material_id", u32), ("object_id", u32), ("object_type", u32),
                ("from_behind", cbool)]


class Trace(C.Structure):
    _fields_ = [("sphere_hit", SphereHit), ("closest_hit", RayHit), ("closest_mesh_hit", RayHit),
                ("current_hit", RayHit), ("quad_light_hits", C.c_void_p),
                ("local_space_ray", Ray), ("scene_stack", C.c_void_p), ("mesh_stack", C.c_void_p),
                ("depth", u8), ("mesh_stack_size", u8), ("scene_stack_size", u8)]


class BVHNode(C.Structure):
    _fields_ = [("aabb", AABB), ("first_child_id", u32), ("child_count", u16), ("depth", u16)]


class BVH(C.Structure):
    _fields_ = [("node_count", u32), ("height", u32), ("leaf_ids", C.c_void_p),
                ("nodes", C.c_void_p)]


class NavigationSettings(C.Structure):
    _fields_ = [(n, f32) for n in ("turn", "zoom", "dolly", "pan", "orbit", "orient",
                                   "max_velocity", "acceleration")]


class Navigation(C.Structure):
    _fields_ = [("settings", NavigationSettings), ("move", cbool * 6), ("turn", cbool * 2),
                ("zoomed", cbool), ("moved", cbool), ("turned", cbool)]


class ProjectionPlane(C.Structure):
    _fields_ = [("start", vec3), ("right", vec3), ("down", vec3), ("cone_angle", f32)]


class ViewportSettings(C.Structure):
    _fields_ = [("background_color", vec3), ("position", vec2i),
                ("near_clipping_plane_distance", f32), ("far_clipping_plane_distance", f32),
                ("background_opacity", f32), ("hud_line_count", u32), ("hud_lines", C.c_void_p),
                ("hud_default_color", C.c_int), ("render_mode", C.c_int),
                ("show_hud", cbool), ("show_wire_frame", cbool), ("antialias", cbool),
                ("use_cube_NDC", cbool), ("flip_z", cbool), ("show_BVH", cbool),
                ("show_SSB", cbool), ("show_selection", cbool), ("background_fill", cbool),
                ("use_GPU", cbool)]


class Viewport(C.Structure):
    _fields_ = [("settings", ViewportSettings), ("navigation", Navigation),
                ("projection_plane", ProjectionPlane), ("hud", HUD),
                ("camera", C.POINTER(Camera)), ("frame_buffer", C.POINTER(PixelGrid)),
                ("trace", Trace), ("default_box", Box), ("position", vec2i),
                ("projection_matrix", mat4)]


class Triangle(C.Structure):
    _fields_ = [("world_to_tangent", mat3), ("position", vec3), ("normal", vec3),
                ("vertex_normals", vec3 * 3), ("uvs", vec2 * 3),
                ("area_of_parallelogram", f32), ("area_of_uv", f32)]


class Mesh(C.Structure):
    _fields_ = [("aabb", AABB), ("triangle_count", u32), ("vertex_count", u32),
                ("edge_count", u32), ("normals_count", u32), ("uvs_count", u32),
                ("vertex_positions", C.c_void_p), ("vertex_normals", C.c_void_p),
                ("vertex_uvs", C.c_void_p), ("vertex_position_indices", C.c_void_p),
                ("vertex_normal_indices", C.c_void_p), ("vertex_uvs_indices", C.c_void_p),
                ("edge_vertex_indices", C.c_void_p), ("triangles", C.c_void_p), ("bvh", BVH)]


class Light(C.Structure):
    _fields_ = [("attenuation", vec3), ("position_or_direction", vec3), ("color", vec3),
                ("intensity", f32), ("is_directional", cbool)]


class Material(C.Structure):
    _fields_ = [("albedo", vec3), ("reflectivity", vec3), ("emission", vec3), ("uv_repeat", vec2),
                ("metallic", f32), ("roughness", f32), ("n1_over_n2", f32), ("n2_over_n1", f32),
                ("is_", u8), ("use", u8), ("texture_count", u8), ("texture_ids", u8 * 16),
                ("brdf", C.c_int)]


class SceneSettings(C.Structure):
    _fields_ = [(n, u32) for n in ("cameras", "primitives", "meshes", "materials", "lights",
                                   "area_lights", "textures")] + \
               [("file", String), ("mesh_files", C.c_void_p), ("texture_files", C.c_void_p)]


class Scene(C.Structure):
    _fields_ = [("settings", SceneSettings), ("selection", C.c_void_p), ("bvh", BVH),
                ("textures", C.c_void_p), ("cameras", C.c_void_p), ("ambient_light", vec3),
                ("lights", C.c_void_p), ("area_lights", C.c_void_p), ("materials", C.c_void_p),
                ("primitives", C.c_void_p), ("meshes", C.c_void_p),
                ("mesh_bvh_node_counts", C.c_void_p), ("mesh_triangle_counts", C.c_void_p),
                ("last_io_ticks", u64), ("last_io_is_save", cbool)]


# --- numpy dtypes (byte-identical to the structs above) ------------------------------------------
V3 = (np.float32, 3)
PRIMITIVE_DT = np.dtype({
    "names": ["screen_bounds", "rotation", "position", "scale", "id", "type", "color", "flags",
              "material_id"],
    "formats": [(np.int32, 4), (np.float32, 4), V3, V3, np.uint32, np.int32, np.int32, np.uint8,
                np.uint8],
    "offsets": [0, 16, 32, 44, 56, 60, 64, 68, 69], "itemsize": 72})
BVHNODE_DT = np.dtype({
    "names": ["aabb", "first_child_id", "child_count", "depth"],
    "formats": [(np.float32, 6), np.uint32, np.uint16, np.uint16],
    "offsets": [0, 24, 28, 30], "itemsize": 32})
TRIANGLE_DT = np.dtype({
    "names": ["world_to_tangent", "position", "normal", "vertex_normals", "uvs",
              "area_of_parallelogram", "area_of_uv"],
    "formats": [(np.float32, 9), V3, V3, (np.float32, 9), (np.float32, 6), np.float32, np.float32],
    "offsets": [0, 36, 48, 60, 96, 120, 124], "itemsize": 128})
MATERIAL_DT = np.dtype({
    "names": ["albedo", "reflectivity", "emission", "uv_repeat", "metallic", "roughness",
              "n1_over_n2", "n2_over_n1", "is_", "use", "texture_count", "texture_ids", "brdf"],
    "formats": [V3, V3, V3, (np.float32, 2), np.float32, np.float32, np.float32, np.float32,
                np.uint8, np.uint8, np.uint8, (np.uint8, 16), np.int32],
    "offsets": [0, 12, 24, 36, 44, 48, 52, 56, 60, 61, 62, 63, 80], "itemsize": 84})
LIGHT_DT = np.dtype({
    "names": ["attenuation", "position_or_direction", "color", "intensity", "is_directional"],
    "formats": [V3, V3, V3, np.float32, np.uint8],
    "offsets": [0, 12, 24, 36, 40], "itemsize": 44})
TEXELQUAD_DT = np.dtype([("R", np.uint8, 4), ("G", np.uint8, 4), ("B", np.uint8, 4)])
FLOATPIXEL_DT = np.dtype({"names": ["color", "opacity", "depth"],
                          "formats": [V3, np.float32, np.float64],
                          "offsets": [0, 12, 16], "itemsize": 24})
PIXEL_DT = np.dtype([("B", np.uint8), ("G", np.uint8), ("R", np.uint8), ("A", np.uint8)])

for _dt, _st in ((PRIMITIVE_DT, Primitive), (BVHNODE_DT, BVHNode), (TRIANGLE_DT, Triangle),
                 (MATERIAL_DT, Material), (LIGHT_DT, Light), (FLOATPIXEL_DT, FloatPixel)):
    assert _dt.itemsize == C.sizeof(_st), (_dt, _st)

# enum values (core/types.h:127-142, 313-318) and flags (core/base.h:130-160)
PT_NONE, PT_MESH, PT_BOX, PT_TETRAHEDRON, PT_QUAD, PT_SPHERE, PT_LIGHT = range(7)
RM_NORMALS, RM_BEAUTY, RM_DEPTH, RM_UVS = range(4)
BRDF_LAMBERT, BRDF_PHONG, BRDF_BLINN, BRDF_COOK_TORRANCE = range(4)
IS_VISIBLE, IS_TRANSLATED, IS_ROTATED, IS_SCALED = 1, 2, 4, 8
IS_SCALED_NON_UNIFORMLY, IS_SHADOWING, IS_TRANSPARENT = 16, 32, 64
ALL_FLAGS = 1 | 2 | 4 | 8 | 16 | 32
REFLECTIVE, REFRACTIVE, EMISSIVE = 1, 2, 4
ALBEDO_MAP, NORMAL_MAP = 1, 2
IOR_AIR = np.float32(1.0003)
IOR_GLASS = np.float32(1.52)

STRUCTS = {c.__name__: c for c in (Primitive, BVHNode, Triangle, Material, Light, FloatPixel,
                                   Scene, Viewport, Camera, Mesh, Texture, TextureMip, Trace,
                                   RayHit, Ray, xform3, BVH, Navigation, ProjectionPlane,
                                   ViewportSettings, SceneSettings, PixelGrid, Dimensions, HUD)}
