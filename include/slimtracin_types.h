/*
 * slimtracin_types.h — the scene/camera/primitive/material/texture data contract of SlimTracin,
 * restated with the reference's own type names and field order so that a SlimTracin host can pass
 * its structs to libslimtracin_b200 unchanged.
 *
 * Layout.  The reference targets Win32, where `unsigned long` is 32 bits, so its `u32`/`i32`
 * (core/base.h:95,98) are 32-bit there.  This header fixes that layout on every platform:
 * u32 = uint32_t, i32 = int32_t, pointers native.  A Linux build of the reference is
 * layout-compatible when it is compiled with 32-bit u32/i32 (for instance by `#define long` empty
 * around the reference's includes, after the system headers); the sizes below are asserted at
 * compile time and exported at run time by st_layout_query().
 *
 * Source of every struct: core/base.h:93-365,742-753 and core/types.h:56-374 of the reference.
 * Unions with aliased member names in the reference (vec2/vec3/vec4/mat3) are written here as plain
 * structs with the first member set (x,y,z,w / X,Y,Z); their size and field offsets are identical.
 *
 * A translation unit that already has the reference's own types in scope (a patched reference
 * build) defines SLIMTRACIN_REFERENCE_TYPES before including slimtracin_b200.h; this file is then
 * skipped and only the entry points are declared.
 */
#ifndef SLIMTRACIN_TYPES_H
#define SLIMTRACIN_TYPES_H

#ifndef SLIMTRACIN_REFERENCE_TYPES

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint8_t  u8;
typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;
typedef int16_t  i16;
typedef int32_t  i32;
typedef float    f32;
typedef double   f64;

#if !defined(__cplusplus) && !defined(bool)
typedef unsigned char bool;
#endif

/* core/base.h:193-208 */
typedef struct u8_3  { u8 x, y, z; } u8_3;
typedef struct vec2i { i32 x, y; } vec2i;
typedef struct vec2u { u32 x, y; } vec2u;
typedef struct vec2  { f32 x, y; } vec2;
typedef struct vec3  { f32 x, y, z; } vec3;
typedef struct vec4  { f32 x, y, z, w; } vec4;
typedef struct mat2  { vec2 X, Y; } mat2;
typedef struct mat3  { vec3 X, Y, Z; } mat3;
typedef struct mat4  { vec4 X, Y, Z, W; } mat4;
typedef struct AABB  { vec3 min, max; } AABB;
typedef struct quat  { vec3 axis; f32 amount; } quat;
typedef struct Edge  { vec3 from, to; } Edge;
typedef struct Rect  { vec2i min, max; } Rect;
typedef struct RGBA  { u8 B, G, R, A; } RGBA;
typedef struct FloatPixel { vec3 color; f32 opacity; f64 depth; } FloatPixel;
typedef union  Pixel { RGBA color; u32 value; } Pixel;

/* core/base.h:335-365 */
typedef struct Dimensions {
    u16 width, height;
    u32 width_times_height;
    f32 height_over_width, width_over_height, f_height, f_width, h_height, h_width;
} Dimensions;

typedef struct PixelGrid {
    Dimensions dimensions;
    Pixel *pixels;
    FloatPixel *float_pixels;
    bool QCAA;
} PixelGrid;

/* core/base.h:413 (only the enum's width matters to the contract) */
enum ColorID { Black, White, Grey, Red, Green, Blue, Cyan, Magenta, Yellow, DarkRed, DarkGreen,
               DarkBlue, DarkGrey, BrightRed, BrightGreen, BrightBlue, BrightGrey, BrightCyan,
               BrightMagenta, BrightYellow, DarkCyan, DarkMagenta, DarkYellow };

/* core/base.h:729-753 */
typedef struct String { u32 length; char *char_ptr; } String;
typedef struct NumberString { char _buffer[13]; String string; } NumberString;
typedef struct HUDLine {
    String title, alternate_value;
    NumberString value;
    enum ColorID title_color, value_color, alternate_value_color;
    bool invert_alternate_use, *use_alternate;
} HUDLine;
typedef struct HUD {
    vec2i position;
    u32 line_count;
    f32 line_height;
    HUDLine *lines;
} HUD;

/* core/types.h:56-74 — texture residency format (bmp2texture.c:324-364 writes it) */
typedef struct TexelQuadComponent { u8 TL, TR, BL, BR; } TexelQuadComponent;
typedef struct TexelQuad { TexelQuadComponent R, G, B; } TexelQuad;
typedef struct TextureMip { u16 width, height; TexelQuad *texel_quads; } TextureMip;
typedef struct Texture {
    u16 width, height;
    u8 mip_count;
    bool wrap, mipmap;
    TextureMip *mips;
} Texture;

/* core/types.h:76-125 */
typedef enum BoxSide { NoSide = 0, Top = 1, Bottom = 2, Left = 4, Right = 8, Front = 16, Back = 32 } BoxSide;
typedef struct BoxCorners {
    vec3 front_top_left, front_top_right, front_bottom_left, front_bottom_right,
         back_top_left, back_top_right, back_bottom_left, back_bottom_right;
} BoxCorners;
typedef union BoxVertices { BoxCorners corners; vec3 buffer[8]; } BoxVertices;
typedef struct BoxEdgeSides {
    Edge front_top, front_bottom, front_left, front_right, back_top, back_bottom, back_left,
         back_right, left_bottom, left_top, right_bottom, right_top;
} BoxEdgeSides;
typedef union BoxEdges { BoxEdgeSides sides; Edge buffer[12]; } BoxEdges;
typedef struct Box { BoxVertices vertices; BoxEdges edges; } Box;

/* core/types.h:127-152 */
enum PrimitiveType {
    PrimitiveType_None = 0,
    PrimitiveType_Mesh,
    PrimitiveType_Box,
    PrimitiveType_Tetrahedron,
    PrimitiveType_Quad,
    PrimitiveType_Sphere,
    PrimitiveType_Light
};
enum RenderMode { RenderMode_Normals, RenderMode_Beauty, RenderMode_Depth, RenderMode_UVs };

typedef struct Primitive {
    Rect screen_bounds;
    quat rotation;
    vec3 position, scale;
    u32 id;
    enum PrimitiveType type;
    enum ColorID color;
    u8 flags, material_id;
} Primitive;

/* core/types.h:154-200 */
typedef struct xform3 {
    mat3 matrix, yaw_matrix, pitch_matrix, roll_matrix, rotation_matrix, rotation_matrix_inverted;
    quat rotation, rotation_inverted;
    vec3 position, scale, *up_direction, *right_direction, *forward_direction;
} xform3;

typedef struct Camera {
    f32 focal_length;
    xform3 transform;
    vec3 current_velocity;
    f32 zoom, dolly, target_distance;
} Camera;

typedef struct SphereHit { f32 b, c, t_near, t_far, furthest, closest_hit_distance, closest_hit_density; } SphereHit;

typedef struct Ray {
    vec3 origin, scaled_origin, direction, direction_reciprocal;
    u8_3 octant;
} Ray;

typedef struct RayHit {
    vec3 position, normal;
    vec2 uv, dUV;
    f32 distance, distance_squared, cone_angle, cone_width, NdotV, area, uv_area;
    u32 material_id, object_id, object_type;
    bool from_behind;
} RayHit;

typedef struct Trace {
    SphereHit sphere_hit;
    RayHit closest_hit, closest_mesh_hit, current_hit, *quad_light_hits;
    Ray local_space_ray;
    u32 *scene_stack, *mesh_stack;
    u8 depth, mesh_stack_size, scene_stack_size;
} Trace;

/* core/types.h:202-213 */
typedef struct BVHNode {
    AABB aabb;
    u32 first_child_id;
    u16 child_count, depth;
} BVHNode;

typedef struct BVH {
    u32 node_count, height, *leaf_ids;
    BVHNode *nodes;
} BVH;

/* core/types.h:215-268 */
typedef struct NavigationSpeedSettings { f32 turn, zoom, dolly, pan, orbit, orient; } NavigationSpeedSettings;
typedef struct NavigationSettings { NavigationSpeedSettings speeds; f32 max_velocity, acceleration; } NavigationSettings;
typedef struct NavigationTurn { bool right, left; } NavigationTurn;
typedef struct NavigationMove { bool right, left, up, down, forward, backward; } NavigationMove;
typedef struct Navigation {
    NavigationSettings settings;
    NavigationMove move;
    NavigationTurn turn;
    bool zoomed, moved, turned;
} Navigation;

typedef struct ProjectionPlane { vec3 start, right, down; f32 cone_angle; } ProjectionPlane;

typedef struct ViewportSettings {
    vec3 background_color;
    vec2i position;
    f32 near_clipping_plane_distance, far_clipping_plane_distance, background_opacity;
    u32 hud_line_count;
    HUDLine *hud_lines;
    enum ColorID hud_default_color;
    enum RenderMode render_mode;
    bool show_hud, show_wire_frame, antialias, use_cube_NDC, flip_z, show_BVH, show_SSB,
         show_selection, background_fill, use_GPU;
} ViewportSettings;

typedef struct Viewport {
    ViewportSettings settings;
    Navigation navigation;
    ProjectionPlane projection_plane;
    HUD hud;
    Camera *camera;
    PixelGrid *frame_buffer;
    Trace trace;
    Box default_box;
    vec2i position;
    mat4 projection_matrix;
} Viewport;

/* core/types.h:270-292 */
typedef struct Triangle {
    mat3 world_to_tangent;
    vec3 position, normal;
    vec3 vertex_normals[3];
    vec2 uvs[3];
    f32 area_of_parallelogram, area_of_uv;
} Triangle;
typedef struct EdgeVertexIndices { u32 from, to; } EdgeVertexIndices;
typedef union TriangleVertexIndices { u32 ids[3]; struct { u32 v1, v2, v3; } v; } TriangleVertexIndices;
typedef struct Mesh {
    AABB aabb;
    u32 triangle_count, vertex_count, edge_count, normals_count, uvs_count;
    vec3 *vertex_positions, *vertex_normals;
    vec2 *vertex_uvs;
    TriangleVertexIndices *vertex_position_indices;
    TriangleVertexIndices *vertex_normal_indices;
    TriangleVertexIndices *vertex_uvs_indices;
    EdgeVertexIndices *edge_vertex_indices;
    Triangle *triangles;
    BVH bvh;
} Mesh;

/* core/types.h:294-326 */
typedef struct AmbientLight { vec3 color; } AmbientLight;
typedef struct Light {
    vec3 attenuation, position_or_direction, color;
    f32 intensity;
    bool is_directional;
} Light;
typedef struct AreaLight {
    vec3 position, normal, color, U, V, v1, v2, v3, v4;
    f32 A, u_length, v_length;
} AreaLight;

enum BRDF { BRDF_Lambert, BRDF_Phong, BRDF_Blinn, BRDF_CookTorrance };

typedef struct Material {
    vec3 albedo, reflectivity, emission;
    vec2 uv_repeat;
    f32 metallic, roughness, n1_over_n2, n2_over_n1;
    u8 is, use, texture_count, texture_ids[16];
    enum BRDF brdf;
} Material;

/* core/types.h:335-374 (Selection is only held by pointer here) */
struct Selection;
typedef struct SceneSettings {
    u32 cameras, primitives, meshes, materials, lights, area_lights, textures;
    String file, *mesh_files, *texture_files;
} SceneSettings;

typedef struct Scene {
    SceneSettings settings;
    struct Selection *selection;
    BVH bvh;
    Texture *textures;
    Camera *cameras;
    AmbientLight ambient_light;
    Light *lights;
    AreaLight *area_lights;
    Material *materials;
    Primitive *primitives;
    Mesh *meshes;
    u32 *mesh_bvh_node_counts, *mesh_triangle_counts;
    u64 last_io_ticks;
    bool last_io_is_save;
} Scene;

#ifdef __cplusplus
}
#define ST_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define ST_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

/* Sizes of the reference structs with 32-bit u32 (checked against the reference headers). */
ST_STATIC_ASSERT(sizeof(Primitive) == 72, "Primitive layout");
ST_STATIC_ASSERT(sizeof(BVHNode) == 32, "BVHNode layout");
ST_STATIC_ASSERT(sizeof(Triangle) == 128, "Triangle layout");
ST_STATIC_ASSERT(sizeof(Material) == 84, "Material layout");
ST_STATIC_ASSERT(sizeof(Light) == 44, "Light layout");
ST_STATIC_ASSERT(sizeof(FloatPixel) == 24, "FloatPixel layout");
ST_STATIC_ASSERT(sizeof(TexelQuad) == 12, "TexelQuad layout");
ST_STATIC_ASSERT(sizeof(Pixel) == 4, "Pixel layout");
ST_STATIC_ASSERT(sizeof(Scene) == 200, "Scene layout");
ST_STATIC_ASSERT(sizeof(Viewport) == 1024, "Viewport layout");
ST_STATIC_ASSERT(sizeof(Camera) == 328, "Camera layout");
ST_STATIC_ASSERT(sizeof(Mesh) == 136, "Mesh layout");
ST_STATIC_ASSERT(sizeof(Texture) == 16, "Texture layout");

/* Flag and constant values the data contract carries (core/base.h:107-173). */
#define IS_VISIBLE              ((u8)1)
#define IS_TRANSLATED           ((u8)2)
#define IS_ROTATED              ((u8)4)
#define IS_SCALED               ((u8)8)
#define IS_SCALED_NON_UNIFORMLY ((u8)16)
#define IS_SHADOWING            ((u8)32)
#define IS_TRANSPARENT          ((u8)64)
#define ALL_FLAGS (IS_VISIBLE | IS_TRANSLATED | IS_ROTATED | IS_SCALED | IS_SCALED_NON_UNIFORMLY | IS_SHADOWING)
#define REFLECTIVE 1
#define REFRACTIVE 2
#define EMISSIVE 4
#define TRANSPARENT_UV 8
#define ALBEDO_MAP 1
#define NORMAL_MAP 2
#define MAX_TRIANGLES_PER_MESH_BVH_NODE 4
#define MAX_OBJS_PER_SCENE_BVH_NODE 2
#define MAX_WIDTH 3840
#define MAX_HEIGHT 2160
#define IOR_AIR 1.0003f
#define IOR_GLASS 1.52f

#endif /* SLIMTRACIN_REFERENCE_TYPES */
#endif /* SLIMTRACIN_TYPES_H */
