// st_device.cuh — device-side layouts and float math of the tracing path.
//
// Layouts (all 16-byte aligned, read with 128-bit loads):
//   NodePair  64 B  both children of one BVH node: two AABBs + (first, count) each.  The reference
//                   stores children as adjacent BVHNode records (builder_top_down.h:172-174), so a
//                   traversal step that tests both (shaders/trace.h:26-29) reads one pair.
//   TriHot    64 B  what a ray/triangle test reads (intersection/mesh.h:5-18): position, normal,
//                   world_to_tangent.  The reference's 128-B Triangle stays resident for the
//                   per-hit interpolation (primitives.h:82-102).
//   PrimDev   64 B  what hitPrimitives needs per candidate (primitives.h:20-37, primitive.h:8):
//                   position, rotation, scale, 1/scale, flags/type/material/id.
//
// Arithmetic: every helper keeps the reference's operation order; the library is compiled with
// --fmad=false so nothing is contracted, and division/sqrt are IEEE (no fast-math), which makes
// results bit-identical to the reference wherever libm is not involved (powf/acosf differ by ulps).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "slimtracin_types.h"

namespace st {

typedef uint32_t u32t;

constexpr int kStack = 64;   // traversal stack entries; uploads and builds refuse BVHs with height + 2 > kStack
constexpr unsigned kNoPair = 0xFFFFFFFFu;   // "no node pair": the walk has nothing left to visit
enum Counter { C_PRIMARY = 0, C_SHADOW, C_BOUNCE, C_AABB, C_TRI, C_PRIM, C_LEAF, C_SHADE, C_TEXEL, C_MESH, C_TEXEL_MIP, C_COUNT };
enum Status { S_STACK_OVERFLOW = 1 };

struct __align__(16) NodePair {
    float4 a;  // lmin.x lmin.y lmin.z lmax.x
    float4 b;  // lmax.y lmax.z rmin.x rmin.y
    float4 c;  // rmin.z rmax.x rmax.y rmax.z
    uint4 d;   // l.first l.count r.first r.count   (count==0: first = child pair index)
};

struct __align__(16) TriHot {
    float4 p;  // position.xyz normal.x
    float4 q;  // normal.yz  w2t.X.x w2t.X.y
    float4 r;  // w2t.X.z w2t.Y.xyz
    float4 s;  // w2t.Z.xyz pad
};

struct __align__(16) PrimDev {
    float4 pos_bits;  // position.xyz, (flags | type << 8 | material << 16) as bits
    float4 rot;       // rotation axis.xyz, amount
    float4 scale_id;  // scale.xyz, id as bits
    float4 inv_scale; // 1/scale .xyz (IEEE division, identical to oneOverVec3), pad
};

struct MeshDev {
    u32t pair_offset;      // into the concatenated NodePair array
    u32t tri_offset;       // into the concatenated TriHot / Triangle arrays
    u32t triangle_count;
    u32t root_count;       // child_count of node 0 (0: internal root)
    u32t root_first;       // first_child_id of node 0
    u32t normals_count, uvs_count, height;
    float aabb[6];         // root node AABB (bvh.nodes[0].aabb)
    float mesh_aabb[6];    // Mesh.aabb (for the TLAS leaf boxes and SSB radius)
};

struct TexDev {
    uint16_t width, height;
    uint8_t mip_count, wrap, mipmap, pad;
    u32t mip_offset;       // into the MipDev table
};

struct MipDev {
    uint16_t width, height;
    u32t quad_offset;      // into the concatenated TexelQuad array
};

// Everything a render reads about one resident scene.
struct SceneDev {
    const PrimDev *prims;
    const Primitive *prims_raw;
    u32t n_prims;
    const Material *materials;
    const Light *lights;           // null when the scene has none (scene->lights == null)
    u32t n_lights;
    vec3 ambient;
    const NodePair *tlas_pairs;
    const u32t *tlas_leaf_ids;
    u32t tlas_root_count, tlas_root_first;
    float tlas_root_aabb[6];
    const MeshDev *meshes;
    const NodePair *mesh_pairs;
    const TriHot *tri_hot;
    const Triangle *tri_full;
    const TexDev *textures;
    const MipDev *mips;
    const TexelQuad *quads;
    const u32t *emissive_quads;    // primitive indices of emissive quads, increasing
    u32t n_emissive;
    const u32t *occluders;         // primitive indices of spheres and quads, increasing
    u32t n_occluders;
};

// ---- float3 math in the reference's operation order ------------------------------------------
struct v3 { float x, y, z; };
__device__ __forceinline__ v3 V(float x, float y, float z) { v3 o; o.x = x; o.y = y; o.z = z; return o; }
__device__ __forceinline__ v3 splat(float f) { return V(f, f, f); }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 vmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ v3 vscale(v3 a, float f) { return V(a.x * f, a.y * f, a.z * f); }
// scaleAddVec3 (math/vec3.h:183): v*f + c, unfused
__device__ __forceinline__ v3 vsfma(v3 v, float f, v3 c) { return V(v.x * f + c.x, v.y * f + c.y, v.z * f + c.z); }
// mulAddVec3 (math/vec3.h:173)
__device__ __forceinline__ v3 vvfma(v3 v, v3 f, v3 c) { return V(v.x * f.x + c.x, v.y * f.y + c.y, v.z * f.z + c.z); }
__device__ __forceinline__ float dot(v3 a, v3 b) { return ((a.x * b.x) + (a.y * b.y)) + (a.z * b.z); }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return V((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
__device__ __forceinline__ float sqlen(v3 v) { return ((v.x * v.x) + (v.y * v.y)) + (v.z * v.z); }
__device__ __forceinline__ float len(v3 v) { return sqrtf(sqlen(v)); }
__device__ __forceinline__ v3 norm(v3 v) { return vscale(v, 1.0f / len(v)); }
__device__ __forceinline__ v3 rcp(v3 v) { return V(1.0f / v.x, 1.0f / v.y, 1.0f / v.z); }
__device__ __forceinline__ v3 neg(v3 v) { return V(-v.x, -v.y, -v.z); }
__device__ __forceinline__ v3 one_minus(v3 v) { return V(1.0f - v.x, 1.0f - v.y, 1.0f - v.z); }
__device__ __forceinline__ float clamp01(float v) { float m = v < 1.0f ? v : 1.0f; return m > 0.0f ? m : 0.0f; }
__device__ __forceinline__ float dot01(v3 a, v3 b) { return clamp01(dot(a, b)); }
__device__ __forceinline__ v3 from(vec3 a) { return V(a.x, a.y, a.z); }

struct q4 { v3 axis; float w; };
// mulVec3Quat (math/quat.h:25)
__device__ __forceinline__ v3 qrot(v3 v, q4 q) {
    v3 out = cross(q.axis, v);
    v3 qqv = cross(q.axis, out);
    out = vsfma(out, q.w, qqv);
    out = vsfma(out, 2.0f, v);
    return out;
}
__device__ __forceinline__ q4 conj(q4 q) { q4 o; o.axis = neg(q.axis); o.w = q.w; return o; }
// normQuat (math/quat.h:15)
__device__ __forceinline__ q4 qnorm(q4 q) {
    float f = 1.0f / sqrtf(q.axis.x * q.axis.x + q.axis.y * q.axis.y + q.axis.z * q.axis.z + q.w * q.w);
    q4 o;
    o.axis = vscale(q.axis, f);
    o.w = q.w * f;
    return o;
}
// mulVec3Mat3 (math/vec3.h:203); m is 9 floats X.xyz Y.xyz Z.xyz
__device__ __forceinline__ v3 vmat3(v3 in, const float *m) {
    return V(in.x * m[0] + in.y * m[3] + in.z * m[6],
             in.x * m[1] + in.y * m[4] + in.z * m[7],
             in.x * m[2] + in.y * m[5] + in.z * m[8]);
}

__device__ __forceinline__ unsigned prim_flags(const PrimDev &p) { return __float_as_uint(p.pos_bits.w) & 0xFFu; }
__device__ __forceinline__ unsigned prim_type(const PrimDev &p) { return (__float_as_uint(p.pos_bits.w) >> 8) & 0xFFu; }
__device__ __forceinline__ unsigned prim_material(const PrimDev &p) { return __float_as_uint(p.pos_bits.w) >> 16; }

}  // namespace st
