// st_trace.cuh — the per-ray tracing and shading functions of the device path.
//
// Each function restates one reference function (file:line given) on the device layouts of
// st_device.cuh.  The per-ray scratch TState mirrors the reference's Trace (core/types.h:193):
// shading overwrites `closest` with light data and shadow-ray hits exactly as the reference does
// (closest_hit/surface.h:14-17, intersection/primitives.h:63-77), because later steps read it back
// (surface.h:55) and the beauty output depends on that sequence.
#pragma once
#include "st_device.cuh"

namespace st {

constexpr float kTraceOffset = 0.0001f;            // TRACE_OFFSET core/base.h:161
constexpr float kEps = 0.0001f;                    // EPS core/base.h:107
constexpr float kPi = 3.14159265f;
constexpr float kOneOverPi = 1.0f / kPi;
constexpr float kSqrt2 = 1.41421356237f;
constexpr float kSqrt3 = 1.73205080757f;
constexpr float kUnitSphereAreaOverSix = (4.0f * kPi) / 6.0f;
constexpr float kColorToFloat = 0.00392156862f;
constexpr float kT0577 = 0.577350259f;
constexpr float kT0288 = 0.288675159f;

struct Hit {                                        // RayHit core/types.h:185
    v3 position, normal;
    float u, v;
    float distance, distance_squared, cone_width, NdotV, area, uv_area;
    u32t material_id, object_id, object_type;
    bool from_behind;
};

struct RayD {                                       // Ray core/types.h:180
    v3 origin, direction, rcp, scaled_origin;
    bool ox, oy, oz;                                // octant == 3 per axis
};

struct SphereHitD { float b, c, t_near, t_far, furthest, closest_distance; };

// Threads per block of the kernels that trace (the stride of the shared-memory stack columns).
constexpr u32t kTraceBlock = 128;

// What the walks read of the closest hit found so far (the reference's trace->closest_hit during
// traceScene/hitPrimitives): its distance (the hit test's own distance until the hitPrimitives call
// that found it ends, then the world distance), squared world distance and world position, and which
// primitive and triangle it is.  The walks carry only these; the full record (normal, uv, areas ...)
// is rebuilt once the walk is over (finalize_hit), from the same inputs and with the same arithmetic,
// so that a lane's nested walks keep few values live.
struct Best {
    float distance, distance_squared;
    v3 position;
    u32t prim;                        // the winning primitive
    u32t tri;                         // meshes: the winning triangle's slot in the mesh's leaf order
};

// SHS: entries of each traversal stack kept in shared memory (the block's stack columns, one per
// thread, entry-major so that a warp's pushes hit distinct banks); the rest live in local memory.
// Where the entries live changes no traversal step.
template <bool CNT, int SHS = 0>
struct TState {
    Hit closest;                      // the finalized closest hit, as shading reads it
    Best best;                        // the walk's view of it (above)
    float mesh_distance;              // the BLAS walk's closest triangle so far (trace->closest_mesh_hit):
    u32t mesh_tri;                    //   its distance along the object-space ray, and its slot
    SphereHitD sphere;
    RayD local;
    u32t depth;
    unsigned status;
    unsigned cnt[CNT ? C_COUNT : 1];
    u32t scene_local[kStack - SHS];   // the TLAS walk (the reference's trace->scene_stack, trace.h:22)
    u32t mesh_local[kStack - SHS];    // the BLAS walk nested inside it (trace->mesh_stack, mesh.h:42)
    u32t *sh;                         // SHS > 0: this thread's column, 2 * SHS entries kTraceBlock apart
    __device__ __forceinline__ void count(int k, unsigned n = 1) { if (CNT) cnt[k] += n; }
    __device__ __forceinline__ void push(bool mesh, u32t i, u32t v) {
        if (SHS > 0 && i < (u32t)SHS) sh[((mesh ? SHS : 0) + i) * kTraceBlock] = v;
        else if (mesh) mesh_local[i - SHS] = v;
        else scene_local[i - SHS] = v;
    }
    __device__ __forceinline__ u32t at(bool mesh, u32t i) const {
        if (SHS > 0 && i < (u32t)SHS) return sh[((mesh ? SHS : 0) + i) * kTraceBlock];
        return mesh ? mesh_local[i - SHS] : scene_local[i - SHS];
    }
};

// A ray that does not move along an axis (a zero direction component, or one so small that
// -origin * rcp overflows) makes hitAABB compute inf - inf = NaN on that axis.  Its min/max chain
// then drops the NaN together with a neighbouring axis, the ray accepts boxes nowhere near it and
// walks nearly every node of a BVH: one such ray through a 1.3M-triangle BLAS made hundreds of
// thousands of box and triangle tests and held its warp for hundreds of milliseconds.  For those
// axes the reciprocal is replaced by +-2^100: the slab then yields a huge negative entry (origin
// inside the slab, no constraint) or a huge positive one (outside, the box is refused), exactly,
// since scaling by a power of two is exact.  The walk visits only boxes that hold points of the
// ray, so it finds the same hits; among boxes the ray crosses it orders children by their true
// entry distances, where hitAABB's NaN chain would have dropped an axis, so of two hits at exactly
// the same distance, or of two occluders of a shadow ray, another may be found first.  Every other
// ray keeps the reference's arithmetic unchanged.
__device__ __forceinline__ void parallel_axis(float dir, float org, float &rcp, float &so) {
    if (!(fabsf(rcp) < INFINITY && fabsf(so) < INFINITY)) {
        rcp = copysignf(0x1p100f, dir);
        so = -org * rcp;
    }
}

// prePrepRay core/init.h:536
__device__ __forceinline__ void pre_prep(RayD &r) {
    r.ox = signbit(r.direction.x);
    r.oy = signbit(r.direction.y);
    r.oz = signbit(r.direction.z);
    r.scaled_origin.x = -r.origin.x * r.rcp.x;
    r.scaled_origin.y = -r.origin.y * r.rcp.y;
    r.scaled_origin.z = -r.origin.z * r.rcp.z;
    parallel_axis(r.direction.x, r.origin.x, r.rcp.x, r.scaled_origin.x);
    parallel_axis(r.direction.y, r.origin.y, r.rcp.y, r.scaled_origin.y);
    parallel_axis(r.direction.z, r.origin.z, r.rcp.z, r.scaled_origin.z);
}

// hitAABB render/AABB.h:6 (the octant offset selects max for the entry plane when negative)
__device__ __forceinline__ bool hit_aabb(v3 bmin, v3 bmax, const RayD &r, float closest, float &dist) {
    v3 mn = V(r.ox ? bmax.x : bmin.x, r.oy ? bmax.y : bmin.y, r.oz ? bmax.z : bmin.z);
    v3 mx = V(r.ox ? bmin.x : bmax.x, r.oy ? bmin.y : bmax.y, r.oz ? bmin.z : bmax.z);
    mn = vvfma(mn, r.rcp, r.scaled_origin);
    mx = vvfma(mx, r.rcp, r.scaled_origin);
    float a = mx.x < mx.y ? mx.x : mx.y;
    a = a < mx.z ? a : mx.z;
    a = a < closest ? a : closest;
    float b = mn.x > mn.y ? mn.x : mn.y;
    b = b > mn.z ? b : mn.z;
    b = b > 0 ? b : 0;
    dist = b;
    return b <= a;
}

// scene/primitive.h:8-51
__device__ __forceinline__ void to_object(v3 pos, v3 dir, const PrimDev &p, v3 &opos, v3 &odir) {
    unsigned f = prim_flags(p);
    v3 P = V(p.pos_bits.x, p.pos_bits.y, p.pos_bits.z);
    opos = (f & IS_TRANSLATED) ? pos - P : pos;
    if (f & IS_ROTATED) {
        q4 inv;
        inv.axis = V(-p.rot.x, -p.rot.y, -p.rot.z);
        inv.w = p.rot.w;
        opos = qrot(opos, inv);
        odir = qrot(dir, inv);
    } else odir = dir;
    if (f & IS_SCALED) {
        v3 is = V(p.inv_scale.x, p.inv_scale.y, p.inv_scale.z);
        opos = vmul(opos, is);
        if (f & IS_SCALED_NON_UNIFORMLY) odir = norm(vmul(odir, is));
    }
}
__device__ __forceinline__ q4 prim_rot(const PrimDev &p) { q4 q; q.axis = V(p.rot.x, p.rot.y, p.rot.z); q.w = p.rot.w; return q; }
__device__ __forceinline__ v3 pos_to_world(v3 pos, const PrimDev &p) {
    unsigned f = prim_flags(p);
    if (f & IS_SCALED) pos = vmul(pos, V(p.scale_id.x, p.scale_id.y, p.scale_id.z));
    if (f & IS_ROTATED) pos = qrot(pos, prim_rot(p));
    if (f & IS_TRANSLATED) pos = pos + V(p.pos_bits.x, p.pos_bits.y, p.pos_bits.z);
    return pos;
}
__device__ __forceinline__ v3 pos_to_object(v3 pos, const PrimDev &p) {
    unsigned f = prim_flags(p);
    if (f & IS_TRANSLATED) pos = pos - V(p.pos_bits.x, p.pos_bits.y, p.pos_bits.z);
    if (f & IS_ROTATED) pos = qrot(pos, conj(prim_rot(p)));
    if (f & IS_SCALED) pos = vmul(pos, V(p.inv_scale.x, p.inv_scale.y, p.inv_scale.z));
    return pos;
}
__device__ __forceinline__ v3 dir_to_world(v3 d, const PrimDev &p) {
    unsigned f = prim_flags(p);
    if (f & IS_SCALED_NON_UNIFORMLY) d = vmul(d, V(p.inv_scale.x, p.inv_scale.y, p.inv_scale.z));
    if (f & IS_ROTATED) d = qrot(d, prim_rot(p));
    return d;
}

// ---- render/shaders/common.h -------------------------------------------------------------------
__device__ __forceinline__ float tone_mapped(float c) {            // toneMappedBaked :86
    float x = c - 0.004f;
    if (x < 0.0f) x = 0.0f;
    float x2s = x * x * 6.2f;
    return (x2s + x * 0.5f) / (x2s + x * 1.7f + 0.06f);
}
__device__ __forceinline__ bool transparent_uv(float u_, float v_) { // isTransparentUV :115
    unsigned v = (unsigned char)(v_ * 4);
    unsigned u = (unsigned char)(u_ * 4);
    return (v % 2 != 0) == (bool)(u % 2);
}
__device__ __forceinline__ int box_side(v3 o, int axis) {          // getBoxSide :121
    switch (axis) {
        case 0: return o.x > 0 ? Right : Left;
        case 3: return o.x > 0 ? Left : Right;
        case 1: return o.y > 0 ? Top : Bottom;
        case 4: return o.y > 0 ? Bottom : Top;
        case 2: return o.z > 0 ? Front : Back;
        default: return o.z > 0 ? Back : Front;
    }
}
__device__ __forceinline__ void cube_uv(v3 p, int side, float &u, float &v) {  // getUVonUnitCube :132
    switch (side) {
        case Top: u = p.x; v = p.z; break;
        case Bottom: u = -p.x; v = -p.z; break;
        case Left: u = -p.z; v = p.y; break;
        case Right: u = p.z; v = p.y; break;
        case Front: u = p.x; v = p.y; break;
        default: u = -p.x; v = p.y; break;
    }
    u += 1; v += 1; u *= 0.5f; v *= 0.5f;
}
__device__ __forceinline__ bool hit_plane(v3 po, v3 pn, v3 ro, v3 rd, Hit &hit) {   // hitPlane :177
    hit.NdotV = -dot(rd, pn);
    if (hit.NdotV == 0) return false;
    bool facing = hit.NdotV > 0;
    float RPdotN = dot(po - ro, pn);
    hit.from_behind = RPdotN > 0;
    if (hit.from_behind == facing) return false;
    hit.distance = fabsf(RPdotN / hit.NdotV);
    hit.position = vscale(rd, hit.distance);
    hit.position = ro + hit.position;
    hit.normal = pn;
    return true;
}
__device__ __forceinline__ v3 area_light_vector(const Primitive &p, v3 P, v3 *v) {  // getAreaLightVector :197
    if (p.scale.x == 0 || p.scale.z == 0) return splat(0);
    v3 U = splat(0), W = splat(0);
    U.x = p.scale.x; if (U.x < 0) U.x = -U.x;
    W.z = p.scale.z; if (W.z < 0) W.z = -W.z;
    q4 q; q.axis = from(p.rotation.axis); q.w = p.rotation.amount;
    U = qrot(U, q);
    W = qrot(W, q);
    v3 pos = from(p.position);
    v[0] = (pos - U) - W;
    v[1] = (pos + U) - W;
    v[2] = (pos + U) + W;
    v[3] = (pos - U) + W;
    v3 u1 = norm(v[0] - P), u2 = norm(v[1] - P), u3 = norm(v[2] - P), u4 = norm(v[3] - P);
    float a12 = acosf(dot(u1, u2)), a23 = acosf(dot(u2, u3)), a34 = acosf(dot(u3, u4)), a41 = acosf(dot(u4, u1));
    v3 out = vscale(cross(u1, u2), a12);
    out = out + vscale(cross(u2, u3), a23);
    out = out + vscale(cross(u3, u4), a34);
    out = out + vscale(cross(u4, u1), a41);
    return vscale(out, 0.5f);
}

struct Shaded {                                                      // core/types.h:328
    u32t prim_index;
    const Material *material;
    v3 albedo, position, normal, viewing_direction, viewing_origin, reflected_direction, light_direction;
    v3 quad_vertices[4];
    float u, v;
};

__device__ __forceinline__ v3 shade_classic(v3 diffuse, float NdotL, v3 spec, float sf, float exponent, float roughness) {
    float shininess = 1.0f - roughness;                              // shadeClassic :294
    sf = NdotL * powf(sf, exponent * shininess) * shininess;
    return vsfma(spec, sf, diffuse);
}
__device__ v3 shade_point(const Shaded &s, float NdotL) {           // shadePointOnSurface :299
    const Material &M = *s.material;
    v3 diffuse = vscale(s.albedo, M.roughness * NdotL * kOneOverPi);
    if (M.brdf == BRDF_Lambert) return diffuse;
    if (M.brdf == BRDF_Phong) {
        float RdotL = dot01(s.reflected_direction, s.light_direction);
        return RdotL ? shade_classic(diffuse, NdotL, from(M.reflectivity), RdotL, 4.0f, M.roughness) : diffuse;
    }
    v3 N = s.normal, L = s.light_direction, Vv = neg(s.viewing_direction);
    v3 H = norm(L + Vv);
    float NdotH = dot01(N, H);
    if (M.brdf == BRDF_Blinn)
        return NdotH ? shade_classic(diffuse, NdotL, from(M.reflectivity), NdotH, 16.0f, M.roughness) : diffuse;
    v3 F = splat(0);
    diffuse = vscale(s.albedo, (1.0f - M.metallic) * NdotL * kOneOverPi);
    float LdotH = dot01(L, H);
    if (LdotH != 1.0f) {
        v3 refl = from(M.reflectivity);
        F = vsfma(one_minus(refl), powf(1.0f - LdotH, 5.0f), refl);  // ggxFresnelSchlick :291
        diffuse = vmul(diffuse, one_minus(F));
    }
    if (!M.roughness && NdotH == 1.0f) return diffuse;
    float NdotV = dot01(N, Vv);
    if (!NdotV) return diffuse;
    float r2 = M.roughness * M.roughness;                            // ggxNDF :277
    float demon = NdotH * NdotH * (r2 - 1.0f) + 1.0f;
    float D = kOneOverPi * r2 / (demon * demon);
    float k = M.roughness * 0.5f;                                    // ggxSmithSchlick :281
    float omk = 1.0f - k;
    float denom = NdotV * omk + k;
    float G = NdotV / fmaxf(denom, kEps);
    denom = NdotL * omk + k;
    G = G * NdotL / fmaxf(denom, kEps);
    return vsfma(F, D * G / (4.0f * NdotV), diffuse);
}
__device__ __forceinline__ float duv_ray_cone(float NdotV, float cone_width, float area, float uv_area) {
    float pcw = cone_width / fabsf(NdotV);                           // dUVbyRayCone :336
    return sqrtf((pcw * pcw) * (uv_area / area));
}

// ---- scene/texture.h ---------------------------------------------------------------------------
template <bool CNT, int SHS>
__device__ v3 sample_texture(TState<CNT, SHS> &t, const SceneDev &S, u32t tex, float U0, float V0, float du, float dv) {
    TexDev T = S.textures[tex];                                      // sampleTexture :32
    unsigned level = 0;
    if (T.mipmap) {
        const float pw = du * (float)T.width, ph = dv * (float)T.height;
        float size = (pw + ph) * 0.5f;
        const unsigned last = (unsigned char)(T.mip_count - 1);
        while (size > 1 && level < last) { size /= 2; level += 1; }
    }
    t.count(C_TEXEL);
    if (level) t.count(C_TEXEL_MIP);
    MipDev m = S.mips[T.mip_offset + level];                         // sampleTextureMip :5
    float u = U0, v = V0;
    if (u > 1) u -= (float)((u32t)u);
    if (v > 1) v -= (float)((u32t)v);
    const float Uf = u * (float)m.width + 0.5f;
    const float Vf = v * (float)m.height + 0.5f;
    // the clamps never bind for finite uv in [0, 1]; they keep a degenerate uv inside the grid
    const u32t x = min((u32t)Uf, (u32t)m.width), y = min((u32t)Vf, (u32t)m.height);
    const float r = Uf - (float)x, b = Vf - (float)y, l = 1 - r, tt = 1 - b;
    const float tl = tt * l * kColorToFloat, tr = tt * r * kColorToFloat;
    const float bl = b * l * kColorToFloat, br = b * r * kColorToFloat;
    const uint32_t *q = reinterpret_cast<const uint32_t *>(S.quads + m.quad_offset + (size_t)y * (m.width + 1) + x);
    uint32_t R = __ldg(q), G = __ldg(q + 1), B = __ldg(q + 2);     // TexelQuad: R{TL,TR,BL,BR} G{..} B{..}
#define ST_CH(w, i) ((float)(((w) >> (8 * (i))) & 0xFFu))
    return V(ST_CH(R, 3) * br + (ST_CH(R, 2) * bl + (ST_CH(R, 1) * tr + ST_CH(R, 0) * tl)),
             ST_CH(G, 3) * br + (ST_CH(G, 2) * bl + (ST_CH(G, 1) * tr + ST_CH(G, 0) * tl)),
             ST_CH(B, 3) * br + (ST_CH(B, 2) * bl + (ST_CH(B, 1) * tr + ST_CH(B, 0) * tl)));
#undef ST_CH
}
template <bool CNT, int SHS>
__device__ __forceinline__ v3 sample_normal(TState<CNT, SHS> &t, const SceneDev &S, u32t tex, float u, float v, float du, float dv) {
    v3 n = sample_texture(t, S, tex, u, v, du, dv);                 // sampleNormal surface.h:131
    float y = n.z; n.z = n.y; n.y = y;
    return norm(vsfma(n, 2.0f, splat(-1.0f)));
}
__device__ __forceinline__ q4 normal_rotation(v3 n) {               // getNormalRotation surface.h:138
    q4 q;
    q.axis = V(n.z * 0.25f, 0, n.x * 0.25f);
    q.w = n.y * 0.25f;
    return qnorm(q);
}

// ---- render/shaders/intersection -------------------------------------------------------------
__device__ __forceinline__ bool hit_quad(Hit &hit, v3 Ro, v3 Rd, unsigned flags) {   // quad.h:7
    if (Rd.y == 0) return false;
    if (Ro.y == 0) return false;
    hit.from_behind = Ro.y < 0;
    if (hit.from_behind == (Rd.y < 0)) return false;
    hit.distance = fabsf(Ro.y / Rd.y);
    hit.position = vsfma(Rd, hit.distance, Ro);
    if (hit.position.x < -1 || hit.position.x > +1 || hit.position.z < -1 || hit.position.z > +1) return false;
    hit.u = (hit.position.x + 1.0f) * 0.5f;
    hit.v = (hit.position.z + 1.0f) * 0.5f;
    if ((flags & IS_TRANSPARENT) && transparent_uv(hit.u, hit.v)) return false;
    hit.normal = V(0, 1, 0);
    hit.NdotV = -Rd.y;
    hit.area = 4;
    hit.uv_area = 1;
    return true;
}
__device__ __forceinline__ bool hit_box(Hit &hit, v3 Ro, v3 Rd, unsigned flags) {    // box.h:7
    v3 rc = rcp(Rd), oc;
    oc.x = signbit(Rd.x) ? 1.0f : -1.0f;
    oc.y = signbit(Rd.y) ? 1.0f : -1.0f;
    oc.z = signbit(Rd.z) ? 1.0f : -1.0f;
    float t[6];
    t[0] = (oc.x - Ro.x) * rc.x;
    t[1] = (oc.y - Ro.y) * rc.y;
    t[2] = (oc.z - Ro.z) * rc.z;
    t[3] = (-oc.x - Ro.x) * rc.x;
    t[4] = (-oc.y - Ro.y) * rc.y;
    t[5] = (-oc.z - Ro.z) * rc.z;
    int max_axis = t[3] < t[4] ? 3 : 4;
    if (t[5] < (max_axis == 3 ? t[3] : t[4])) max_axis = 5;
    float maxt = max_axis == 3 ? t[3] : (max_axis == 4 ? t[4] : t[5]);
    if (maxt < 0) return false;
    int min_axis = t[0] > t[1] ? 0 : 1;
    if (t[2] > (min_axis == 0 ? t[0] : t[1])) min_axis = 2;
    float mint = min_axis == 0 ? t[0] : (min_axis == 1 ? t[1] : t[2]);
    if (maxt < (mint > 0 ? mint : 0)) return false;
    hit.from_behind = mint < 0;
    if (hit.from_behind) { mint = maxt; min_axis = max_axis; }
    int side = box_side(oc, min_axis);
    hit.position = vsfma(Rd, mint, Ro);
    cube_uv(hit.position, side, hit.u, hit.v);
    if ((flags & IS_TRANSPARENT) && transparent_uv(hit.u, hit.v)) {
        if (hit.from_behind) return false;
        side = box_side(oc, max_axis);
        hit.position = vsfma(Rd, maxt, Ro);
        cube_uv(hit.position, side, hit.u, hit.v);
        if (transparent_uv(hit.u, hit.v)) return false;
        hit.from_behind = true;
    }
    hit.normal = splat(0);
    switch (side) {
        case Left:   hit.normal.x = -1.0f; hit.NdotV = +Rd.x; break;
        case Right:  hit.normal.x = +1.0f; hit.NdotV = -Rd.x; break;
        case Bottom: hit.normal.y = -1.0f; hit.NdotV = +Rd.y; break;
        case Top:    hit.normal.y = +1.0f; hit.NdotV = -Rd.y; break;
        case Back:   hit.normal.z = -1.0f; hit.NdotV = +Rd.z; break;
        case Front:  hit.normal.z = +1.0f; hit.NdotV = -Rd.z; break;
        default: return false;
    }
    if (hit.from_behind) { hit.normal = neg(hit.normal); hit.NdotV = -hit.NdotV; }
    hit.area = 4;
    hit.uv_area = 1;
    return true;
}
__device__ __forceinline__ void sphere_uv(v3 d, float &u, float &v) {   // getUVonUnitSphere sphere.h:7
    float x = d.x, y = d.y, z = d.z;
    float zx = x ? (z / x) : 2, yx = x ? (y / x) : 2;
    if (zx <= 1 && zx >= -1 && yx <= 1 && yx >= -1) {
        u = zx;
        v = x > 0 ? yx : -yx;
    } else {
        float xz = z ? (x / z) : 2, yz = z ? (y / z) : 2;
        if (xz <= 1 && xz >= -1 && yz <= 1 && yz >= -1) {
            u = -xz;
            v = z > 0 ? yz : -yz;
        } else {
            u = x / (y > 0 ? y : -y);
            v = z / y;
        }
    }
    u += 1; u /= 2;
    v += 1; v /= 2;
}
__device__ __forceinline__ bool hit_sphere_simple(v3 Ro, v3 Rd, v3 target, float oor, SphereHitD &h) {  // sphere.h:44
    v3 rc = vscale(target - Ro, oor);
    h.b = dot(Rd, rc);
    h.c = dot(rc, rc) - 1;
    float d = h.b * h.b - h.c;
    if (d < 0) return false;
    d = sqrtf(d);
    h.t_near = h.b - d;
    h.t_far = h.b + d;
    return h.t_far > 0 && h.t_near < h.furthest;
}
__device__ __forceinline__ bool hit_sphere(Hit &hit, v3 Ro, v3 Rd, unsigned flags) {   // sphere.h:61
    float tc = -dot(Ro, Rd);
    if (tc <= 0) return false;
    hit.distance_squared = sqlen(Ro) - tc * tc;
    float ds = 1 - hit.distance_squared;
    if (ds <= 0) { hit.distance = tc; return false; }
    float delta = sqrtf(ds);
    hit.distance = tc - delta;
    bool outer = hit.distance > 0;
    if (outer) {
        hit.position = vsfma(Rd, hit.distance, Ro);
        sphere_uv(hit.position, hit.u, hit.v);
        if ((flags & IS_TRANSPARENT) && transparent_uv(hit.u, hit.v)) outer = false;
    }
    if (!outer) {
        hit.distance = tc + delta;
        hit.position = vsfma(Rd, hit.distance, Ro);
        sphere_uv(hit.position, hit.u, hit.v);
        if ((flags & IS_TRANSPARENT) && transparent_uv(hit.u, hit.v)) return false;
    }
    hit.from_behind = !outer;
    hit.normal = hit.position;
    hit.NdotV = -dot(hit.normal, Rd);
    hit.area = hit.uv_area = kUnitSphereAreaOverSix;
    return true;
}
__device__ __forceinline__ bool hit_tetra(Hit &closest, v3 Ro, v3 Rd, unsigned flags) {   // tetrahedra.h:9
    // tangent matrices of the four faces, tetrahedra.h:55-101 (X.xyz Y.xyz Z.xyz)
    const float M[4][9] = {
        { kT0577, -kT0288, -kT0577,  kT0288,  kT0288,  kT0577, -kT0288,  kT0577, -kT0577},
        { kT0288,  kT0288,  kT0577, -kT0288,  kT0577, -kT0577,  kT0577, -kT0288, -kT0577},
        {-kT0288,  kT0577, -kT0577,  kT0577, -kT0288, -kT0577,  kT0288,  kT0288,  kT0577},
        {-kT0577,  kT0288,  kT0577,  kT0288,  kT0288,  kT0577,  kT0288, -kT0577,  kT0577}};
    bool found = false;
    float cd = INFINITY;
    Hit hit = closest;
    hit.cone_width = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        v3 tp = splat(t == 3 ? kT0577 : -kT0577);
        v3 n = tp;
        if (t == 0) n.y = kT0577;
        if (t == 1) n.x = kT0577;
        if (t == 2) n.z = kT0577;
        if (t == 3) tp.y = -kT0577;
        if (!hit_plane(tp, n, Ro, Rd, hit)) continue;
        hit.position = vsfma(Rd, hit.distance, Ro);
        v3 q = vmat3(hit.position - tp, M[t]);
        if (q.x < 0 || q.y < 0 || q.y + q.x > 1) continue;
        hit.u = q.x;
        hit.v = q.y;
        if ((flags & IS_TRANSPARENT) && transparent_uv(hit.u, hit.v)) continue;
        if (hit.distance < cd) {
            cd = hit.distance;
            hit.area = kSqrt3 / 4.0f;
            hit.uv_area = 1;
            hit.NdotV = -dot(hit.normal, Rd);
            closest = hit;
            found = true;
        }
    }
    return found;
}

}  // namespace st
