/*
 * oracle.c — TEST INFRASTRUCTURE: a CPU restatement of SlimTracin's per-pixel tracing path and its
 * BVH builds, written from the reference's behaviour (every function names the reference lines it
 * follows), used only to check the device path.  It keeps the reference's floating-point operation
 * order (compiled without contraction, see Makefile) so that, where the arithmetic is IEEE-exact,
 * its output is bit-identical to the reference's; tests pin it against oracle/_ref (the reference's
 * own code) and against the golden monkey.mesh.
 *
 * Two documented choices where the reference reads uninitialised memory:
 *   - hitTetrahedron (intersection/tetrahedra.h:14) copies a partly uninitialised local RayHit into
 *     current_hit; the fields it never writes (cone_angle, dUV, ...) are taken as 0 here, as a
 *     zero-initialised struct gives.  They only reach an output through the ray-cone texture
 *     footprint of a later hit.
 *   - shadeSurface's dUV.v (closest_hit/surface.h:152,230) is stale on bounce hits and
 *     uninitialised when the first hit has no texture; it starts at 0 here.
 *
 * The LBVH30 builder at the end has no reference counterpart (builder_bottom_up.h is dead code);
 * it is the project's specification of the 30-bit Morton LBVH the device builder must reproduce.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define TRACE_OFFSET 0.0001f
#define ORC_EPS 0.0001f
#define ORC_PI 3.14159265f
#define ONE_OVER_PI (1.0f / ORC_PI)
#define SQRT2 1.41421356237f
#define SQRT3 1.73205080757f
#define UNIT_SPHERE_AREA_OVER_SIX ((4.0f * ORC_PI) / 6.0f)
#define COLOR_COMPONENT_TO_FLOAT 0.00392156862f
#define FLOAT_TO_COLOR_COMPONENT 255.0f
#define T_0577 0.577350259f
#define T_0288 0.288675159f
#define ORC_STACK 256

#define CNT(tr, k) ((tr)->cnt[(k)]++)
#ifndef true
#define true 1
#define false 0
#endif

/* ---- vector math: math/vec3.h, math/quat.h, math/mat3.h ------------------------------------- */
static inline vec3 V3(f32 x, f32 y, f32 z) { vec3 o; o.x = x; o.y = y; o.z = z; return o; }
static inline vec3 splat(f32 v) { return V3(v, v, v); }
static inline vec3 vsub(vec3 a, vec3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline vec3 vadd(vec3 a, vec3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline vec3 vmul(vec3 a, vec3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline vec3 vscale(vec3 a, f32 f) { return V3(a.x * f, a.y * f, a.z * f); }
/* scaleAddVec3 (vec3.h:183) with fast_mul_add = a*b+c (base.h:75) */
static inline vec3 vsfma(vec3 v, f32 f, vec3 c) { return V3(v.x * f + c.x, v.y * f + c.y, v.z * f + c.z); }
/* mulAddVec3 (vec3.h:173) */
static inline vec3 vvfma(vec3 v, vec3 f, vec3 c) { return V3(v.x * f.x + c.x, v.y * f.y + c.y, v.z * f.z + c.z); }
static inline f32 vdot(vec3 a, vec3 b) { return ((a.x * b.x) + (a.y * b.y)) + (a.z * b.z); }
static inline vec3 vcross(vec3 a, vec3 b) {
    return V3((a.y * b.z) - (a.z * b.y), (a.z * b.x) - (a.x * b.z), (a.x * b.y) - (a.y * b.x));
}
static inline f32 vsqlen(vec3 v) { return ((v.x * v.x) + (v.y * v.y)) + (v.z * v.z); }
static inline f32 vlen(vec3 v) { return sqrtf(vsqlen(v)); }
static inline vec3 vnorm(vec3 v) { return vscale(v, 1.0f / vlen(v)); }
static inline vec3 vrcp(vec3 v) { return V3(1.0f / v.x, 1.0f / v.y, 1.0f / v.z); }
static inline vec3 vneg(vec3 v) { return V3(-v.x, -v.y, -v.z); }
static inline vec3 vone_minus(vec3 v) { return V3(1.0f - v.x, 1.0f - v.y, 1.0f - v.z); }
static inline f32 clamp01(f32 v) { f32 mn = v < 1.0f ? v : 1.0f; return mn > 0.0f ? mn : 0.0f; }
static inline f32 vdot01(vec3 a, vec3 b) { return clamp01(vdot(a, b)); }        /* DotVec3 vec3.h:247 */
static inline f32 maxcoord(vec3 v) { f32 o = v.x; if (v.y > o) o = v.y; if (v.z > o) o = v.z; return o; }
/* mulVec3Quat quat.h:25 */
static inline vec3 qrot(vec3 v, quat q) {
    vec3 out = vcross(q.axis, v);
    vec3 qqv = vcross(q.axis, out);
    out = vsfma(out, q.amount, qqv);
    out = vsfma(out, 2.0f, v);
    return out;
}
static inline quat qconj(quat q) { quat o; o.amount = q.amount; o.axis = vneg(q.axis); return o; }
/* normQuat quat.h:15 */
static inline quat qnorm(quat q) {
    quat o;
    f32 f = 1.0f / sqrtf(q.axis.x * q.axis.x + q.axis.y * q.axis.y + q.axis.z * q.axis.z + q.amount * q.amount);
    o.axis = vscale(q.axis, f);
    o.amount = q.amount * f;
    return o;
}
/* mulVec3Mat3 vec3.h:203 */
static inline vec3 vmat3(vec3 in, mat3 m) {
    return V3(in.x * m.X.x + in.y * m.Y.x + in.z * m.Z.x,
              in.x * m.X.y + in.y * m.Y.y + in.z * m.Z.y,
              in.x * m.X.z + in.y * m.Y.z + in.z * m.Z.z);
}
/* invMat3 mat3.h:97 */
static mat3 minv3(mat3 m) {
    mat3 o;
    f32 d = 1.0f / (
        + m.X.x * (m.Y.y * m.Z.z - m.Z.y * m.Y.z)
        - m.Y.x * (m.X.y * m.Z.z - m.Z.y * m.X.z)
        + m.Z.x * (m.X.y * m.Y.z - m.Y.y * m.X.z));
    o.X.x = + (m.Y.y * m.Z.z - m.Z.y * m.Y.z) * d;
    o.Y.x = - (m.Y.x * m.Z.z - m.Z.x * m.Y.z) * d;
    o.Z.x = + (m.Y.x * m.Z.y - m.Z.x * m.Y.y) * d;
    o.X.y = - (m.X.y * m.Z.z - m.Z.y * m.X.z) * d;
    o.Y.y = + (m.X.x * m.Z.z - m.Z.x * m.X.z) * d;
    o.Z.y = - (m.X.x * m.Z.y - m.Z.x * m.X.y) * d;
    o.X.z = + (m.X.y * m.Y.z - m.Y.y * m.X.z) * d;
    o.Y.z = - (m.X.x * m.Y.z - m.Y.x * m.X.z) * d;
    o.Z.z = + (m.X.x * m.Y.y - m.Y.x * m.X.y) * d;
    return o;
}

/* ---- primitive spaces: scene/primitive.h:8-59 ------------------------------------------------- */
static inline void to_object(vec3 pos, vec3 dir, const Primitive *p, vec3 *opos, vec3 *odir) {
    *opos = (p->flags & IS_TRANSLATED) ? vsub(pos, p->position) : pos;
    if (p->flags & IS_ROTATED) {
        quat inv = qconj(p->rotation);
        *opos = qrot(*opos, inv);
        *odir = qrot(dir, inv);
    } else *odir = dir;
    if (p->flags & IS_SCALED) {
        vec3 inv_scale = vrcp(p->scale);
        *opos = vmul(*opos, inv_scale);
        if (p->flags & IS_SCALED_NON_UNIFORMLY) *odir = vnorm(vmul(*odir, inv_scale));
    }
}
static inline vec3 pos_to_world(vec3 pos, const Primitive *p) {
    if (p->flags & IS_SCALED) pos = vmul(pos, p->scale);
    if (p->flags & IS_ROTATED) pos = qrot(pos, p->rotation);
    if (p->flags & IS_TRANSLATED) pos = vadd(pos, p->position);
    return pos;
}
static inline vec3 pos_to_object(vec3 pos, const Primitive *p) {
    if (p->flags & IS_TRANSLATED) pos = vsub(pos, p->position);
    if (p->flags & IS_ROTATED) pos = qrot(pos, qconj(p->rotation));
    if (p->flags & IS_SCALED) pos = vmul(pos, vrcp(p->scale));
    return pos;
}
static inline vec3 dir_to_world(vec3 d, const Primitive *p) {
    if (p->flags & IS_SCALED_NON_UNIFORMLY) d = vmul(d, vrcp(p->scale));
    if (p->flags & IS_ROTATED) d = qrot(d, p->rotation);
    return d;
}

/* ---- per-ray scratch (the reference's Trace, core/types.h:193) ------------------------------- */
typedef struct {
    SphereHit sphere_hit;
    RayHit closest_hit, closest_mesh_hit, current_hit;
    Ray local;
    u32 scene_stack[ORC_STACK], mesh_stack[ORC_STACK];
    u32 mesh_stack_size;
    u8 depth;
    uint64_t cnt[ORC_COUNTERS];
} OTrace;

/* prePrepRay core/init.h:536 */
static inline void pre_prep(Ray *r) {
    r->octant.x = signbit(r->direction.x) ? 3 : 0;
    r->octant.y = signbit(r->direction.y) ? 3 : 0;
    r->octant.z = signbit(r->direction.z) ? 3 : 0;
    r->scaled_origin.x = -r->origin.x * r->direction_reciprocal.x;
    r->scaled_origin.y = -r->origin.y * r->direction_reciprocal.y;
    r->scaled_origin.z = -r->origin.z * r->direction_reciprocal.z;
}

/* hitAABB render/AABB.h:6 — the octant offset picks min or max as a flat array of 6 floats */
static inline bool hit_aabb(const AABB *b, const Ray *r, f32 closest, f32 *dist) {
    const f32 *f = &b->min.x;
    vec3 mn = V3(f[0 + r->octant.x], f[1 + r->octant.y], f[2 + r->octant.z]);
    vec3 mx = V3(f[3 - r->octant.x], f[4 - r->octant.y], f[5 - r->octant.z]);
    mn = vvfma(mn, r->direction_reciprocal, r->scaled_origin);
    mx = vvfma(mx, r->direction_reciprocal, r->scaled_origin);
    mx.x = mx.x < mx.y ? mx.x : mx.y;
    mx.x = mx.x < mx.z ? mx.x : mx.z;
    mx.x = mx.x < closest ? mx.x : closest;
    mn.x = mn.x > mn.y ? mn.x : mn.y;
    mn.x = mn.x > mn.z ? mn.x : mn.z;
    mn.x = mn.x > 0 ? mn.x : 0;
    *dist = mn.x;
    return mn.x <= mx.x;
}
static inline AABB merge_aabb(AABB l, AABB r) {                         /* AABB.h:25 */
    AABB m;
    m.min.x = l.min.x < r.min.x ? l.min.x : r.min.x;
    m.min.y = l.min.y < r.min.y ? l.min.y : r.min.y;
    m.min.z = l.min.z < r.min.z ? l.min.z : r.min.z;
    m.max.x = l.max.x > r.max.x ? l.max.x : r.max.x;
    m.max.y = l.max.y > r.max.y ? l.max.y : r.max.y;
    m.max.z = l.max.z > r.max.z ? l.max.z : r.max.z;
    return m;
}
static inline f32 half_area(AABB a) {                                   /* AABB.h:39 */
    vec3 e = vsub(a.max, a.min);
    return e.x * e.y + e.y * e.z + e.z * e.x;
}
static void transform_aabb(AABB *a, const Primitive *p) {               /* AABB.h:44 */
    f32 x = a->min.x, y = a->min.y, z = a->min.z, X = a->max.x, Y = a->max.y, Z = a->max.z;
    vec3 v[8] = {{x, y, z}, {x, y, Z}, {x, Y, z}, {x, Y, Z},
                 {X, y, z}, {X, y, Z}, {X, Y, z}, {X, Y, Z}};
    x = y = z = +INFINITY;
    X = Y = Z = -INFINITY;
    for (int i = 0; i < 8; i++) {
        vec3 q = pos_to_world(v[i], p);
        if (q.x > X) X = q.x;
        if (q.y > Y) Y = q.y;
        if (q.z > Z) Z = q.z;
        if (q.x < x) x = q.x;
        if (q.y < y) y = q.y;
        if (q.z < z) z = q.z;
    }
    a->min = V3(x, y, z);
    a->max = V3(X, Y, Z);
}

/* ---- shading helpers: render/shaders/common.h ------------------------------------------------ */
static inline f32 tone_mapped(f32 c) {                                  /* common.h:86 */
    f32 x = c - 0.004f;
    if (x < 0.0f) x = 0.0f;
    f32 x2s = x * x * 6.2f;
    return (x2s + x * 0.5f) / (x2s + x * 1.7f + 0.06f);
}
static inline f32 inv_dot(vec3 a, vec3 b) { return clamp01(-vdot(a, b)); }       /* common.h:97 */
static inline vec3 reflect_dot(vec3 V, vec3 N, f32 NdotV) { return vsfma(N, -2.0f * NdotV, V); } /* :101 */
static inline vec3 refract_dir(vec3 V, vec3 N, f32 n1_over_n2, f32 NdotV) {                    /* :105 */
    f32 c = n1_over_n2 * n1_over_n2 * (1 - (NdotV * NdotV));
    if (c > 1) return splat(0);
    V = vscale(V, n1_over_n2);
    V = vsfma(N, n1_over_n2 * -NdotV - sqrtf(1 - c), V);
    return vnorm(V);
}
static inline bool transparent_uv(vec2 uv) {                            /* common.h:115 */
    u8 v = (u8)(uv.y * 4);
    u8 u = (u8)(uv.x * 4);
    return (v % 2 != 0) == (u % 2);
}
static inline BoxSide box_side(vec3 o, u8 axis) {                       /* common.h:121 */
    switch (axis) {
        case 0: return o.x > 0 ? Right : Left;
        case 3: return o.x > 0 ? Left : Right;
        case 1: return o.y > 0 ? Top : Bottom;
        case 4: return o.y > 0 ? Bottom : Top;
        case 2: return o.z > 0 ? Front : Back;
        default: return o.z > 0 ? Back : Front;
    }
}
static inline vec2 cube_uv(vec3 p, BoxSide side) {                      /* common.h:132 */
    vec2 uv;
    switch (side) {
        case Top: uv.x = p.x; uv.y = p.z; break;
        case Bottom: uv.x = -p.x; uv.y = -p.z; break;
        case Left: uv.x = -p.z; uv.y = p.y; break;
        case Right: uv.x = p.z; uv.y = p.y; break;
        case Front: uv.x = p.x; uv.y = p.y; break;
        default: uv.x = -p.x; uv.y = p.y; break;
    }
    uv.x += 1; uv.y += 1; uv.x *= 0.5f; uv.y *= 0.5f;
    return uv;
}
static inline bool hit_plane(vec3 po, vec3 pn, const vec3 *ro, const vec3 *rd, RayHit *hit) { /* :177 */
    hit->NdotV = -vdot(*rd, pn);
    if (hit->NdotV == 0) return false;
    bool facing = hit->NdotV > 0;
    vec3 RP = vsub(po, *ro);
    f32 RPdotN = vdot(RP, pn);
    hit->from_behind = RPdotN > 0;
    if (hit->from_behind == facing) return false;
    hit->distance = fabsf(RPdotN / hit->NdotV);
    hit->position = vscale(*rd, hit->distance);
    hit->position = vadd(*ro, hit->position);
    hit->normal = pn;
    return true;
}
static vec3 area_light_vector(const Primitive *p, vec3 P, vec3 *v) {   /* common.h:197 */
    if (p->scale.x == 0 || p->scale.z == 0) return splat(0);
    vec3 U = splat(0), W = splat(0);
    U.x = p->scale.x; if (U.x < 0) U.x = -U.x;
    W.z = p->scale.z; if (W.z < 0) W.z = -W.z;
    U = qrot(U, p->rotation);
    W = qrot(W, p->rotation);
    v[0] = vsub(vsub(p->position, U), W);
    v[1] = vsub(vadd(p->position, U), W);
    v[2] = vadd(vadd(p->position, U), W);
    v[3] = vadd(vsub(p->position, U), W);
    vec3 u1 = vnorm(vsub(v[0], P)), u2 = vnorm(vsub(v[1], P)), u3 = vnorm(vsub(v[2], P)), u4 = vnorm(vsub(v[3], P));
    f32 a12 = acosf(vdot(u1, u2)), a23 = acosf(vdot(u2, u3)), a34 = acosf(vdot(u3, u4)), a41 = acosf(vdot(u4, u1));
    vec3 out = vscale(vcross(u1, u2), a12);
    out = vadd(out, vscale(vcross(u2, u3), a23));
    out = vadd(out, vscale(vcross(u3, u4), a34));
    out = vadd(out, vscale(vcross(u4, u1), a41));
    return vscale(out, 0.5f);
}
static inline f32 ggx_ndf(f32 r2, f32 NdotH) {                           /* common.h:277 */
    f32 demon = NdotH * NdotH * (r2 - 1.0f) + 1.0f;
    return ONE_OVER_PI * r2 / (demon * demon);
}
static inline f32 ggx_smith(f32 NdotL, f32 NdotV, f32 roughness) {     /* common.h:281 */
    f32 k = roughness * 0.5f;
    f32 omk = 1.0f - k;
    f32 denom = NdotV * omk + k;
    f32 result = NdotV / fmaxf(denom, ORC_EPS);
    denom = NdotL * omk + k;
    return result * NdotL / fmaxf(denom, ORC_EPS);
}
static inline vec3 ggx_fresnel(vec3 refl, f32 LdotH) {                  /* common.h:291 */
    return vsfma(vone_minus(refl), powf(1.0f - LdotH, 5.0f), refl);
}
static inline vec3 shade_classic(vec3 diffuse, f32 NdotL, vec3 spec, f32 sf, f32 exponent, f32 roughness) { /* :294 */
    f32 shininess = 1.0f - roughness;
    sf = NdotL * powf(sf, exponent * shininess) * shininess;
    return vsfma(spec, sf, diffuse);
}

typedef struct {
    const Primitive *primitive;
    const Material *material;
    vec3 albedo, position, normal, viewing_direction, viewing_origin, reflected_direction, light_direction,
         emissive_quad_vertices[4];
    vec2 uv;
} OShaded;

static vec3 shade_point(const OShaded *s, f32 NdotL) {                 /* common.h:299 */
    const Material *M = s->material;
    vec3 nothing = splat(0);
    vec3 diffuse = vscale(s->albedo, M->roughness * NdotL * ONE_OVER_PI);
    if (M->brdf == BRDF_Lambert) return diffuse;
    if (M->brdf == BRDF_Phong) {
        f32 RdotL = vdot01(s->reflected_direction, s->light_direction);
        return RdotL ? shade_classic(diffuse, NdotL, M->reflectivity, RdotL, 4.0f, M->roughness) : diffuse;
    }
    vec3 N = s->normal, L = s->light_direction, Vv = vneg(s->viewing_direction);
    vec3 H = vnorm(vadd(L, Vv));
    f32 NdotH = vdot01(N, H);
    if (M->brdf == BRDF_Blinn)
        return NdotH ? shade_classic(diffuse, NdotL, M->reflectivity, NdotH, 16.0f, M->roughness) : diffuse;
    vec3 F = nothing;
    diffuse = vscale(s->albedo, (1.0f - M->metallic) * NdotL * ONE_OVER_PI);
    f32 LdotH = vdot01(L, H);
    if (LdotH != 1.0f) {
        F = ggx_fresnel(M->reflectivity, LdotH);
        diffuse = vmul(diffuse, vone_minus(F));
    }
    if (!M->roughness && NdotH == 1.0f) return diffuse;
    f32 NdotV = vdot01(N, Vv);
    if (!NdotV) return diffuse;
    f32 D = ggx_ndf(M->roughness * M->roughness, NdotH);
    f32 G = ggx_smith(NdotL, NdotV, M->roughness);
    return vsfma(F, D * G / (4.0f * NdotV), diffuse);
}
static inline f32 duv_ray_cone(f32 NdotV, f32 cone_width, f32 area, f32 uv_area) { /* common.h:336 */
    f32 pcw = cone_width / fabsf(NdotV);
    return sqrtf((pcw * pcw) * (uv_area / area));
}

/* ---- textures: scene/texture.h ----------------------------------------------------------------- */
static vec3 sample_mip(const TextureMip *mip, vec2 UV) {                  /* texture.h:5 */
    f32 u = UV.x, v = UV.y;
    if (u > 1) u -= (f32)((u32)u);
    if (v > 1) v -= (f32)((u32)v);
    const f32 U = u * (f32)mip->width + 0.5f;
    const f32 Vv = v * (f32)mip->height + 0.5f;
    const u32 x = (u32)U;
    const u32 y = (u32)Vv;
    const f32 r = U - (f32)x, b = Vv - (f32)y, l = 1 - r, t = 1 - b;
    const f32 tl = t * l * COLOR_COMPONENT_TO_FLOAT, tr = t * r * COLOR_COMPONENT_TO_FLOAT;
    const f32 bl = b * l * COLOR_COMPONENT_TO_FLOAT, br = b * r * COLOR_COMPONENT_TO_FLOAT;
    const TexelQuad q = mip->texel_quads[y * (mip->width + 1) + x];
    return V3((f32)q.R.BR * br + ((f32)q.R.BL * bl + ((f32)q.R.TR * tr + (f32)q.R.TL * tl)),
              (f32)q.G.BR * br + ((f32)q.G.BL * bl + ((f32)q.G.TR * tr + (f32)q.G.TL * tl)),
              (f32)q.B.BR * br + ((f32)q.B.BL * bl + ((f32)q.B.TR * tr + (f32)q.B.TL * tl)));
}
static vec3 sample_texture(const Texture *t, vec2 UV, vec2 dUV, OTrace *tr) { /* texture.h:32 */
    u8 level = 0;
    if (t->mipmap) {
        const f32 pw = dUV.x * (f32)t->width, ph = dUV.y * (f32)t->height;
        f32 size = (f32)(pw + ph) * 0.5f;
        const u8 last = t->mip_count - 1;
        while (size > 1 && level < last) { size /= 2; level += 1; }
    }
    CNT(tr, ORC_TEXEL_FETCHES);
    if (level) CNT(tr, ORC_TEXEL_MIP_FETCHES);
    return sample_mip(t->mips + level, UV);
}
static vec3 sample_normal(const Texture *t, vec2 uv, vec2 dUV, OTrace *tr) { /* surface.h:131 */
    vec3 n = sample_texture(t, uv, dUV, tr);
    f32 y = n.z; n.z = n.y; n.y = y;
    return vnorm(vsfma(n, 2.0f, splat(-1.0f)));
}
static quat normal_rotation(vec3 n) {                                    /* surface.h:138 */
    quat q;
    q.axis.x = n.z * 0.25f; q.axis.y = 0; q.axis.z = n.x * 0.25f; q.amount = n.y * 0.25f;
    return qnorm(q);
}

/* ---- intersections: render/shaders/intersection/ (all) ----------------------------------------- */
static bool hit_quad(RayHit *hit, const vec3 *Ro, const vec3 *Rd, u8 flags) {   /* quad.h:7 */
    if (Rd->y == 0) return false;
    if (Ro->y == 0) return false;
    hit->from_behind = Ro->y < 0;
    if (hit->from_behind == (Rd->y < 0)) return false;
    hit->distance = fabsf(Ro->y / Rd->y);
    hit->position = vsfma(*Rd, hit->distance, *Ro);
    if (hit->position.x < -1 || hit->position.x > +1 || hit->position.z < -1 || hit->position.z > +1) return false;
    hit->uv.x = (hit->position.x + 1.0f) * 0.5f;
    hit->uv.y = (hit->position.z + 1.0f) * 0.5f;
    if ((flags & IS_TRANSPARENT) && transparent_uv(hit->uv)) return false;
    hit->normal = V3(0, 1, 0);
    hit->NdotV = -Rd->y;
    hit->area = 4;
    hit->uv_area = 1;
    return true;
}
static BoxSide hit_box(RayHit *hit, const vec3 *Ro, const vec3 *Rd, u8 flags) {  /* box.h:7 */
    vec3 oc, rcp = vrcp(*Rd);
    oc.x = signbit(Rd->x) ? 1.0f : -1.0f;
    oc.y = signbit(Rd->y) ? 1.0f : -1.0f;
    oc.z = signbit(Rd->z) ? 1.0f : -1.0f;
    f32 t[6];
    t[0] = (oc.x - Ro->x) * rcp.x;
    t[1] = (oc.y - Ro->y) * rcp.y;
    t[2] = (oc.z - Ro->z) * rcp.z;
    t[3] = (-oc.x - Ro->x) * rcp.x;
    t[4] = (-oc.y - Ro->y) * rcp.y;
    t[5] = (-oc.z - Ro->z) * rcp.z;
    u8 max_axis = t[3] < t[4] ? 3 : 4; if (t[5] < t[max_axis]) max_axis = 5;
    f32 maxt = t[max_axis];
    if (maxt < 0) return NoSide;
    u8 min_axis = t[0] > t[1] ? 0 : 1; if (t[2] > t[min_axis]) min_axis = 2;
    f32 mint = t[min_axis];
    if (maxt < (mint > 0 ? mint : 0)) return NoSide;
    hit->from_behind = mint < 0;
    if (hit->from_behind) { mint = maxt; min_axis = max_axis; }
    BoxSide side = box_side(oc, min_axis);
    hit->position = vsfma(*Rd, mint, *Ro);
    hit->uv = cube_uv(hit->position, side);
    if ((flags & IS_TRANSPARENT) && transparent_uv(hit->uv)) {
        if (hit->from_behind) return NoSide;
        side = box_side(oc, max_axis);
        hit->position = vsfma(*Rd, maxt, *Ro);
        hit->uv = cube_uv(hit->position, side);
        if (transparent_uv(hit->uv)) return NoSide;
        hit->from_behind = true;
    }
    hit->normal = splat(0);
    switch (side) {
        case Left:   hit->normal.x = -1.0f; hit->NdotV = +Rd->x; break;
        case Right:  hit->normal.x = +1.0f; hit->NdotV = -Rd->x; break;
        case Bottom: hit->normal.y = -1.0f; hit->NdotV = +Rd->y; break;
        case Top:    hit->normal.y = +1.0f; hit->NdotV = -Rd->y; break;
        case Back:   hit->normal.z = -1.0f; hit->NdotV = +Rd->z; break;
        case Front:  hit->normal.z = +1.0f; hit->NdotV = -Rd->z; break;
        default: return NoSide;
    }
    if (hit->from_behind) { hit->normal = vneg(hit->normal); hit->NdotV = -hit->NdotV; }
    hit->area = 4;
    hit->uv_area = 1;
    return side;
}
static vec2 sphere_uv(vec3 d) {                                           /* sphere.h:7 */
    vec2 uv;
    f32 x = d.x, y = d.y, z = d.z;
    f32 zx = x ? (z / x) : 2, yx = x ? (y / x) : 2;
    if (zx <= 1 && zx >= -1 && yx <= 1 && yx >= -1) {
        uv.x = zx;
        uv.y = x > 0 ? yx : -yx;
    } else {
        f32 xz = z ? (x / z) : 2, yz = z ? (y / z) : 2;
        if (xz <= 1 && xz >= -1 && yz <= 1 && yz >= -1) {
            uv.x = -xz;
            uv.y = z > 0 ? yz : -yz;
        } else {
            uv.x = x / (y > 0 ? y : -y);
            uv.y = z / y;
        }
    }
    uv.x += 1; uv.x /= 2;
    uv.y += 1; uv.y /= 2;
    return uv;
}
static bool hit_sphere_simple(vec3 Ro, vec3 Rd, vec3 target, f32 oor, SphereHit *h) { /* sphere.h:44 */
    vec3 rc = vscale(vsub(target, Ro), oor);
    h->b = vdot(Rd, rc);
    h->c = vdot(rc, rc) - 1;
    f32 d = h->b * h->b - h->c;
    if (d < 0) return false;
    d = sqrtf(d);
    h->t_near = h->b - d;
    h->t_far = h->b + d;
    return h->t_far > 0 && h->t_near < h->furthest;
}
static bool hit_sphere(RayHit *hit, const vec3 *Ro, const vec3 *Rd, u8 flags) {  /* sphere.h:61 */
    f32 tc = -vdot(*Ro, *Rd);
    if (tc <= 0) return false;
    hit->distance_squared = vsqlen(*Ro) - tc * tc;
    f32 ds = 1 - hit->distance_squared;
    if (ds <= 0) { hit->distance = tc; return false; }
    f32 delta = sqrtf(ds);
    hit->distance = tc - delta;
    bool outer = hit->distance > 0;
    if (outer) {
        hit->position = vsfma(*Rd, hit->distance, *Ro);
        hit->uv = sphere_uv(hit->position);
        if ((flags & IS_TRANSPARENT) && transparent_uv(hit->uv)) outer = false;
    }
    if (!outer) {
        hit->distance = tc + delta;
        hit->position = vsfma(*Rd, hit->distance, *Ro);
        hit->uv = sphere_uv(hit->position);
        if ((flags & IS_TRANSPARENT) && transparent_uv(hit->uv)) return false;
    }
    hit->from_behind = !outer;
    hit->normal = hit->position;
    hit->NdotV = -vdot(hit->normal, *Rd);
    hit->area = hit->uv_area = UNIT_SPHERE_AREA_OVER_SIX;
    return true;
}
static const f32 TETRA_M[4][9] = {                                        /* tetrahedra.h:55-101 */
    { T_0577, -T_0288, -T_0577,  T_0288,  T_0288,  T_0577, -T_0288,  T_0577, -T_0577},
    { T_0288,  T_0288,  T_0577, -T_0288,  T_0577, -T_0577,  T_0577, -T_0288, -T_0577},
    {-T_0288,  T_0577, -T_0577,  T_0577, -T_0288, -T_0577,  T_0288,  T_0288,  T_0577},
    {-T_0577,  T_0288,  T_0577,  T_0288,  T_0288,  T_0577,  T_0288, -T_0577,  T_0577}};
static bool hit_tetra(RayHit *closest, const vec3 *Ro, const vec3 *Rd, u8 flags) {     /* tetrahedra.h:9 */
    bool found = false;
    f32 cd = INFINITY;
    RayHit hit;
    memset(&hit, 0, sizeof(hit));
    for (int t = 0; t < 4; t++) {
        vec3 tp = splat(t == 3 ? T_0577 : -T_0577);
        hit.normal = tp;
        switch (t) {
            case 0: hit.normal.y = T_0577; break;
            case 1: hit.normal.x = T_0577; break;
            case 2: hit.normal.z = T_0577; break;
            case 3: tp.y = -T_0577; break;
        }
        if (!hit_plane(tp, hit.normal, Ro, Rd, &hit)) continue;
        mat3 m;
        memcpy(&m, TETRA_M[t], sizeof(m));
        hit.position = vsfma(*Rd, hit.distance, *Ro);
        tp = vsub(hit.position, tp);
        tp = vmat3(tp, m);
        if (tp.x < 0 || tp.y < 0 || tp.y + tp.x > 1) continue;
        hit.uv.x = tp.x;
        hit.uv.y = tp.y;
        if ((flags & IS_TRANSPARENT) && transparent_uv(hit.uv)) continue;
        if (hit.distance < cd) {
            cd = hit.distance;
            hit.area = SQRT3 / 4.0f;
            hit.uv_area = 1;
            hit.NdotV = -vdot(hit.normal, *Rd);
            *closest = hit;
            found = true;
        }
    }
    return found;
}
static bool hit_triangles(OTrace *tr, const Ray *ray, RayHit *hit, RayHit *closest, const Triangle *tris,
                          u32 n, bool any_hit) {                             /* mesh.h:5 */
    bool found = false;
    for (u32 i = 0; i < n; i++) {
        const Triangle *t = tris + i;
        CNT(tr, ORC_TRIANGLE_TESTS);
        if (hit_plane(t->position, t->normal, &ray->origin, &ray->direction, hit) && hit->distance < closest->distance) {
            vec3 UV = vsub(hit->position, t->position);
            UV = vmat3(UV, t->world_to_tangent);
            if (UV.x < 0 || UV.y < 0 || (UV.x + UV.y) > 1) continue;
            closest->NdotV = hit->NdotV;
            closest->normal = hit->normal;
            closest->uv.x = UV.x;
            closest->uv.y = UV.y;
            closest->object_id = i;
            closest->from_behind = hit->from_behind;
            closest->distance = hit->distance;
            closest->position = hit->position;
            closest->area = t->area_of_parallelogram;
            closest->uv_area = t->area_of_uv;
            found = true;
            if (any_hit) break;
        }
    }
    return found;
}
static bool trace_mesh(OTrace *tr, const Mesh *mesh, bool any_hit) {      /* mesh.h:38 */
    Ray *ray = &tr->local;
    RayHit *closest = &tr->closest_mesh_hit, *hit = &tr->current_hit;
    u32 *stack = tr->mesh_stack;
    bool found = false;
    f32 ld, rd;
    CNT(tr, ORC_MESH_ENTRIES);
    CNT(tr, ORC_AABB_TESTS);
    if (!hit_aabb(&mesh->bvh.nodes->aabb, ray, closest->distance, &ld)) return false;
    if (mesh->bvh.nodes->child_count)
        return hit_triangles(tr, ray, hit, closest, mesh->triangles, mesh->triangle_count, any_hit);
    const BVHNode *left = mesh->bvh.nodes + mesh->bvh.nodes->first_child_id, *right, *tmp;
    u32 sp = 0;
    for (;;) {
        right = left + 1;
        tr->cnt[ORC_AABB_TESTS] += 2;
        bool hl = hit_aabb(&left->aabb, ray, closest->distance, &ld);
        bool hr = hit_aabb(&right->aabb, ray, closest->distance, &rd);
        if (hl) {
            if (left->child_count) {
                if (hit_triangles(tr, ray, hit, closest, mesh->triangles + left->first_child_id, left->child_count, any_hit)) {
                    closest->object_id += left->first_child_id;
                    found = true;
                    if (any_hit) break;
                }
                left = NULL;
            }
        } else left = NULL;
        if (hr) {
            if (right->child_count) {
                if (hit_triangles(tr, ray, hit, closest, mesh->triangles + right->first_child_id, right->child_count, any_hit)) {
                    closest->object_id += right->first_child_id;
                    found = true;
                    if (any_hit) break;
                }
                right = NULL;
            }
        } else right = NULL;
        if (left) {
            if (right) {
                if (!any_hit && ld > rd) { tmp = left; left = right; right = tmp; }
                stack[sp++] = right->first_child_id;
                if (sp == tr->mesh_stack_size) return false;
            }
            left = mesh->bvh.nodes + left->first_child_id;
        } else if (right) {
            left = mesh->bvh.nodes + right->first_child_id;
        } else {
            if (sp == 0) break;
            left = mesh->bvh.nodes + stack[--sp];
        }
    }
    return found;
}
/* hitPrimitives intersection/primitives.h:9 */
static bool hit_primitives(OTrace *tr, const Ray *ray, const Scene *sc, const u32 *ids, u32 count,
                           bool any_hit, bool check_vis, u16 x, u16 y) {
    bool cur = false, found = false;
    vec3 *Rd = &tr->local.direction, *Ro = &tr->local.origin;
    RayHit *hit = &tr->current_hit, *closest = &tr->closest_hit;
    f32 cone_angle = closest->cone_angle;
    const Primitive *hp = NULL;
    u32 hid = 0;
    for (u32 i = 0; i < count; i++) {
        CNT(tr, ORC_LEAF_ID_READS);
        u32 pid = ids[i];
        const Primitive *p = sc->primitives + pid;
        if (any_hit && !(p->flags & IS_SHADOWING)) continue;
        if (check_vis) {
            if (!(p->flags & IS_VISIBLE)) continue;
            if (x < p->screen_bounds.min.x || x >= p->screen_bounds.max.x ||
                y < p->screen_bounds.min.y || y >= p->screen_bounds.max.y) continue;
        }
        CNT(tr, ORC_PRIMITIVE_TESTS);
        to_object(ray->origin, ray->direction, p, Ro, Rd);
        *Ro = vsfma(*Rd, TRACE_OFFSET, *Ro);
        switch (p->type) {
            case PrimitiveType_Quad: cur = hit_quad(hit, Ro, Rd, p->flags); break;
            case PrimitiveType_Box: cur = hit_box(hit, Ro, Rd, p->flags) != NoSide; break;
            case PrimitiveType_Sphere: cur = hit_sphere(hit, Ro, Rd, p->flags); break;
            case PrimitiveType_Tetrahedron: cur = hit_tetra(hit, Ro, Rd, p->flags); break;
            case PrimitiveType_Mesh:
                tr->local.direction_reciprocal = vrcp(*Rd);
                tr->closest_mesh_hit.distance = closest->distance == INFINITY ? INFINITY :
                    vlen(vsub(pos_to_object(closest->position, p), *Ro));
                pre_prep(&tr->local);
                cur = trace_mesh(tr, sc->meshes + p->id, any_hit);
                if (cur) *hit = tr->closest_mesh_hit;
                break;
            default: continue;
        }
        if (cur) {
            hit->position = pos_to_world(hit->position, p);
            hit->distance_squared = vsqlen(vsub(hit->position, ray->origin));
            if (hit->distance_squared < closest->distance_squared) {
                *closest = *hit;
                hid = pid;
                hp = p;
                closest->object_type = p->type;
                closest->material_id = p->material_id;
                found = true;
                if (any_hit) break;
            }
        }
    }
    if (found) {
        if (closest->object_type == PrimitiveType_Mesh) {
            const Mesh *mesh = sc->meshes + hp->id;
            const Triangle *t = mesh->triangles + closest->object_id;
            if (mesh->normals_count | mesh->uvs_count) {
                f32 u = closest->uv.x, v = closest->uv.y;
                f32 w = 1 - u - v;
                if (mesh->uvs_count) {
                    closest->uv.x = t->uvs[2].x * u + (t->uvs[1].x * v + t->uvs[0].x * w);
                    closest->uv.y = t->uvs[2].y * u + (t->uvs[1].y * v + t->uvs[0].y * w);
                }
                if (mesh->normals_count) {
                    closest->normal.x = t->vertex_normals[2].x * u + (t->vertex_normals[1].x * v + t->vertex_normals[0].x * w);
                    closest->normal.y = t->vertex_normals[2].y * u + (t->vertex_normals[1].y * v + t->vertex_normals[0].y * w);
                    closest->normal.z = t->vertex_normals[2].z * u + (t->vertex_normals[1].z * v + t->vertex_normals[0].z * w);
                    closest->normal = vnorm(closest->normal);
                }
            }
        }
        closest->object_id = hid;
        closest->normal = vnorm(dir_to_world(closest->normal, hp));
        closest->distance = sqrtf(closest->distance_squared);
        closest->cone_width = 2.0f * cone_angle * closest->distance;
        vec3 rs = qrot(hp->scale, hp->rotation);
        closest->area *= vdot(vone_minus(closest->normal), rs);
    }
    return found;
}
/* traceScene shaders/trace.h:8 */
static bool trace_scene(OTrace *tr, Ray *ray, const Scene *sc, bool any_hit) {
    ray->direction_reciprocal = vrcp(ray->direction);
    pre_prep(ray);
    bool found = false;
    f32 ld, rd;
    CNT(tr, ORC_AABB_TESTS);
    if (!hit_aabb(&sc->bvh.nodes->aabb, ray, tr->closest_hit.distance, &ld)) return false;
    if (sc->bvh.nodes->child_count)
        return hit_primitives(tr, ray, sc, sc->bvh.leaf_ids, sc->settings.primitives, any_hit, false, 0, 0);
    const BVHNode *left = sc->bvh.nodes + sc->bvh.nodes->first_child_id, *right, *tmp;
    u32 *stack = tr->scene_stack, sp = 0;
    for (;;) {
        right = left + 1;
        tr->cnt[ORC_AABB_TESTS] += 2;
        bool hl = hit_aabb(&left->aabb, ray, tr->closest_hit.distance, &ld);
        bool hr = hit_aabb(&right->aabb, ray, tr->closest_hit.distance, &rd);
        if (hl) {
            if (left->child_count) {
                if (hit_primitives(tr, ray, sc, sc->bvh.leaf_ids + left->first_child_id, left->child_count, any_hit, false, 0, 0)) {
                    found = true;
                    if (any_hit) break;
                }
                left = NULL;
            }
        } else left = NULL;
        if (hr) {
            if (right->child_count) {
                if (hit_primitives(tr, ray, sc, sc->bvh.leaf_ids + right->first_child_id, right->child_count, any_hit, false, 0, 0)) {
                    found = true;
                    if (any_hit) break;
                }
                right = NULL;
            }
        } else right = NULL;
        if (left) {
            if (right) {
                if (!any_hit && ld > rd) { tmp = left; left = right; right = tmp; }
                if (sp < ORC_STACK) stack[sp++] = right->first_child_id;
            }
            left = sc->bvh.nodes + left->first_child_id;
        } else if (right) {
            left = sc->bvh.nodes + right->first_child_id;
        } else {
            if (sp == 0) break;
            left = sc->bvh.nodes + stack[--sp];
        }
    }
    return found;
}
static inline bool in_shadow(OTrace *tr, Ray *ray, const Scene *sc) {    /* trace.h:85 */
    CNT(tr, ORC_SHADOW_RAYS);
    return trace_scene(tr, ray, sc, true);
}
static inline bool trace_ray(OTrace *tr, Ray *ray, const Scene *sc) {     /* trace.h:89 */
    CNT(tr, ORC_BOUNCE_RAYS);
    tr->closest_hit.distance = tr->closest_hit.distance_squared = INFINITY;
    return trace_scene(tr, ray, sc, false);
}

/* ---- closest-hit shaders: closest_hit/surface.h, lights.h, debug.h -------------------------- */
static vec3 shade_from_lights(OShaded *s, Ray *ray, OTrace *tr, const Scene *sc, vec3 color) { /* surface.h:9 */
    RayHit *hit = &tr->closest_hit;
    const Light *light = sc->lights;
    for (u32 i = 0; i < sc->settings.lights; i++, light++) {
        hit->position = light->position_or_direction;
        s->light_direction = vsub(hit->position, s->position);
        hit->distance_squared = vsqlen(s->light_direction);
        hit->distance = sqrtf(hit->distance_squared);
        s->light_direction = vscale(s->light_direction, 1.0f / hit->distance);
        f32 NdotL = vdot(s->normal, s->light_direction);
        if (NdotL <= 0) continue;
        f32 li = light->intensity / hit->distance_squared;
        ray->origin = s->position;
        ray->direction = s->light_direction;
        if (in_shadow(tr, ray, sc)) continue;
        color = vvfma(shade_point(s, NdotL), vscale(light->color, li), color);
    }
    return color;
}
static bool shade_from_emissive_quads(OShaded *s, Ray *ray, OTrace *tr, const Scene *sc, vec3 *color) { /* surface.h:37 */
    RayHit *hit = &tr->current_hit;
    const Primitive *quad = sc->primitives;
    vec3 *Rd = &tr->local.direction, *Ro = &tr->local.origin;
    bool found = false;
    for (u32 i = 0; i < sc->settings.primitives; i++, quad++) {
        const Material *em = sc->materials + quad->material_id;
        if (quad->type != PrimitiveType_Quad || !(em->is & EMISSIVE)) continue;
        to_object(s->viewing_origin, s->viewing_direction, quad, Ro, Rd);
        if (hit_quad(hit, Ro, Rd, quad->flags)) {
            hit->position = pos_to_world(hit->position, quad);
            hit->distance_squared = vsqlen(vsub(hit->position, s->viewing_origin));
            if (hit->distance_squared < tr->closest_hit.distance_squared) {
                hit->object_id = i;
                hit->object_type = PrimitiveType_Quad;
                hit->material_id = quad->material_id;
                tr->closest_hit = *hit;
                found = true;
            }
        }
        vec3 qn = V3(0, 1, 0);
        qn = qrot(qn, quad->rotation);
        s->light_direction = ray->direction = vsub(quad->position, s->position);
        if (vdot(qn, s->light_direction) >= 0) continue;
        f32 ei = vdot(s->normal, area_light_vector(quad, s->position, s->emissive_quad_vertices));
        if (ei > 0) {
            bool skip = true;
            for (int j = 0; j < 4; j++)
                if (vdot(s->normal, vsub(s->emissive_quad_vertices[j], s->position)) >= 0) { skip = false; break; }
            if (skip) continue;
            f32 shaded_light = 1;
            const Primitive *sp = sc->primitives;
            for (u32 k = 0; k < sc->settings.primitives; k++, sp++) {
                if (quad == s->primitive || quad == sp || vdot(qn, vsub(sp->position, quad->position)) <= 0) continue;
                to_object(s->position, s->light_direction, sp, Ro, Rd);
                *Ro = vsfma(*Rd, TRACE_OFFSET, *Ro);
                f32 d = 1;
                if (sp->type == PrimitiveType_Sphere) {
                    if (hit_sphere(hit, Ro, Rd, sp->flags))
                        d -= (1.0f - sqrtf(hit->distance_squared)) / (hit->distance * ei * 3);
                } else if (sp->type == PrimitiveType_Quad) {
                    if (hit_quad(hit, Ro, Rd, sp->flags)) {
                        hit->position.y = 0;
                        hit->position.x = hit->position.x < 0 ? -hit->position.x : hit->position.x;
                        hit->position.z = hit->position.z < 0 ? -hit->position.z : hit->position.z;
                        if (hit->position.x > hit->position.z) {
                            hit->position.y = hit->position.z;
                            hit->position.z = hit->position.x;
                            hit->position.x = hit->position.y;
                            hit->position.y = 0;
                        }
                        d -= (1.0f - hit->position.z) / (hit->distance * ei);
                    }
                }
                if (d < shaded_light) shaded_light = d;
            }
            if (shaded_light > 0) {
                f32 NdotL = vdot01(s->normal, s->light_direction);
                if (NdotL)
                    *color = vvfma(shade_point(s, NdotL), vscale(em->emission, ei * shaded_light), *color);
            }
        }
    }
    if (found) tr->closest_hit.distance = sqrtf(tr->closest_hit.distance_squared);
    return found;
}
static f32 volume_density(const SphereHit *h) {                          /* lights.h:7 */
    f32 t1 = h->t_near > 0 ? h->t_near : 0;
    f32 t2 = h->t_far < h->furthest ? h->t_far : h->furthest;
    return (h->c * t1 - h->b * t1 * t1 + t1 * t1 * t1 / 3.0f - (
            h->c * t2 - h->b * t2 * t2 + t2 * t2 * t2 / 3.0f)) * (3.0f / 4.0f);
}
static bool shade_lights(const Light *lights, u32 n, vec3 Ro, vec3 Rd, f32 max_distance, SphereHit *sh, vec3 *color) { /* lights.h:17 */
    bool hit_light = false;
    sh->closest_hit_distance = INFINITY;
    for (u32 i = 0; i < n; i++) {
        const Light *light = lights + i;
        f32 size = light->intensity * (1.0f / 16.0f);
        f32 oor = 8.0f / size;
        sh->furthest = max_distance * oor;
        if (hit_sphere_simple(Ro, Rd, light->position_or_direction, oor, sh)) {
            f32 distance = sh->t_far - size * 8;
            f32 density = powf(volume_density(sh), 8) * 8;
            if (distance < sh->closest_hit_distance) {
                sh->closest_hit_distance = distance;
                sh->closest_hit_density = density;
            }
            *color = vsfma(light->color, density, *color);
            hit_light = true;
        }
    }
    return hit_light;
}
static void apply_textures(OShaded *s, RayHit *hit, const Material *M, const Scene *sc, vec2 *dUV, bool first, OTrace *tr) {
    s->uv.x = hit->uv.x * M->uv_repeat.x;
    s->uv.y = hit->uv.y * M->uv_repeat.y;
    hit->uv_area /= M->uv_repeat.x / M->uv_repeat.y;
    f32 d = duv_ray_cone(hit->NdotV, hit->cone_width, hit->area, hit->uv_area);
    dUV->x = d;
    if (first) dUV->y = d;       /* surface.h:162 sets both; the bounce path (:230) only .u */
    if (M->use & ALBEDO_MAP) s->albedo = sample_texture(sc->textures + M->texture_ids[0], s->uv, *dUV, tr);
    if ((M->use & NORMAL_MAP) && M->texture_count > 1) {
        quat rot = normal_rotation(sample_normal(sc->textures + M->texture_ids[1], s->uv, *dUV, tr));
        hit->normal = qrot(hit->normal, rot);
    }
}
static vec3 shade_surface(Ray *ray, OTrace *tr, const Scene *sc, bool *lights_shaded) {  /* surface.h:146 */
    RayHit *hit = &tr->closest_hit;
    vec3 color = splat(0);
    const Material *M = sc->materials + hit->material_id;
    CNT(tr, ORC_SHADED_HITS);
    if (M->is & EMISSIVE) return hit->from_behind ? color : M->emission;
    vec2 dUV;
    dUV.x = dUV.y = 0;
    OShaded s;
    memset(&s, 0, sizeof(s));
    s.viewing_origin = ray->origin;
    s.viewing_direction = ray->direction;
    s.primitive = sc->primitives + hit->object_id;
    s.material = M;
    s.albedo = M->albedo;
    if (M->use && M->texture_count) apply_textures(&s, hit, M, sc, &dUV, true, tr);
    f32 NdotRd = 0, ior, max_distance = hit->distance;
    bool has_emissive_quads = false;
    for (u32 i = 0; i < sc->settings.primitives; i++)
        if (sc->primitives[i].type == PrimitiveType_Quad && (sc->materials[sc->primitives[i].material_id].is & EMISSIVE)) {
            has_emissive_quads = true;
            break;
        }
    vec3 current, throughput = splat(1);
    u32 depth = tr->depth;
    while (depth) {
        s.position = ray->origin = hit->position;
        s.normal = hit->from_behind ? vneg(hit->normal) : hit->normal;
        ior = hit->from_behind ? s.material->n2_over_n1 : s.material->n1_over_n2;
        bool is_ref = (M->is & REFLECTIVE) || (M->is & REFRACTIVE);
        if (is_ref || M->brdf == BRDF_Phong) {
            NdotRd = -inv_dot(s.normal, s.viewing_direction);
            s.reflected_direction = reflect_dot(s.viewing_direction, s.normal, NdotRd);
        }
        current = is_ref ? splat(0) : sc->ambient_light.color;
        if (sc->lights) current = shade_from_lights(&s, ray, tr, sc, current);
        if (has_emissive_quads)
            if (shade_from_emissive_quads(&s, ray, tr, sc, &current)) max_distance = hit->distance;
        color = vvfma(current, throughput, color);
        if (sc->lights && shade_lights(sc->lights, sc->settings.lights, s.viewing_origin, s.viewing_direction,
                                       max_distance, &tr->sphere_hit, &color))
            *lights_shaded = true;
        if (is_ref && --depth) {
            if (M->is & REFLECTIVE) ray->direction = s.reflected_direction;
            else {
                ray->direction = refract_dir(s.viewing_direction, s.normal, ior, NdotRd);
                if (ray->direction.x == 0 && ray->direction.y == 0 && ray->direction.z == 0)
                    ray->direction = s.reflected_direction;
            }
            if (trace_ray(tr, ray, sc)) {
                CNT(tr, ORC_SHADED_HITS);
                s.primitive = sc->primitives + hit->object_id;
                s.material = M = sc->materials + hit->material_id;
                s.albedo = M->albedo;
                if (M->use && M->texture_count) apply_textures(&s, hit, M, sc, &dUV, false, tr);
                if (hit->object_type == PrimitiveType_Quad && (M->is & EMISSIVE)) {
                    color = hit->from_behind ? splat(0) : M->emission;
                    break;
                }
                if (M->brdf != BRDF_CookTorrance) throughput = vmul(throughput, M->reflectivity);
                s.viewing_origin = ray->origin;
                s.viewing_direction = ray->direction;
                continue;
            }
        }
        break;
    }
    return color;
}

/* setPixel core/types.h:422 */
static void set_pixel(FloatPixel *pixel, vec3 color, f32 opacity, f64 depth) {
    FloatPixel np;
    np.opacity = opacity;
    np.color = color;
    np.depth = depth;
    if (!(opacity == 1 && depth == 0)) {
        FloatPixel bg, fg, old = *pixel;
        if (old.depth < np.depth) { bg = np; fg = old; } else { bg = old; fg = np; }
        if (fg.opacity != 1) {
            f32 omf = 1.0f - fg.opacity;
            opacity = fg.opacity + bg.opacity * omf;
            f32 oo = opacity ? 1.0f / opacity : 1;
            f32 bf = bg.opacity * oo * omf;
            f32 ff = fg.opacity * oo;
            pixel->color.x = fg.color.x * ff + bg.color.x * bf;
            pixel->color.y = fg.color.y * ff + bg.color.y * bf;
            pixel->color.z = fg.color.z * ff + bg.color.z * bf;
            pixel->opacity = opacity;
            pixel->depth = fg.depth;
        } else *pixel = fg;
    } else *pixel = np;
}

/* rayTrace render/raytracer.h:81 */
static void ray_trace(Ray *ray, OTrace *tr, const Scene *sc, int mode, FloatPixel *pixel, u16 x, u16 y,
                      vec3 cam_pos, quat cam_rot, uint32_t *prim_id) {
    RayHit *hit = &tr->closest_hit;
    vec3 Ro = ray->origin, Rd = ray->direction, color = splat(0);
    bool lights_shaded = false;
    CNT(tr, ORC_PRIMARY_RAYS);
    bool hit_found = hit_primitives(tr, ray, sc, sc->bvh.leaf_ids, sc->settings.primitives, false, true, x, y);
    if (prim_id) *prim_id = hit_found ? hit->object_id : 0xFFFFFFFFu;
    f32 closest_distance = hit_found ? hit->distance : INFINITY;
    f32 z = INFINITY;
    if (hit_found) {
        z = qrot(vsub(hit->position, cam_pos), cam_rot).z;
        switch (mode) {
            case RenderMode_Beauty: color = shade_surface(ray, tr, sc, &lights_shaded); break;
            case RenderMode_Depth: color = splat(4 / hit->distance); break;
            case RenderMode_Normals: {
                const Material *M = sc->materials + hit->material_id;
                if (M->texture_count > 1 && (M->use & NORMAL_MAP)) {
                    vec2 uv;
                    uv.x = hit->uv.x * M->uv_repeat.x;
                    uv.y = hit->uv.y * M->uv_repeat.y;
                    hit->uv_area /= M->uv_repeat.x / M->uv_repeat.y;
                    vec2 dUV;
                    dUV.x = duv_ray_cone(hit->NdotV, hit->cone_width, hit->area, hit->uv_area);
                    dUV.y = 0; /* raytracer.h:103-104 leaves dUV.v unset */
                    quat rot = normal_rotation(sample_normal(sc->textures + M->texture_ids[1], uv, dUV, tr));
                    hit->normal = qrot(hit->normal, rot);
                }
                color = V3(0.5f * (hit->normal.x + 1), 0.5f * (hit->normal.y + 1), 0.5f * (hit->normal.z + 1));
            } break;
            case RenderMode_UVs: color = V3(0.5f * hit->uv.x, 0.5f * hit->uv.y, 0.5f); break;
        }
    }
    if (mode == RenderMode_Beauty && sc->lights && !lights_shaded) {
        if (shade_lights(sc->lights, sc->settings.lights, Ro, Rd, closest_distance, &tr->sphere_hit, &color)) {
            hit_found = true;
            z = tr->sphere_hit.closest_hit_distance;
        }
    }
    if (hit_found) {
        if (mode == RenderMode_Beauty) {
            color.x = tone_mapped(color.x);
            color.y = tone_mapped(color.y);
            color.z = tone_mapped(color.z);
        }
        color = vscale(color, FLOAT_TO_COLOR_COMPONENT);
        color = vmul(color, color);
        set_pixel(pixel, color, 1, z);
    }
}

/* ---- frame: renderSceneOnCPU raytracer.h:136, fillViewport viewport.h:68, resolve :12 -------- */
typedef struct {
    const Scene *scene;
    Viewport *vp;
    vec3 *row_starts;
    uint32_t *prim_ids;
    uint64_t counters[ORC_COUNTERS];
    u32 next_row;
    pthread_mutex_t lock;
} OJob;

static void *render_rows(void *arg) {
    OJob *job = (OJob*)arg;
    Viewport *vp = job->vp;
    Dimensions *dim = &vp->frame_buffer->dimensions;
    OTrace *tr = (OTrace*)calloc(1, sizeof(OTrace));
    tr->depth = vp->trace.depth;
    tr->mesh_stack_size = 255;
    tr->closest_mesh_hit.object_type = job->scene->settings.meshes ? PrimitiveType_Mesh : 0;
    quat cam_rot = vp->camera->transform.rotation_inverted;
    vec3 cam_pos = vp->camera->transform.position;
    vec3 right = vp->projection_plane.right;
    Ray ray;
    memset(&ray, 0, sizeof(ray));
    for (;;) {
        pthread_mutex_lock(&job->lock);
        u32 y = job->next_row++;
        pthread_mutex_unlock(&job->lock);
        if (y >= dim->height) break;
        vec3 current = job->row_starts[y];
        u32 base = y * dim->width;
        for (u16 x = 0; x < dim->width; x++) {
            ray.origin = cam_pos;
            ray.direction = vnorm(current);
            ray.direction_reciprocal = vrcp(ray.direction);
            tr->closest_hit.distance = tr->closest_hit.distance_squared = INFINITY;
            tr->closest_hit.cone_angle = vp->projection_plane.cone_angle;
            tr->closest_hit.cone_width = 0;
            ray_trace(&ray, tr, job->scene, vp->settings.render_mode, vp->frame_buffer->float_pixels + base + x,
                      x, (u16)y, cam_pos, cam_rot, job->prim_ids ? job->prim_ids + base + x : NULL);
            current = vadd(current, right);
        }
    }
    pthread_mutex_lock(&job->lock);
    for (int k = 0; k < ORC_COUNTERS; k++) job->counters[k] += tr->cnt[k];
    pthread_mutex_unlock(&job->lock);
    free(tr);
    return NULL;
}

static void resolve(Viewport *vp) {                                     /* viewport.h:12 (QCAA branch) */
    PixelGrid *fb = vp->frame_buffer;
    u16 stride = fb->dimensions.width, width = stride - 1, height = fb->dimensions.height - 1;
    for (u16 y = 0; y < height; y++) {
        const FloatPixel *TL = fb->float_pixels + (u32)y * stride;
        for (u16 x = 0; x < width; x++, TL++) {
            const FloatPixel *TR = TL + 1, *BL = TL + stride, *BR = BL + 1;
            Pixel *out = fb->pixels + (u32)y * width + x;
            if (BL->depth == INFINITY && BR->depth == INFINITY && TL->depth == INFINITY && TR->depth == INFINITY) {
                out->color.R = out->color.G = out->color.B = 0;
            } else {
                vec3 c = vscale(vsfma(TL->color, TL->opacity, vsfma(TR->color, TR->opacity,
                          vsfma(BL->color, BL->opacity, vscale(BR->color, BR->opacity)))), 0.25f);
                out->color.R = (u8)(c.x > (255 * 255) ? 255 : sqrt(c.x));
                out->color.G = (u8)(c.y > (255 * 255) ? 255 : sqrt(c.y));
                out->color.B = (u8)(c.z > (255 * 255) ? 255 : sqrt(c.z));
            }
            out->color.A = 255;
        }
    }
}

int orc_render_frame(const Scene *scene, Viewport *vp, int threads, uint32_t *prim_ids, uint64_t *counters) {
    Dimensions *dim = &vp->frame_buffer->dimensions;
    FloatPixel clear;
    clear.color = splat(0);
    clear.opacity = 0;
    clear.depth = INFINITY;
    for (u32 i = 0; i < (u32)dim->width * dim->height; i++) vp->frame_buffer->float_pixels[i] = clear;
    OJob job;
    memset(&job, 0, sizeof(job));
    job.scene = scene;
    job.vp = vp;
    job.prim_ids = prim_ids;
    job.row_starts = (vec3*)malloc(sizeof(vec3) * (dim->height ? dim->height : 1));
    vec3 start = vp->projection_plane.start;
    for (u32 y = 0; y < dim->height; y++) { job.row_starts[y] = start; start = vadd(start, vp->projection_plane.down); }
    pthread_mutex_init(&job.lock, NULL);
    if (threads <= 1) render_rows(&job);
    else {
        pthread_t *t = (pthread_t*)malloc(sizeof(pthread_t) * threads);
        for (int i = 0; i < threads; i++) pthread_create(&t[i], NULL, render_rows, &job);
        for (int i = 0; i < threads; i++) pthread_join(t[i], NULL);
        free(t);
    }
    pthread_mutex_destroy(&job.lock);
    free(job.row_starts);
    if (vp->frame_buffer->pixels) resolve(vp);
    if (counters) memcpy(counters, job.counters, sizeof(job.counters));
    return 0;
}

/* ---- screen-space bounds: render/SSB.h:5-173 -------------------------------------------------- */
static bool compute_ssb(Rect *b, const vec3 *pos, f32 r, f32 fl, const Dimensions *d) {
    b->min.x = d->width + 1;
    b->max.x = d->width + 1;
    b->min.y = d->height + 1;
    b->max.y = d->height + 1;
    if (pos->z <= -r) return false;
    f32 x = pos->x, y = pos->y, z = pos->z, left, right, top, bottom, factor;
    if (z <= r) {
        f32 h = fabsf(z) / fl;
        top = y + r;
        bottom = y - r;
        if (h < bottom || top < -h) return false;
        f32 w = h * d->width_over_height;
        right = x + r;
        left = x - r;
        if (w < left || right < -w) return false;
        b->min.x = -w < left ? (u16)(d->f_width * (left + w) / (2 * w)) : 0;
        b->max.x = right < w ? (u16)(d->f_width * (right + w) / (2 * w)) : d->width;
        b->min.y = top < h ? (u16)(d->f_height * (h - top) / (2 * h)) : 0;
        b->max.y = -h < bottom ? (u16)(d->f_height * (h - bottom) / (2 * h)) : d->height;
        return true;
    }
    f32 den = z * z - r * r;
    factor = fl / den;
    f32 yz = y * z;
    f32 sqr = y * y + den;
    sqr = r * sqrtf(sqr);
    bottom = factor * (yz - sqr);
    top = factor * (yz + sqr);
    if (bottom < 1 && top > -1) {
        factor *= d->height_over_width;
        f32 xz = x * z;
        sqr = r * sqrtf(x * x + den);
        left = factor * (xz - sqr);
        right = factor * (xz + sqr);
        if (left < 1 && right > -1) {
            bottom = bottom > -1 ? bottom : -1; bottom += 1;
            top = top < 1 ? top : 1; top += 1;
            left = left > -1 ? left : -1; left += 1;
            right = right < 1 ? right : 1; right += 1;
            top = 2 - top;
            bottom = 2 - bottom;
            b->min.x = (u16)(d->h_width * left);
            b->max.x = (u16)(d->h_width * right);
            b->max.y = (u16)(d->h_height * bottom);
            b->min.y = (u16)(d->h_height * top);
            return true;
        }
    }
    return false;
}

void orc_update_scene_ssb(Scene *sc, const Viewport *vp) {
    const xform3 *xf = &vp->camera->transform;
    for (u32 i = 0; i < sc->settings.primitives; i++) {
        Primitive *p = sc->primitives + i;
        f32 radius, mn, mx;
        vec3 view = vmat3(vsub(p->position, xf->position), xf->rotation_matrix_inverted);
        switch (p->type) {
            case PrimitiveType_Quad: radius = vlen(p->scale); break;
            case PrimitiveType_Box: radius = vlen(p->scale); break;
            case PrimitiveType_Tetrahedron: radius = maxcoord(p->scale) * SQRT2; break;
            case PrimitiveType_Sphere: radius = maxcoord(p->scale); break;
            case PrimitiveType_Mesh: {
                const AABB *a = &sc->meshes[p->id].aabb;
                mn = vlen(vmul(p->scale, a->min));
                mx = vlen(vmul(p->scale, a->max));
                radius = mx > mn ? mx : mn;
            } break;
            default: continue;
        }
        p->flags &= ~IS_VISIBLE;
        if (compute_ssb(&p->screen_bounds, &view, radius, vp->camera->focal_length, &vp->frame_buffer->dimensions))
            p->flags |= IS_VISIBLE;
    }
}

/* ---- top-down SAH builder: acceleration_structures/builder_top_down.h:25-380 ---------------- */
typedef struct { AABB *laabb, *raabb; f32 *lsa, *rsa; u32 left_count, *sorted; f32 best; } OAxis;
typedef struct { u32 start, end, node_id; } OIter;
typedef struct { OIter *iters; BVHNode *leaf_nodes; u32 *leaf_ids; i32 *sort_stack; OAxis axis[3]; } OBuilder;

static void builder_init(OBuilder *b, u32 n) {
    b->iters = (OIter*)calloc(n, sizeof(OIter));
    b->leaf_nodes = (BVHNode*)calloc(n, sizeof(BVHNode));
    b->leaf_ids = (u32*)calloc(n, sizeof(u32));
    b->sort_stack = (i32*)calloc(n + 2, sizeof(i32));
    for (int a = 0; a < 3; a++) {
        b->axis[a].sorted = (u32*)calloc(n, sizeof(u32));
        b->axis[a].laabb = (AABB*)calloc(n, sizeof(AABB));
        b->axis[a].raabb = (AABB*)calloc(n, sizeof(AABB));
        b->axis[a].lsa = (f32*)calloc(n, sizeof(f32));
        b->axis[a].rsa = (f32*)calloc(n, sizeof(f32));
    }
}
static void builder_free(OBuilder *b) {
    free(b->iters); free(b->leaf_nodes); free(b->leaf_ids); free(b->sort_stack);
    for (int a = 0; a < 3; a++) {
        free(b->axis[a].sorted); free(b->axis[a].laabb); free(b->axis[a].raabb); free(b->axis[a].lsa); free(b->axis[a].rsa);
    }
}
static inline f32 key_max(const BVHNode *n, int axis) { return axis == 0 ? n->aabb.max.x : axis == 1 ? n->aabb.max.y : n->aabb.max.z; }
/* partitionNodesByAxis :66 — Lomuto, pivot = last */
static i32 lomuto(const BVHNode *nodes, int axis, i32 start, i32 end, u32 *ids) {
    i32 p = start, t;
    i32 pivot = (i32)ids[end];
    for (i32 i = start; i < end; i++) {
        if (key_max(&nodes[ids[i]], axis) < key_max(&nodes[pivot], axis)) {
            t = (i32)ids[i]; ids[i] = ids[p]; ids[p] = (u32)t; p++;
        }
    }
    t = (i32)ids[end]; ids[end] = ids[p]; ids[p] = (u32)t;
    return p;
}
/* sortNodesByAxis :92 — iterative quicksort, explicit stack, left range pushed first */
static void quicksort(const BVHNode *nodes, int axis, i32 start, i32 end, i32 *stack, u32 *ids) {
    i32 top = -1;
    stack[++top] = start;
    stack[++top] = end;
    while (top >= 0) {
        end = stack[top--];
        start = stack[top--];
        i32 p = lomuto(nodes, axis, start, end, ids);
        if (p - 1 > start) { stack[++top] = start; stack[++top] = p - 1; }
        if (p + 1 < end) { stack[++top] = p + 1; stack[++top] = end; }
    }
}
/* partitionBVHNodeIDs :125 */
static void partition_ids(OAxis *pa, int axis, const BVHNode *nodes, i32 *stack, u32 N) {
    u32 li = 0, ri = N - 1, ci, ni;
    quicksort(nodes, axis, 0, (i32)N - 1, stack, pa->sorted);
    AABB L = nodes[pa->sorted[li]].aabb, R = nodes[pa->sorted[ri]].aabb;
    pa->laabb[li] = L;
    pa->raabb[ri] = R;
    for (li = 0; li < N; li++, ri--) {
        if (li) {
            L = merge_aabb(L, nodes[pa->sorted[li]].aabb);
            R = merge_aabb(R, nodes[pa->sorted[ri]].aabb);
            pa->laabb[li] = L;
            pa->raabb[ri] = R;
        }
        pa->lsa[li] = half_area(L);
        pa->rsa[ri] = half_area(R);
    }
    u32 last = ri = N - 1;
    pa->left_count = li = ni = 1;
    pa->best = INFINITY;
    for (ci = 0; ci < last; ci++, ni++, li++, ri--) {
        f32 cost = pa->lsa[ci] * (f32)li + pa->rsa[ni] * (f32)ri;
        if (pa->best > cost) { pa->best = cost; pa->left_count = ni; }
    }
}
static void init_node(BVHNode *n) { memset(n, 0, sizeof(*n)); }
/* splitBVHNode :168 */
static u32 split_node(BVHNode *nodes, u32 *node_count, OBuilder *b, BVHNode *node, u32 start, u32 end) {
    u32 N = end - start;
    u32 *ids = b->leaf_ids + start;
    node->first_child_id = *node_count;
    BVHNode *l = nodes + (*node_count)++;
    BVHNode *r = nodes + (*node_count)++;
    init_node(l);
    init_node(r);
    f32 best = INFINITY;
    OAxis *chosen = b->axis;
    for (int a = 0; a < 3; a++) {
        OAxis *pa = b->axis + a;
        for (u32 i = 0; i < N; i++) pa->sorted[i] = ids[i];
        partition_ids(pa, a, b->leaf_nodes, b->sort_stack, N);
        if (pa->best < best) { best = pa->best; chosen = pa; }
    }
    u32 lc = chosen->left_count;
    l->aabb = chosen->laabb[lc - 1];
    r->aabb = chosen->raabb[lc];
    for (u32 i = 0; i < N; i++) ids[i] = chosen->sorted[i];
    return start + lc;
}
/* buildBVH :204 */
static void build_bvh(BVH *bvh, OBuilder *b, u32 N, u16 max_leaf) {
    bvh->node_count = 1;
    init_node(bvh->nodes);
    if (N <= max_leaf) {
        bvh->nodes->aabb.min = splat(INFINITY);
        bvh->nodes->aabb.max = splat(-INFINITY);
        for (u32 i = 0; i < N; i++) {
            bvh->leaf_ids[i] = b->leaf_nodes[i].first_child_id;
            bvh->nodes->aabb = merge_aabb(bvh->nodes->aabb, b->leaf_nodes[i].aabb);
        }
        bvh->nodes->depth = 0;
        bvh->nodes->child_count = (u16)N;
        bvh->nodes->first_child_id = 0;
        bvh->height = 1;
        return;
    }
    u32 middle = split_node(bvh->nodes, &bvh->node_count, b, bvh->nodes, 0, N);
    OIter *stack = b->iters;
    stack[0].start = 0; stack[0].end = middle; stack[0].node_id = 1;
    stack[1].start = middle; stack[1].end = N; stack[1].node_id = 2;
    /* `depth` is the index into this explicit build stack, as in the reference: a left child keeps
     * its parent's index and a right child takes the next, so the depth fields and the height
     * written here count right turns on a path, not the tree depth */
    i32 depth = 1;
    u32 leaf_count = 0;
    bvh->height = 1;
    while (depth >= 0) {
        OIter left = stack[depth], right;
        BVHNode *node = bvh->nodes + left.node_id;
        N = left.end - left.start;
        if (N <= max_leaf) {
            node->depth = (u16)depth;
            node->child_count = (u16)N;
            node->first_child_id = leaf_count;
            u32 *lid = b->leaf_ids + left.start;
            for (u32 i = 0; i < N; i++, lid++) bvh->leaf_ids[leaf_count + i] = b->leaf_nodes[*lid].first_child_id;
            leaf_count += N;
            depth--;
        } else {
            middle = split_node(bvh->nodes, &bvh->node_count, b, node, left.start, left.end);
            bvh->nodes[bvh->node_count - 1].depth = bvh->nodes[bvh->node_count - 2].depth = (u16)depth;
            right.end = left.end;
            right.start = left.end = middle;
            left.node_id = node->first_child_id;
            right.node_id = node->first_child_id + 1;
            stack[depth] = left;
            stack[++depth] = right;
            if (depth > (i32)bvh->height) bvh->height = (u32)depth;
        }
    }
    bvh->nodes->aabb = merge_aabb(bvh->nodes[1].aabb, bvh->nodes[2].aabb);
}

static AABB primitive_local_aabb(const Scene *sc, const Primitive *p) {    /* getPrimitiveAABB primitive.h:53 */
    AABB a;
    if (p->type == PrimitiveType_Mesh) return sc->meshes[p->id].aabb;
    a.max = splat(p->type == PrimitiveType_Tetrahedron ? (SQRT3 / 3) : 1);
    a.min = vneg(a.max);
    return a;
}
void orc_primitive_aabbs(const Scene *sc, float *out) {
    for (u32 i = 0; i < sc->settings.primitives; i++) {
        AABB a = primitive_local_aabb(sc, sc->primitives + i);
        transform_aabb(&a, sc->primitives + i);
        memcpy(out + 6 * i, &a, sizeof(a));
    }
}
/* updateSceneBVH :366 */
void orc_update_scene_bvh(Scene *sc) {
    u32 n = sc->settings.primitives;
    OBuilder b;
    builder_init(&b, n ? n : 1);
    for (u32 i = 0; i < n; i++) {
        BVHNode *ln = b.leaf_nodes + i;
        ln->aabb = primitive_local_aabb(sc, sc->primitives + i);
        transform_aabb(&ln->aabb, sc->primitives + i);
        ln->first_child_id = b.leaf_ids[i] = i;
    }
    build_bvh(&sc->bvh, &b, n, MAX_OBJS_PER_SCENE_BVH_NODE);
    builder_free(&b);
}
/* triangle leaf AABB with EPS padding on flat axes (:283-318) */
static AABB triangle_aabb(const vec3 *v1, const vec3 *v2, const vec3 *v3) {
    AABB a;
    a.min.x = v2->x < v3->x ? v2->x : v3->x; a.min.y = v2->y < v3->y ? v2->y : v3->y; a.min.z = v2->z < v3->z ? v2->z : v3->z;
    a.max.x = v2->x > v3->x ? v2->x : v3->x; a.max.y = v2->y > v3->y ? v2->y : v3->y; a.max.z = v2->z > v3->z ? v2->z : v3->z;
    a.min.x = a.min.x < v1->x ? a.min.x : v1->x; a.min.y = a.min.y < v1->y ? a.min.y : v1->y; a.min.z = a.min.z < v1->z ? a.min.z : v1->z;
    a.max.x = a.max.x > v1->x ? a.max.x : v1->x; a.max.y = a.max.y > v1->y ? a.max.y : v1->y; a.max.z = a.max.z > v1->z ? a.max.z : v1->z;
    f32 d;
    d = a.max.x - a.min.x; if (d < 0) d = -d; if (d < ORC_EPS) { a.min.x -= ORC_EPS; a.max.x += ORC_EPS; }
    d = a.max.y - a.min.y; if (d < 0) d = -d; if (d < ORC_EPS) { a.min.y -= ORC_EPS; a.max.y += ORC_EPS; }
    d = a.max.z - a.min.z; if (d < 0) d = -d; if (d < ORC_EPS) { a.min.z -= ORC_EPS; a.max.z += ORC_EPS; }
    return a;
}
/* the Triangle record of updateMeshBVH (:330-363) for source triangle `t` */
static void triangle_record(const Mesh *m, u32 t, Triangle *out) {
    const TriangleVertexIndices *ix = m->vertex_position_indices + t;
    const vec3 *v1 = m->vertex_positions + ix->ids[0], *v2 = m->vertex_positions + ix->ids[1], *v3 = m->vertex_positions + ix->ids[2];
    mat3 m3;
    m3.X = vsub(*v3, *v1);
    m3.Y = vsub(*v2, *v1);
    m3.Z = vcross(m3.X, m3.Y);
    out->area_of_parallelogram = vlen(m3.Z);
    m3.Z = vscale(m3.Z, 1.0f / out->area_of_parallelogram);
    const TriangleVertexIndices *nx = m->vertex_normal_indices + t;
    out->world_to_tangent = minv3(m3);
    out->normal = m3.Z;
    out->position = *v1;
    out->vertex_normals[0] = m->vertex_normals[nx->ids[0]];
    out->vertex_normals[1] = m->vertex_normals[nx->ids[1]];
    out->vertex_normals[2] = m->vertex_normals[nx->ids[2]];
    if (m->uvs_count) {
        const TriangleVertexIndices *ux = m->vertex_uvs_indices + t;
        vec2 a = out->uvs[0] = m->vertex_uvs[ux->ids[0]];
        vec2 b = out->uvs[1] = m->vertex_uvs[ux->ids[1]];
        vec2 c = out->uvs[2] = m->vertex_uvs[ux->ids[2]];
        out->area_of_uv = fabsf((b.x - a.x) * (c.y - a.y) - (c.x - a.x) * (b.y - a.y));
    }
}
/* updateMeshBVH :272 */
void orc_update_mesh_bvh(Mesh *m) {
    u32 n = m->triangle_count;
    OBuilder b;
    builder_init(&b, n ? n : 1);
    for (u32 i = 0; i < n; i++) {
        const TriangleVertexIndices *ix = m->vertex_position_indices + i;
        b.leaf_nodes[i].aabb = triangle_aabb(m->vertex_positions + ix->ids[0], m->vertex_positions + ix->ids[1],
                                             m->vertex_positions + ix->ids[2]);
        b.leaf_nodes[i].first_child_id = b.leaf_ids[i] = i;
    }
    build_bvh(&m->bvh, &b, n, MAX_TRIANGLES_PER_MESH_BVH_NODE);
    for (u32 i = 0; i < n; i++) b.leaf_ids[i] = m->bvh.leaf_ids[i];
    for (u32 i = 0; i < n; i++) {
        u32 t = b.leaf_ids[i];
        m->bvh.leaf_ids[t] = i;
        triangle_record(m, t, m->triangles + i);
    }
    builder_free(&b);
}

/* ---- 30-bit Morton LBVH (project specification; no reference counterpart) ------------------- */
static inline u32 ordered_bits(f32 f) {
    u32 u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
static inline f32 tmin(f32 a, f32 b) { return ordered_bits(b) < ordered_bits(a) ? b : a; }
static inline f32 tmax(f32 a, f32 b) { return ordered_bits(b) > ordered_bits(a) ? b : a; }
static AABB union_range(const float *aabbs, const u32 *order, u32 f, u32 l) {
    AABB box;
    box.min = splat(INFINITY);
    box.max = splat(-INFINITY);
    for (u32 i = f; i <= l; i++) {
        const float *a = aabbs + 6 * order[i];
        box.min.x = tmin(box.min.x, a[0]); box.min.y = tmin(box.min.y, a[1]); box.min.z = tmin(box.min.z, a[2]);
        box.max.x = tmax(box.max.x, a[3]); box.max.y = tmax(box.max.y, a[4]); box.max.z = tmax(box.max.z, a[5]);
    }
    return box;
}
static inline u32 spread10(u32 v) {            /* 10 bits -> every third bit of 30 */
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
static inline u32 quantize(f32 c, f32 lo, f32 scale) {
    f32 t = (c - lo) * scale;
    if (!(t > 0.0f)) return 0;
    if (t >= 1023.0f) return 1023;
    return (u32)t;
}
static inline int delta64(const uint64_t *k, u32 n, i32 i, i32 j) {
    if (j < 0 || j >= (i32)n) return -1;
    return __builtin_clzll(k[i] ^ k[j]);
}
static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

int orc_lbvh30(const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *codes, uint32_t *order,
               BVHNode *nodes, uint32_t *leaf_ids, uint32_t *info) {
    /* 1. scene bounds = union of the item AABBs; centroid = (min + max) * 0.5 */
    f32 lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (u32 i = 0; i < n; i++)
        for (int a = 0; a < 3; a++) {
            f32 mn = aabbs[6 * i + a], mx = aabbs[6 * i + 3 + a];
            lo[a] = tmin(lo[a], mn);
            hi[a] = tmax(hi[a], mx);
        }
    f32 scale[3];
    for (int a = 0; a < 3; a++) {
        f32 ext = hi[a] - lo[a];
        scale[a] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    /* 2. Morton code: x in the highest of each bit triple */
    uint64_t *keys = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
    for (u32 i = 0; i < n; i++) {
        u32 q[3];
        for (int a = 0; a < 3; a++) {
            f32 c = (aabbs[6 * i + a] + aabbs[6 * i + 3 + a]) * 0.5f;
            q[a] = quantize(c, lo[a], scale[a]);
        }
        codes[i] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
        keys[i] = ((uint64_t)codes[i] << 32) | i;
    }
    /* 3. sort by (code, index): the keys are unique, so any correct sort gives this order */
    qsort(keys, n, sizeof(uint64_t), cmp_u64);
    for (u32 i = 0; i < n; i++) order[i] = (u32)(keys[i] & 0xFFFFFFFFu);
    for (u32 i = 0; i < n; i++) leaf_ids[i] = order[i];

    if (n <= max_leaf) {
        memset(nodes, 0, sizeof(BVHNode));
        nodes[0].aabb = n ? union_range(aabbs, order, 0, n - 1) : nodes[0].aabb;
        nodes[0].child_count = (u16)n;
        nodes[0].first_child_id = 0;
        info[0] = 1;
        info[1] = 1;
        free(keys);
        return 0;
    }
    /* 4. Karras (2012) binary radix tree over the sorted keys: internal nodes 0..n-2 */
    u32 ni = n - 1;
    u32 *first = (u32*)malloc(sizeof(u32) * ni), *last = (u32*)malloc(sizeof(u32) * ni);
    u32 *lchild = (u32*)malloc(sizeof(u32) * ni), *rchild = (u32*)malloc(sizeof(u32) * ni);
    u32 *parent = (u32*)malloc(sizeof(u32) * ni);
    for (u32 k = 0; k < ni; k++) parent[k] = 0xFFFFFFFFu;
    for (i32 i = 0; i < (i32)ni; i++) {
        int d = (delta64(keys, n, i, i + 1) - delta64(keys, n, i, i - 1)) > 0 ? 1 : -1;
        int dmin = delta64(keys, n, i, i - d);
        i32 lmax = 2;
        while (delta64(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
        i32 l = 0;
        for (i32 t = lmax / 2; t >= 1; t /= 2)
            if (delta64(keys, n, i, i + (l + t) * d) > dmin) l += t;
        i32 j = i + l * d;
        int dnode = delta64(keys, n, i, j);
        i32 s = 0;
        for (i32 t = (l + 1) / 2; ; t = (t + 1) / 2) {
            if (delta64(keys, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        i32 g = i + s * d + (d < 0 ? -1 : 0);
        i32 lo_i = i < j ? i : j, hi_i = i < j ? j : i;
        first[i] = (u32)lo_i;
        last[i] = (u32)hi_i;
        lchild[i] = (lo_i == g) ? (0x80000000u | (u32)g) : (u32)g;
        rchild[i] = (hi_i == g + 1) ? (0x80000000u | (u32)(g + 1)) : (u32)(g + 1);
        if (!(lchild[i] & 0x80000000u)) parent[lchild[i]] = (u32)i;
        if (!(rchild[i] & 0x80000000u)) parent[rchild[i]] = (u32)i;
    }
    /* 5. collapse: an internal node is kept when it covers more than max_leaf items; kept nodes
     *    are ranked in index order, and kept node r's children go to output slots 1+2r, 2+2r */
    u32 *rank = (u32*)malloc(sizeof(u32) * ni);
    u32 kept = 0;
    for (u32 k = 0; k < ni; k++) rank[k] = (last[k] - first[k] + 1 > max_leaf) ? kept++ : 0xFFFFFFFFu;
    /* depth of internal node k = number of ancestors */
    u32 height = 0;
    memset(nodes, 0, sizeof(BVHNode) * (1 + 2 * kept));
    nodes[0].first_child_id = 1 + 2 * rank[0];   /* the root is kept (it covers n > max_leaf items) */
    for (u32 k = 0; k < ni; k++) {
        if (rank[k] == 0xFFFFFFFFu) continue;
        u32 dep = 0;
        for (u32 p = parent[k]; p != 0xFFFFFFFFu; p = parent[p]) dep++;
        u32 kids[2] = {lchild[k], rchild[k]};
        for (int c = 0; c < 2; c++) {
            BVHNode *o = nodes + 1 + 2 * rank[k] + c;
            u32 ch = kids[c];
            u32 f, l;
            if (ch & 0x80000000u) { f = l = ch & 0x7FFFFFFFu; }
            else { f = first[ch]; l = last[ch]; }
            o->depth = (u16)(dep + 1);
            if (dep + 1 > height) height = dep + 1;
            if (!(ch & 0x80000000u) && rank[ch] != 0xFFFFFFFFu) {
                o->first_child_id = 1 + 2 * rank[ch];
                o->child_count = 0;
            } else {
                o->first_child_id = f;
                o->child_count = (u16)(l - f + 1);
            }
        }
    }
    /* 6. AABBs: every node's box is the union of its item range's boxes, taken with the IEEE
     *    total order (-0 < +0) so that the union does not depend on the order it is formed in */
    /* kept nodes' output slots: the root is slot 0; others are the slot their parent wrote */
    u32 *slot = (u32*)malloc(sizeof(u32) * ni);
    slot[0] = 0;
    for (u32 k = 0; k < ni; k++) {
        if (rank[k] == 0xFFFFFFFFu) continue;
        if (!(lchild[k] & 0x80000000u) && rank[lchild[k]] != 0xFFFFFFFFu) slot[lchild[k]] = 1 + 2 * rank[k];
        if (!(rchild[k] & 0x80000000u) && rank[rchild[k]] != 0xFFFFFFFFu) slot[rchild[k]] = 2 + 2 * rank[k];
    }
    /* every output node's box = union of its item range's boxes */
    for (u32 s = 0; s < 1 + 2 * kept; s++) {
        BVHNode *o = nodes + s;
        u32 f, l;
        if (s == 0) { f = 0; l = n - 1; }
        else if (o->child_count) { f = o->first_child_id; l = f + o->child_count - 1; }
        else continue;
        o->aabb = union_range(aabbs, order, f, l);
    }
    for (u32 k = 0; k < ni; k++) {
        if (rank[k] == 0xFFFFFFFFu || k == 0) continue;
        nodes[slot[k]].aabb = union_range(aabbs, order, first[k], last[k]);
    }
    info[0] = 1 + 2 * kept;
    info[1] = height;
    free(slot); free(rank); free(first); free(last); free(lchild); free(rchild); free(parent); free(keys);
    return 0;
}

/* ---- binned SAH (project specification; the reference's builder is the full-sweep SAH above) -- */
#define ORC_BINS 32
typedef struct { u32 begin, end, slot; AABB box, cbox; } OTask;

static inline f32 half_area_t(const AABB *a) {
    f32 ex = a->max.x - a->min.x, ey = a->max.y - a->min.y, ez = a->max.z - a->min.z;
    return ex * ey + ey * ez + ez * ex;
}
static inline void grow(AABB *a, const float *b) {
    a->min.x = tmin(a->min.x, b[0]); a->min.y = tmin(a->min.y, b[1]); a->min.z = tmin(a->min.z, b[2]);
    a->max.x = tmax(a->max.x, b[3]); a->max.y = tmax(a->max.y, b[4]); a->max.z = tmax(a->max.z, b[5]);
}
static inline void grow_box(AABB *a, const AABB *b) { grow(a, &b->min.x); }
static inline void empty_box(AABB *a) { a->min = splat(INFINITY); a->max = splat(-INFINITY); }
static inline u32 bin_of(f32 c, f32 lo, f32 scale) {
    f32 t = (c - lo) * scale;
    if (!(t > 0.0f)) return 0;
    if (t >= (f32)(ORC_BINS - 1)) return ORC_BINS - 1;
    return (u32)t;
}

/* Breadth-first binned SAH over n item boxes, leaves of at most max_leaf items:
 *   centroid (min+max)*0.5; a node's centroid box and box are unions under the IEEE total order;
 *   per axis with a non-zero centroid extent e, bin = clamp((c - lo) * (32/e)) into 32 bins;
 *   split candidates after bin k (k = 0..30) cost halfArea(L)*nL + halfArea(R)*nR (the
 *   reference's surface-area formula, AABB.h:39), skipping empty sides; the lowest cost wins,
 *   ties to the lower axis then the lower k; with no candidate the range is split at its middle;
 *   the partition is stable; the split nodes of one level get child pairs in level order
 *   (pair p -> slots 1+2p, 2+2p); depth = level, height = deepest leaf (1 for a root leaf). */
int orc_binned_sah(const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *order, BVHNode *nodes,
                   uint32_t *info) {
    f32 *cent = (f32*)malloc(sizeof(f32) * 3 * (n ? n : 1));
    u32 *ids = (u32*)malloc(sizeof(u32) * (n ? n : 1)), *tmp = (u32*)malloc(sizeof(u32) * (n ? n : 1));
    OTask *cur = (OTask*)malloc(sizeof(OTask) * (n ? n : 1)), *next = (OTask*)malloc(sizeof(OTask) * (n ? n : 1));
    AABB root, rootc;
    empty_box(&root);
    empty_box(&rootc);
    for (u32 i = 0; i < n; i++) {
        ids[i] = i;
        for (int a = 0; a < 3; a++) cent[3 * i + a] = (aabbs[6 * i + a] + aabbs[6 * i + 3 + a]) * 0.5f;
        grow(&root, aabbs + 6 * i);
        f32 c6[6] = {cent[3 * i], cent[3 * i + 1], cent[3 * i + 2], cent[3 * i], cent[3 * i + 1], cent[3 * i + 2]};
        grow(&rootc, c6);
    }
    u32 ncur = 1, pairs = 0, height = 1, level = 0;
    cur[0].begin = 0; cur[0].end = n; cur[0].slot = 0; cur[0].box = root; cur[0].cbox = rootc;
    while (ncur) {
        u32 nnext = 0;
        for (u32 t = 0; t < ncur; t++) {
            OTask *T = cur + t;
            BVHNode *node = nodes + T->slot;
            u32 cnt = T->end - T->begin;
            memset(node, 0, sizeof(*node));
            node->aabb = T->box;
            node->depth = (u16)level;
            if (cnt <= max_leaf) {
                node->first_child_id = T->begin;
                node->child_count = (u16)cnt;
                if (level > height) height = level;
                continue;
            }
            /* bins of the three axes */
            u32 bc[3][ORC_BINS];
            AABB bb[3][ORC_BINS], bcb[3][ORC_BINS];
            f32 lo[3], scale[3];
            int valid[3];
            const f32 *cl = &T->cbox.min.x;
            for (int a = 0; a < 3; a++) {
                f32 e = cl[3 + a] - cl[a];
                valid[a] = e > 0.0f;
                lo[a] = cl[a];
                scale[a] = valid[a] ? (f32)ORC_BINS / e : 0.0f;
                for (int b = 0; b < ORC_BINS; b++) { bc[a][b] = 0; empty_box(&bb[a][b]); empty_box(&bcb[a][b]); }
            }
            for (u32 k = T->begin; k < T->end; k++) {
                u32 i = ids[k];
                f32 c6[6] = {cent[3 * i], cent[3 * i + 1], cent[3 * i + 2], cent[3 * i], cent[3 * i + 1], cent[3 * i + 2]};
                for (int a = 0; a < 3; a++) {
                    if (!valid[a]) continue;
                    u32 b = bin_of(cent[3 * i + a], lo[a], scale[a]);
                    bc[a][b]++;
                    grow(&bb[a][b], aabbs + 6 * i);
                    grow(&bcb[a][b], c6);
                }
            }
            int best_axis = -1, best_k = -1;
            f32 best = INFINITY;
            for (int a = 0; a < 3; a++) {
                if (!valid[a]) continue;
                AABB R[ORC_BINS];
                u32 nR[ORC_BINS];
                AABB acc;
                empty_box(&acc);
                u32 an = 0;
                for (int b = ORC_BINS - 1; b >= 1; b--) { grow_box(&acc, &bb[a][b]); an += bc[a][b]; R[b] = acc; nR[b] = an; }
                empty_box(&acc);
                an = 0;
                for (int k = 0; k < ORC_BINS - 1; k++) {
                    grow_box(&acc, &bb[a][k]);
                    an += bc[a][k];
                    if (!an || !nR[k + 1]) continue;
                    f32 cost = half_area_t(&acc) * (f32)an + half_area_t(&R[k + 1]) * (f32)nR[k + 1];
                    if (cost < best) { best = cost; best_axis = a; best_k = k; }
                }
            }
            OTask L, Rt;
            u32 mid;
            if (best_axis >= 0) {
                u32 nl = 0, p = T->begin;
                for (u32 k = T->begin; k < T->end; k++)
                    if (bin_of(cent[3 * ids[k] + best_axis], lo[best_axis], scale[best_axis]) <= (u32)best_k) tmp[p++] = ids[k], nl++;
                for (u32 k = T->begin; k < T->end; k++)
                    if (bin_of(cent[3 * ids[k] + best_axis], lo[best_axis], scale[best_axis]) > (u32)best_k) tmp[p++] = ids[k];
                memcpy(ids + T->begin, tmp + T->begin, sizeof(u32) * cnt);
                mid = T->begin + nl;
                empty_box(&L.box); empty_box(&L.cbox); empty_box(&Rt.box); empty_box(&Rt.cbox);
                for (int b = 0; b < ORC_BINS; b++) {
                    if (b <= best_k) { grow_box(&L.box, &bb[best_axis][b]); grow_box(&L.cbox, &bcb[best_axis][b]); }
                    else { grow_box(&Rt.box, &bb[best_axis][b]); grow_box(&Rt.cbox, &bcb[best_axis][b]); }
                }
            } else {
                mid = T->begin + cnt / 2;
                empty_box(&L.box); empty_box(&L.cbox); empty_box(&Rt.box); empty_box(&Rt.cbox);
                for (u32 k = T->begin; k < T->end; k++) {
                    u32 i = ids[k];
                    f32 c6[6] = {cent[3 * i], cent[3 * i + 1], cent[3 * i + 2], cent[3 * i], cent[3 * i + 1], cent[3 * i + 2]};
                    if (k < mid) { grow(&L.box, aabbs + 6 * i); grow(&L.cbox, c6); }
                    else { grow(&Rt.box, aabbs + 6 * i); grow(&Rt.cbox, c6); }
                }
            }
            node->first_child_id = 1 + 2 * pairs;
            L.begin = T->begin; L.end = mid; L.slot = 1 + 2 * pairs;
            Rt.begin = mid; Rt.end = T->end; Rt.slot = 2 + 2 * pairs;
            pairs++;
            next[nnext++] = L;
            next[nnext++] = Rt;
        }
        OTask *sw = cur; cur = next; next = sw;
        ncur = nnext;
        level++;
    }
    memcpy(order, ids, sizeof(u32) * n);
    info[0] = 1 + 2 * pairs;
    info[1] = height;
    free(cent); free(ids); free(tmp); free(cur); free(next);
    return 0;
}

/* updateMeshBVH (builder_top_down.h:272) with the binned-SAH topology in place of the full sweep:
 * the same padded triangle boxes (:283-318), leaves of at most MAX_TRIANGLES_PER_MESH_BVH_NODE,
 * Triangle records in leaf order with the same precompute (:330-363), and leaf_ids mapping each
 * source triangle to its slot (:327). */
int orc_update_mesh_bvh_binned(Mesh *m) {
    u32 n = m->triangle_count;
    if (!n) return -1;
    float *boxes = (float*)malloc(sizeof(float) * 6 * n);
    u32 *order = (u32*)malloc(sizeof(u32) * n);
    if (!boxes || !order) { free(boxes); free(order); return -1; }
    for (u32 i = 0; i < n; i++) {
        const TriangleVertexIndices *ix = m->vertex_position_indices + i;
        AABB a = triangle_aabb(m->vertex_positions + ix->ids[0], m->vertex_positions + ix->ids[1],
                               m->vertex_positions + ix->ids[2]);
        memcpy(boxes + 6 * i, &a, sizeof(float) * 6);
    }
    u32 info[2];
    orc_binned_sah(boxes, n, MAX_TRIANGLES_PER_MESH_BVH_NODE, order, m->bvh.nodes, info);
    m->bvh.node_count = info[0];
    m->bvh.height = info[1];
    for (u32 i = 0; i < n; i++) {
        m->bvh.leaf_ids[order[i]] = i;
        triangle_record(m, order[i], m->triangles + i);
    }
    free(boxes);
    free(order);
    return 0;
}

/* ---- picking: manipulateSelection viewport/manipulation.h:55-123 ------------------------------- */
/* setRayFromCoords (shaders/common.h:170): start + right*x + down*y, normalised; then hitPrimitives
 * over the TLAS leaf list with the visibility cull at (x, y) and every light's glow sphere
 * (radius intensity/128, hitSphereSimple sphere.h:44).  Primitive screen bounds as the scene
 * holds them (call orc_update_scene_ssb for the viewport first). */
int orc_pick(const Scene *sc, const Viewport *vp, int x, int y, OrcPick *out) {
    OTrace *tr = (OTrace*)calloc(1, sizeof(OTrace));
    if (!tr) return -1;
    if (sc->settings.meshes) tr->closest_mesh_hit.object_type = PrimitiveType_Mesh;
    Ray ray;
    memset(&ray, 0, sizeof(ray));
    ray.origin = vp->camera->transform.position;
    ray.direction = vsfma(vp->projection_plane.right, (f32)x, vp->projection_plane.start);
    ray.direction = vsfma(vp->projection_plane.down, (f32)y, ray.direction);
    ray.direction = vnorm(ray.direction);
    ray.direction_reciprocal = vrcp(ray.direction);
    RayHit *hit = &tr->closest_hit;
    hit->distance = hit->distance_squared = INFINITY;
    bool found = hit_primitives(tr, &ray, sc, sc->bvh.leaf_ids, sc->settings.primitives, false, true, (u16)x, (u16)y);
    if (sc->lights) {
        for (u32 i = 0; i < sc->settings.lights; i++) {
            const Light *light = sc->lights + i;
            f32 radius = light->intensity * (1.0f / (8.0f * 16.0f));
            tr->sphere_hit.furthest = hit->distance / radius;
            if (hit_sphere_simple(ray.origin, ray.direction, light->position_or_direction, 1.0f / radius, &tr->sphere_hit)) {
                hit->distance = tr->sphere_hit.t_near * radius;
                hit->position = vsfma(ray.direction, hit->distance, ray.origin);
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
        out->object_distance = vmat3(vsub(hit->position, ray.origin), vp->camera->transform.rotation_matrix_inverted).z;
    }
    free(tr);
    return 0;
}

/* ---- debug overlays: drawBVH (render/raytracer.h:46) and drawSSB (render/SSB.h:175) ----------- */
/* The unit box initBox (core/init.h:279) leaves in viewport->default_box, corners in BoxCorners
 * order (core/types.h:86), and the 12 edges of setBoxEdgesFromVertices (core/init.h:250) in
 * BoxEdgeSides order (core/types.h:102): the order in which drawBox draws them. */
static const f32 kBoxCorner[8][3] = {{-1, 1, 1}, {1, 1, 1}, {-1, -1, 1}, {1, -1, 1},
                                     {-1, 1, -1}, {1, 1, -1}, {-1, -1, -1}, {1, -1, -1}};
static const u8 kBoxEdge[12][2] = {{0, 1}, {2, 3}, {2, 0}, {3, 1}, {4, 5}, {6, 7},
                                   {6, 4}, {7, 5}, {2, 6}, {0, 4}, {3, 7}, {1, 5}};

/* A float -> i32 conversion as x86's truncating convert performs it: out-of-range values and NaN
 * give INT32_MIN (the "integer indefinite" value), which is what the reference's (i32) casts
 * produce on the machines it runs on. */
static inline i32 trunc_i32(f32 v) { return (v >= -2147483648.0f && v < 2147483648.0f) ? (i32)v : INT32_MIN; }
static inline f32 frac_of(f32 v) { return v - floorf(v); }              /* fractionOf line.h:39 */
static inline f32 one_minus_frac_of(f32 v) { return 1 - frac_of(v); }  /* oneMinusFractionOf line.h:43 */
static inline int in_range(i32 v, i32 end, i32 start) { return v >= start && v < end; }   /* base.h:381 */

typedef struct {
    FloatPixel *px;
    u16 stride;
    i32 x_left, y_top, w, h;   /* viewport position and frame extent + position */
} OCanvas;

static inline void plot(const OCanvas *c, i32 x, i32 y, f64 z, vec3 color, f32 opacity) {
    set_pixel(c->px + (c->stride * y) + x, color, opacity, z);   /* setPixelByCoords types.h:453 */
}

/* drawLine shapes/line.h:46 (an anti-aliased line of 1 + line_width + 1 pixels across) */
static void draw_line(const OCanvas *c, f32 x1, f32 y1, f64 z1, f32 x2, f32 y2, f64 z2, vec3 color, f32 opacity,
                      u8 line_width) {
    if (x1 < 0 && y1 < 0 && x2 < 0 && y2 < 0) return;
    const i32 x_left = c->x_left, y_top = c->y_top, w = c->w, h = c->h;
    x1 += (f32)x_left; x2 += (f32)x_left;
    y1 += (f32)y_top;  y2 += (f32)y_top;
    color = vmul(color, color);
    f64 tmp, z_range, range_remap, z = 0, z_curr = 0, z_step = 0;
    f32 dx = x2 - x1, dy = y2 - y1, gap, grad, first_offset, last_offset;
    vec3 first, last;
    i32 x, y, sx, sy, ex, ey;
    const int has_depth = z1 || z2;
    if (fabsf(dx) > fabsf(dy)) {   /* shallow: one column per x */
        if (x2 < x1) { tmp = x2; x2 = x1; x1 = (f32)tmp; tmp = y2; y2 = y1; y1 = (f32)tmp; tmp = z2; z2 = z1; z1 = tmp; }
        grad = dy / dx;
        first.x = roundf(x1); last.x = roundf(x2);
        first_offset = first.x - x1; last_offset = last.x - x2;
        first.y = y1 + grad * first_offset; last.y = y2 + grad * last_offset;
        sx = trunc_i32(first.x); sy = trunc_i32(first.y); ex = trunc_i32(last.x); ey = trunc_i32(last.y);
        x = sx; y = sy;
        gap = one_minus_frac_of(x1 + 0.5f);
        if (in_range(x, w, x_left)) {
            if (in_range(y, h, y_top)) plot(c, x, y, z1, color, one_minus_frac_of(first.y) * gap * opacity);
            for (u8 i = 0; i < line_width; i++) { y++; if (in_range(y, h, y_top)) plot(c, x, y, z1, color, opacity); }
            y++;
            if (in_range(y, h, y_top)) plot(c, x, y, z1, color, frac_of(first.y) * gap * opacity);
        }
        x = ex; y = ey;
        gap = frac_of(x2 + 0.5f);
        if (in_range(x, w, x_left)) {
            if (in_range(y, h, y_top)) plot(c, x, y, z2, color, one_minus_frac_of(last.y) * gap * opacity);
            for (u8 i = 0; i < line_width; i++) { y++; if (in_range(y, h, y_top)) plot(c, x, y, z2, color, opacity); }
            y++;
            if (in_range(y, h, y_top)) plot(c, x, y, z2, color, frac_of(last.y) * gap * opacity);
        }
        if (has_depth) {   /* 1/z interpolated across the interior columns */
            z1 = 1.0 / z1; z2 = 1.0 / z2;
            z_range = z2 - z1;
            range_remap = z_range / (f64)(x2 - x1);
            z1 += range_remap * (f64)(first_offset + 1);
            z2 += range_remap * (f64)(last_offset - 1);
            z_range = z2 - z1;
            z_step = z_range / (f64)(last.x - first.x - 1);
            z_curr = z1;
        } else z = 0;
        gap = first.y + grad;
        for (x = sx + 1; x < ex; x++) {
            if (in_range(x, w, x_left)) {
                if (has_depth) z = 1.0 / z_curr;
                y = trunc_i32(gap);
                if (in_range(y, h, y_top)) plot(c, x, y, z, color, one_minus_frac_of(gap) * opacity);
                for (u8 i = 0; i < line_width; i++) { y++; if (in_range(y, h, y_top)) plot(c, x, y, z, color, opacity); }
                y++;
                if (in_range(y, h, y_top)) plot(c, x, y, z, color, frac_of(gap) * opacity);
            }
            gap += grad;
            if (has_depth) z_curr += z_step;
        }
    } else {   /* steep: one row per y */
        if (y2 < y1) { tmp = x2; x2 = x1; x1 = (f32)tmp; tmp = y2; y2 = y1; y1 = (f32)tmp; tmp = z2; z2 = z1; z1 = tmp; }
        grad = dx / dy;
        first.y = roundf(y1); last.y = roundf(y2);
        first_offset = y1 - first.y; last_offset = last.y - y2;
        first.x = x1 + grad * first_offset; last.x = x2 + grad * last_offset;
        sy = trunc_i32(first.y); sx = trunc_i32(first.x); ey = trunc_i32(last.y); ex = trunc_i32(last.x);
        x = sx; y = sy;
        gap = one_minus_frac_of(y1 + 0.5f);
        if (in_range(y, h, y_top)) {
            if (in_range(x, w, x_left)) plot(c, x, y, z1, color, one_minus_frac_of(first.x) * gap * opacity);
            for (u8 i = 0; i < line_width; i++) { x++; if (in_range(x, w, x_left)) plot(c, x, y, z1, color, opacity); }
            x++;
            if (in_range(x, w, x_left)) plot(c, x, y, z1, color, frac_of(first.x) * gap * opacity);
        }
        x = ex; y = ey;
        gap = frac_of(y2 + 0.5f);
        if (in_range(y, h, y_top)) {
            if (in_range(x, w, x_left)) plot(c, x, y, z2, color, one_minus_frac_of(last.x) * gap * opacity);
            for (u8 i = 0; i < line_width; i++) { x++; if (in_range(x, w, x_left)) plot(c, x, y, z2, color, opacity); }
            x++;
            if (in_range(x, w, x_left)) plot(c, x, y, z2, color, frac_of(last.x) * gap * opacity);
        }
        if (has_depth) {
            z1 = 1.0 / z1; z2 = 1.0 / z2;
            z_range = z2 - z1;
            range_remap = z_range / (f64)(y2 - y1);
            z1 += range_remap * (f64)(first_offset + 1);
            z2 += range_remap * (f64)(last_offset - 1);
            z_range = z2 - z1;
            z_step = z_range / (f64)(last.y - first.y - 1);
            z_curr = z1;
        } else z = 0;
        gap = first.x + grad;
        for (y = sy + 1; y < ey; y++) {
            if (in_range(y, h, y_top)) {
                if (has_depth) z = 1.0 / z_curr;
                x = trunc_i32(gap);
                if (in_range(x, w, x_left)) plot(c, x, y, z, color, one_minus_frac_of(gap) * opacity);
                for (u8 i = 0; i < line_width; i++) { x++; if (in_range(x, w, x_left)) plot(c, x, y, z, color, opacity); }
                x++;
                if (in_range(x, w, x_left)) plot(c, x, y, z, color, frac_of(gap) * opacity);
            }
            gap += grad;
            if (has_depth) z_curr += z_step;
        }
    }
}

/* lerpVec3 vec3.h:265 */
static inline vec3 vlerp(vec3 from, vec3 to, f32 by) { return vsfma(vsub(to, from), by, from); }

/* cullAndClipEdge shapes/edge.h:8: near, far, then the left/right/bottom/top frustum planes */
static int clip_edge(vec3 *pa, vec3 *pb, const Viewport *vp) {
    vec3 A = *pa, B = *pb, N;
    f32 d = vp->settings.near_clipping_plane_distance, na, nb;
    u8 out = (A.z < d) | ((B.z < d) << 1);
    if (out) {
        if (out == 3) return 0;
        if (out & 1) A = vlerp(A, B, (d - A.z) / (B.z - A.z));
        else         B = vlerp(B, A, (d - B.z) / (A.z - B.z));
    }
    d = vp->settings.far_clipping_plane_distance;
    out = (A.z > d) | ((B.z > d) << 1);
    if (out) {
        if (out == 3) return 0;
        if (out & 1) A = vlerp(A, B, (A.z - d) / (A.z - B.z));
        else         B = vlerp(B, A, (B.z - d) / (B.z - A.z));
    }
    for (int plane = 0; plane < 4; plane++) {
        if (plane == 0) N = V3(vp->camera->focal_length, 0, vp->frame_buffer->dimensions.width_over_height);
        else if (plane == 1) N.x = -N.x;
        else if (plane == 2) N = V3(0, vp->camera->focal_length, 1);
        else N.y = -N.y;
        na = vdot(N, A);
        nb = vdot(N, B);
        out = (na < 0) | ((nb < 0) << 1);
        if (out) {
            if (out == 3) return 0;
            if (out & 1) A = vlerp(A, B, na / (na - nb));
            else         B = vlerp(B, A, nb / (nb - na));
        }
    }
    *pa = A;
    *pb = B;
    return 1;
}

/* mulVec4Mat4 vec4.h:96 with w = 1, then the perspective divide */
static inline vec3 project_point(vec3 p, const mat4 *m) {
    vec4 o;
    o.x = p.x * m->X.x + p.y * m->Y.x + p.z * m->Z.x + 1.0f * m->W.x;
    o.y = p.x * m->X.y + p.y * m->Y.y + p.z * m->Z.y + 1.0f * m->W.y;
    o.z = p.x * m->X.z + p.y * m->Y.z + p.z * m->Z.z + 1.0f * m->W.z;
    o.w = p.x * m->X.w + p.y * m->Y.w + p.z * m->Z.w + 1.0f * m->W.w;
    return vscale(V3(o.x, o.y, o.z), 1.0f / o.w);
}

/* drawEdge shapes/edge.h:112 = projectEdge (:83) + drawLine */
static void draw_edge(const OCanvas *c, const Viewport *vp, vec3 A, vec3 B, vec3 color, f32 opacity, u8 line_width) {
    if (!clip_edge(&A, &B, vp)) return;
    const f32 az = A.z, bz = B.z;
    const Dimensions *dim = &vp->frame_buffer->dimensions;
    vec3 a = project_point(A, &vp->projection_matrix), b = project_point(B, &vp->projection_matrix);
    a.x += 1; a.x *= dim->h_width;
    b.x += 1; b.x *= dim->h_width;
    a.y += 1; a.y *= dim->h_height;
    b.y += 1; b.y *= dim->h_height;
    a.y = dim->f_height - a.y;
    b.y = dim->f_height - b.y;
    draw_line(c, a.x, a.y, az, b.x, b.y, bz, color, opacity, line_width);
}

/* drawBox scene/box.h:20 with BOX__ALL_SIDES: corners to world (convertPositionToWorldSpace) and to
 * view space (camera position, inverted camera rotation), then the 12 edges */
static void draw_box(const OCanvas *c, const Viewport *vp, const Primitive *p, vec3 color, f32 opacity, u8 line_width) {
    vec3 v[8];
    const xform3 *xf = &vp->camera->transform;
    for (int i = 0; i < 8; i++) {
        vec3 q = pos_to_world(V3(kBoxCorner[i][0], kBoxCorner[i][1], kBoxCorner[i][2]), p);
        v[i] = qrot(vsub(q, xf->position), xf->rotation_inverted);
    }
    for (int e = 0; e < 12; e++) draw_edge(c, vp, v[kBoxEdge[e][0]], v[kBoxEdge[e][1]], color, opacity, line_width);
}

/* setBoxPrimitiveFromAABB raytracer.h:18 */
static void box_from_aabb(Primitive *box, const AABB *a) {
    box->rotation.axis = splat(0);
    box->rotation.amount = 1;
    box->position = vscale(vadd(a->min, a->max), 0.5f);
    box->scale = vscale(vsub(a->max, a->min), 0.5f);
    box->flags = IS_TRANSLATED | IS_SCALED | IS_SCALED_NON_UNIFORMLY;
}

/* The reference's Color() (core/base.h:577) values of the colours the overlays use */
static vec3 overlay_color(int id) {
    const f32 M = 255.0f;
    switch (id) {
        case 1: return V3(M, M, M);                     /* White */
        case 2: return V3(M / 2.0f, M / 2.0f, M / 2.0f); /* Grey */
        case 3: return V3(M, 0, 0);                     /* Red */
        case 4: return V3(0, M, 0);                     /* Green */
        case 5: return V3(0, 0, M);                     /* Blue */
        case 6: return V3(0, M, M);                     /* Cyan */
        case 7: return V3(M, 0, M);                     /* Magenta */
        case 8: return V3(M, M, 0);                     /* Yellow */
        default: return splat(0);
    }
}

void orc_draw_overlays(const Scene *sc, const Viewport *vp, int what) {
    const Dimensions *dim = &vp->frame_buffer->dimensions;
    OCanvas c;
    c.px = vp->frame_buffer->float_pixels;
    c.stride = dim->width;
    c.x_left = vp->position.x;
    c.y_top = vp->position.y;
    c.w = dim->width + c.x_left;
    c.h = dim->height + c.y_top;
    if (what & ORC_OVERLAY_BVH) {   /* drawBVH raytracer.h:46 */
        Primitive box;
        memset(&box, 0, sizeof(box));
        for (u32 node_id = 0; node_id < sc->bvh.node_count; node_id++) {
            const BVHNode *node = sc->bvh.nodes + node_id;
            int color;
            if (node->child_count) {
                for (u32 i = 0; i < node->child_count; i++) {
                    const Primitive *p = sc->primitives + sc->bvh.leaf_ids[node->first_child_id + i];
                    switch (p->type) {
                        case PrimitiveType_Box: color = 6; break;
                        case PrimitiveType_Quad: color = 1; break;
                        case PrimitiveType_Sphere: color = 8; break;
                        case PrimitiveType_Tetrahedron: color = 7; break;
                        case PrimitiveType_Mesh: {   /* drawMeshAccelerationStructure raytracer.h:33 */
                            const BVH *bvh = &sc->meshes[p->id].bvh;
                            for (u32 m = 0; m < bvh->node_count; m++) {
                                const BVHNode *mn = bvh->nodes + m;
                                if (mn->depth > 5) continue;
                                box_from_aabb(&box, &mn->aabb);   /* setBoxPrimitiveFromPrimitiveAndAABB :25 */
                                box.scale = vmul(box.scale, p->scale);
                                box.rotation = p->rotation;
                                box.flags |= IS_ROTATED;
                                box.position = pos_to_world(box.position, p);
                                draw_box(&c, vp, &box, overlay_color(mn->child_count ? 7 : (m ? 4 : 5)), 0.125f, 0);
                            }
                        } continue;
                        default: continue;
                    }
                    draw_box(&c, vp, p, overlay_color(color), 1, 1);
                }
                color = 1;
            } else color = node_id ? 2 : 5;
            box_from_aabb(&box, &node->aabb);
            draw_box(&c, vp, &box, overlay_color(color), 1, 1);
        }
    }
    if (what & ORC_OVERLAY_SSB) {   /* drawSSB SSB.h:175 with drawHLine/drawVLine line.h:5,22 */
        for (u32 i = 0; i < sc->settings.primitives; i++) {
            const Primitive *p = sc->primitives + i;
            if (!(p->flags & IS_VISIBLE)) continue;
            int color;
            switch (p->type) {
                case PrimitiveType_Box: color = 6; break;
                case PrimitiveType_Quad: color = 1; break;
                case PrimitiveType_Sphere: color = 8; break;
                case PrimitiveType_Tetrahedron: color = 7; break;
                case PrimitiveType_Mesh: color = 3; break;
                default: continue;
            }
            vec3 col = overlay_color(color);
            col = vmul(col, col);
            const vec2i mn = p->screen_bounds.min, mx = p->screen_bounds.max;
            /* two horizontal lines (rows min.y, max.y), then two vertical ones (columns min.x, max.x) */
            for (int k = 0; k < 4; k++) {
                const int horizontal = k < 2;
                i32 from = horizontal ? mn.x : mn.y, to = horizontal ? mx.x : mx.y;
                i32 at = k == 0 ? mn.y : k == 1 ? mx.y : k == 2 ? mn.x : mx.x;
                const i32 along0 = horizontal ? c.x_left : c.y_top, across0 = horizontal ? c.y_top : c.x_left;
                const i32 along_end = (horizontal ? dim->width : dim->height) + along0;
                const i32 across_end = (horizontal ? dim->height : dim->width) + across0;
                from += along0; to += along0; at += across0;
                if (!in_range(at, across_end, across0)) continue;
                i32 first = from, last = to;   /* subRange base.h:373 */
                if (to < from) { first = to; last = from; }
                first = first > along0 ? first : along0;
                last = (last < along_end ? last : along_end) - 1;
                for (i32 s = first; s <= last; s++) {
                    if (horizontal) plot(&c, s, at, 0, col, 1);
                    else plot(&c, at, s, 0, col, 1);
                }
            }
        }
    }
}
