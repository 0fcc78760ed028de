// st_render.cu — the per-frame kernels: screen-space bounds, ray-direction rows, the trace+shade
// megakernel and the QCAA resolve.
#include <cstdio>
#include "st_trace.cuh"
#include "st_kernels.h"

namespace st {

// ---- triangles and the BLAS walk: intersection/mesh.h ----------------------------------------
// hitTriangles (mesh.h:5) over the leaf's triangles: an accepted triangle (in front of the closest
// so far, inside by its tangent-space UV) becomes the closest; only its distance and slot are kept
// (finalize_hit rebuilds the rest of the record from them).
template <bool CNT, int SHS>
__device__ bool hit_triangles(TState<CNT, SHS> &t, const SceneDev &S, u32t base, u32t slot0, u32t n, bool any_hit) {
    const RayD &ray = t.local;
    bool found = false;
    for (u32t i = 0; i < n; i++) {
        TriHot T;
        {
            const float4 *f = reinterpret_cast<const float4 *>(S.tri_hot + base + i);
            asm("ld.global.nc.L1::evict_first.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(T.p.x), "=f"(T.p.y), "=f"(T.p.z), "=f"(T.p.w) : "l"(f));
            asm("ld.global.nc.L1::evict_first.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(T.q.x), "=f"(T.q.y), "=f"(T.q.z), "=f"(T.q.w) : "l"(f + 1));
            asm("ld.global.nc.L1::evict_first.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(T.r.x), "=f"(T.r.y), "=f"(T.r.z), "=f"(T.r.w) : "l"(f + 2));
            asm("ld.global.nc.L1::evict_first.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(T.s.x), "=f"(T.s.y), "=f"(T.s.z), "=f"(T.s.w) : "l"(f + 3));
        }
        t.count(C_TRI);
        v3 pos = V(T.p.x, T.p.y, T.p.z), nrm = V(T.p.w, T.q.x, T.q.y);
        Hit hit;
        if (hit_plane(pos, nrm, ray.origin, ray.direction, hit) && hit.distance < t.mesh_distance) {
            const float m[9] = {T.q.z, T.q.w, T.r.x, T.r.y, T.r.z, T.r.w, T.s.x, T.s.y, T.s.z};
            v3 UV = vmat3(hit.position - pos, m);
            if (UV.x < 0 || UV.y < 0 || (UV.x + UV.y) > 1) continue;
            t.mesh_distance = hit.distance;
            t.mesh_tri = slot0 + i;
            found = true;
            if (any_hit) break;
        }
    }
    return found;
}

// Cache hints: node pairs are marked to stay in L1 (evict_last; the top of every BLAS is read by
// every ray that enters an instance), triangle records to leave first (evict_first; a triangle is
// tested by the few neighbouring rays that reach its leaf; the 128-byte record of the winning
// triangle is read once per hit).  Hints change no value read.  Measured on the 1080p mesh frame:
// 2.14 against 2.18 ms, the triangle hints making the difference.
__device__ __forceinline__ NodePair load_pair(const NodePair *p) {
    NodePair r;
    const float4 *f = reinterpret_cast<const float4 *>(p);
    asm("ld.global.nc.L1::evict_last.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(r.a.x), "=f"(r.a.y), "=f"(r.a.z), "=f"(r.a.w) : "l"(f));
    asm("ld.global.nc.L1::evict_last.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(r.b.x), "=f"(r.b.y), "=f"(r.b.z), "=f"(r.b.w) : "l"(f + 1));
    asm("ld.global.nc.L1::evict_last.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(r.c.x), "=f"(r.c.y), "=f"(r.c.z), "=f"(r.c.w) : "l"(f + 2));
    asm("ld.global.nc.L1::evict_last.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(r.d.x), "=r"(r.d.y), "=r"(r.d.z), "=r"(r.d.w) : "l"(f + 3));
    return r;
}

template <bool CNT, int SHS>
__device__ __forceinline__ bool trace_mesh(TState<CNT, SHS> &t, const SceneDev &S, const MeshDev &M, bool any_hit) {   // mesh.h:38
    const RayD &ray = t.local;
    float ld, rd;
    t.count(C_MESH);
    t.count(C_AABB);
    if (!hit_aabb(V(M.aabb[0], M.aabb[1], M.aabb[2]), V(M.aabb[3], M.aabb[4], M.aabb[5]), ray, t.mesh_distance, ld))
        return false;
    // Leaves met at a node are tested (left, then right) before the walk moves on, as in the
    // reference; they are queued so that the triangle loop has a single call site.
    // the queue is two named slots, not an indexed array, so that it stays in registers
    u32t q0_first = 0, q0_count = 0, q1_first = 0, q1_count = 0;
    int leaves = 0;
    const NodePair *pairs = S.mesh_pairs + M.pair_offset;
    u32t pair = kNoPair;
    if (M.root_count) { q0_first = 0; q0_count = M.triangle_count; leaves = 1; }
    else pair = (M.root_first - 1) >> 1;
    u32t sp = 0;
    bool found = false;
    for (;;) {
        // inner nodes until this lane has leaves queued ("while-while": lanes of a warp walk nodes
        // together and test triangles together; each lane's own order of tests is unchanged)
        while (leaves == 0 && pair != kNoPair) {
            const NodePair P = load_pair(pairs + pair);
            t.count(C_AABB, 2);
            bool hl = hit_aabb(V(P.a.x, P.a.y, P.a.z), V(P.a.w, P.b.x, P.b.y), ray, t.mesh_distance, ld);
            bool hr = hit_aabb(V(P.b.z, P.b.w, P.c.x), V(P.c.y, P.c.z, P.c.w), ray, t.mesh_distance, rd);
            bool lgo = hl, rgo = hr;
            if (hl && P.d.y) { q0_first = P.d.x; q0_count = P.d.y; leaves = 1; lgo = false; }
            if (hr && P.d.w) {
                if (leaves) { q1_first = P.d.z; q1_count = P.d.w; }
                else { q0_first = P.d.z; q0_count = P.d.w; }
                leaves++;
                rgo = false;
            }
            if (lgo) {
                u32t near_pair = P.d.x, far_pair = P.d.z;
                if (rgo) {
                    if (!any_hit && ld > rd) { near_pair = P.d.z; far_pair = P.d.x; }
                    if (sp >= kStack) {           // the queued leaves still run, then the walk ends
                        t.status |= S_STACK_OVERFLOW;
                        pair = kNoPair;
                        continue;
                    }
                    t.push(true, sp++, far_pair);
                }
                pair = near_pair;
            } else if (rgo) {
                pair = P.d.z;
            } else {
                pair = sp ? t.at(true, --sp) : kNoPair;
            }
        }
        if (!leaves) break;
#pragma unroll 1
        for (;;) {                       // the queued leaves in order: q0, then q1
            if (hit_triangles(t, S, M.tri_offset + q0_first, q0_first, q0_count, any_hit)) {
                found = true;
                if (any_hit) return true;
            }
            if (--leaves == 0) break;
            q0_first = q1_first;
            q0_count = q1_count;
        }
        if (pair == kNoPair) break;
    }
    return found;
}

// The primitive record again, by a load the compiler cannot merge with the first one: after a BLAS
// walk the candidate's transform is reloaded (an L1 hit) instead of being held in registers, or
// spilled, through the walk.
__device__ __forceinline__ PrimDev load_prim_again(const PrimDev *p) {
    PrimDev r;
    asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(r.pos_bits.x), "=f"(r.pos_bits.y), "=f"(r.pos_bits.z), "=f"(r.pos_bits.w) : "l"(&p->pos_bits));
    asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(r.rot.x), "=f"(r.rot.y), "=f"(r.rot.z), "=f"(r.rot.w) : "l"(&p->rot));
    asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(r.scale_id.x), "=f"(r.scale_id.y), "=f"(r.scale_id.z), "=f"(r.scale_id.w) : "l"(&p->scale_id));
    asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(r.inv_scale.x), "=f"(r.inv_scale.y), "=f"(r.inv_scale.z), "=f"(r.inv_scale.w) : "l"(&p->inv_scale));
    return r;
}

// ---- hitPrimitives intersection/primitives.h:9 ----------------------------------------------------
// ids == nullptr: the candidates are primitives first..first+count-1 in index order.
// The candidate loop keeps the reference's order and comparisons; a winner updates t.best (the
// hit test's distance, the world position and its squared distance, which the next candidates and
// the walk read), and a call that found one ends with the world distance, as hitPrimitives' final
// step leaves it (primitives.h:105).  The rest of that final step is finalize_hit's.
template <bool CNT, int SHS>
__device__ __forceinline__ bool hit_primitives(TState<CNT, SHS> &t, const SceneDev &S, const RayD &ray, const u32t *ids, u32t first,
                               u32t count, bool any_hit, const int4 *ssb, int x, int y) {
    Best &best = t.best;
    bool found = false;
    for (u32t i = 0; i < count; i++) {
        t.count(C_LEAF);
        const u32t pid = ids ? __ldg(ids + first + i) : first + i;
        if (ssb) {  // primary rays: IS_VISIBLE and the screen-space rect, folded into one rect per view
            const int4 b = __ldg(ssb + pid);
            if (x < b.x || x >= b.z || y < b.y || y >= b.w) continue;
        }
        const PrimDev P = S.prims[pid];
        const unsigned flags = prim_flags(P);
        if (any_hit && !(flags & IS_SHADOWING)) continue;
        t.count(C_PRIM);
        to_object(ray.origin, ray.direction, P, t.local.origin, t.local.direction);
        t.local.origin = vsfma(t.local.direction, kTraceOffset, t.local.origin);
        bool cur;
        float dist = 0.0f;
        v3 pos = splat(0.0f);
        u32t tri = 0;
        const unsigned type = prim_type(P);
        if (type == PrimitiveType_Mesh) {
            t.local.rcp = rcp(t.local.direction);
            t.mesh_distance = best.distance == INFINITY ? INFINITY :
                len(pos_to_object(best.position, P) - t.local.origin);
            pre_prep(t.local);
            const u32t mesh = __float_as_uint(P.scale_id.w);
            cur = trace_mesh(t, S, S.meshes[mesh], any_hit);
            if (cur) {
                // the accepted triangle's object-space hit point, recomputed exactly as
                // hit_triangles computed it (same triangle, same ray, same operations)
                const MeshDev &M = S.meshes[mesh];
                tri = t.mesh_tri;
                const float4 tp = __ldg(reinterpret_cast<const float4 *>(S.tri_hot + M.tri_offset + tri));
                const float4 tq = __ldg(reinterpret_cast<const float4 *>(S.tri_hot + M.tri_offset + tri) + 1);
                Hit h;
                hit_plane(V(tp.x, tp.y, tp.z), V(tp.w, tq.x, tq.y), t.local.origin, t.local.direction, h);
                pos = h.position;
                dist = t.mesh_distance;
            }
        } else {
            Hit hit;
            switch (type) {
                case PrimitiveType_Quad: cur = hit_quad(hit, t.local.origin, t.local.direction, flags); break;
                case PrimitiveType_Box: cur = hit_box(hit, t.local.origin, t.local.direction, flags); break;
                case PrimitiveType_Sphere: cur = hit_sphere(hit, t.local.origin, t.local.direction, flags); break;
                case PrimitiveType_Tetrahedron: cur = hit_tetra(hit, t.local.origin, t.local.direction, flags); break;
                default: continue;
            }
            pos = hit.position;
            dist = hit.distance;
        }
        if (cur) {
            pos = pos_to_world(pos, type == PrimitiveType_Mesh ? load_prim_again(S.prims + pid) : P);
            const float dsq = sqlen(pos - ray.origin);
            if (dsq < best.distance_squared) {
                best.distance_squared = dsq;
                best.distance = dist;
                best.position = pos;
                best.prim = pid;
                best.tri = tri;
                found = true;
                if (any_hit) break;
            }
        }
    }
    if (found) best.distance = sqrtf(best.distance_squared);
    return found;
}

// The closest hit's full record (hitPrimitives' copy of the winner's RayHit and its final step,
// primitives.h:63-108), rebuilt after a walk that found t.best: the winner's hit test runs again on
// the same object-space ray (to_object and the offset as in the candidate loop), which gives the
// record the candidate loop saw bit for bit; then the barycentric interpolation of mesh normals and
// uvs, the primitive id, the world normal, distance, cone width and area.
template <bool CNT, int SHS>
__device__ __forceinline__ void finalize_hit(TState<CNT, SHS> &t, const SceneDev &S, const RayD &ray, float cone_angle) {
    Hit &closest = t.closest;
    const u32t hid = t.best.prim;
    const PrimDev HP = S.prims[hid];
    const unsigned flags = prim_flags(HP), type = prim_type(HP);
    v3 lo, ld;
    to_object(ray.origin, ray.direction, HP, lo, ld);
    lo = vsfma(ld, kTraceOffset, lo);
    switch (type) {
        case PrimitiveType_Quad: hit_quad(closest, lo, ld, flags); break;
        case PrimitiveType_Box: hit_box(closest, lo, ld, flags); break;
        case PrimitiveType_Sphere: hit_sphere(closest, lo, ld, flags); break;
        case PrimitiveType_Tetrahedron: hit_tetra(closest, lo, ld, flags); break;
        default: {                                              // PrimitiveType_Mesh
            const MeshDev &M = S.meshes[__float_as_uint(HP.scale_id.w)];
            const u32t tri = t.best.tri;
            const TriHot T = S.tri_hot[M.tri_offset + tri];
            const v3 pos = V(T.p.x, T.p.y, T.p.z);
            hit_plane(pos, V(T.p.w, T.q.x, T.q.y), lo, ld, closest);
            const float m[9] = {T.q.z, T.q.w, T.r.x, T.r.y, T.r.z, T.r.w, T.s.x, T.s.y, T.s.z};
            const v3 UV = vmat3(closest.position - pos, m);
            closest.u = UV.x;
            closest.v = UV.y;
            Triangle TF;
            {
                const float4 *f = reinterpret_cast<const float4 *>(S.tri_full + M.tri_offset + tri);
                float4 *o = reinterpret_cast<float4 *>(&TF);
#pragma unroll
                for (int k = 0; k < 8; k++)
                    asm("ld.global.nc.L1::evict_first.v4.f32 {%0,%1,%2,%3}, [%4];"
                        : "=f"(o[k].x), "=f"(o[k].y), "=f"(o[k].z), "=f"(o[k].w) : "l"(f + k));
            }
            closest.area = TF.area_of_parallelogram;
            closest.uv_area = TF.area_of_uv;
            if (M.normals_count | M.uvs_count) {
                float u = closest.u, v = closest.v;
                float w = 1 - u - v;
                if (M.uvs_count) {
                    closest.u = TF.uvs[2].x * u + (TF.uvs[1].x * v + TF.uvs[0].x * w);
                    closest.v = TF.uvs[2].y * u + (TF.uvs[1].y * v + TF.uvs[0].y * w);
                }
                if (M.normals_count) {
                    const vec3 *vn = TF.vertex_normals;
                    closest.normal.x = vn[2].x * u + (vn[1].x * v + vn[0].x * w);
                    closest.normal.y = vn[2].y * u + (vn[1].y * v + vn[0].y * w);
                    closest.normal.z = vn[2].z * u + (vn[1].z * v + vn[0].z * w);
                    closest.normal = norm(closest.normal);
                }
            }
        } break;
    }
    closest.position = t.best.position;
    closest.distance_squared = t.best.distance_squared;
    closest.object_type = type;
    closest.material_id = prim_material(HP);
    closest.object_id = hid;
    closest.normal = norm(dir_to_world(closest.normal, HP));
    closest.distance = t.best.distance;
    closest.cone_width = 2.0f * cone_angle * closest.distance;
    v3 rs = qrot(V(HP.scale_id.x, HP.scale_id.y, HP.scale_id.z), prim_rot(HP));
    closest.area *= dot(one_minus(closest.normal), rs);
}

// ---- traceScene shaders/trace.h:8 (TLAS walk); with ssb != null it also serves primary rays ----
// The primitive loop, the BLAS walk and the triangle loop each have one call site here, so every
// inlined copy of the walk carries one copy of them (the instruction footprint of the megakernel).
// all_prims: test every primitive in leaf-id order without the root box (the primary-ray path of
// scenes with few primitives, raytracer.h:100).
template <bool CNT, int SHS>
__device__ __forceinline__ bool trace_scene(TState<CNT, SHS> &t, const SceneDev &S, RayD &ray, bool any_hit, const int4 *ssb,
                                            int x, int y, bool prepped, bool all_prims) {
    if (!prepped) {
        ray.rcp = rcp(ray.direction);
        pre_prep(ray);
    }
    float ld, rd;
    u32t q0_first = 0, q0_count = 0, q1_first = 0, q1_count = 0;   // the leaf queue, as in trace_mesh
    int leaves = 0;
    u32t pair = kNoPair;
    if (!all_prims) {
        t.count(C_AABB);
        if (!hit_aabb(V(S.tlas_root_aabb[0], S.tlas_root_aabb[1], S.tlas_root_aabb[2]),
                      V(S.tlas_root_aabb[3], S.tlas_root_aabb[4], S.tlas_root_aabb[5]), ray, t.best.distance, ld))
            return false;
    }
    if (all_prims || S.tlas_root_count) { q0_first = 0; q0_count = S.n_prims; leaves = 1; }
    else pair = (S.tlas_root_first - 1) >> 1;
    u32t sp = 0;
    bool found = false;
    for (;;) {
        while (leaves == 0 && pair != kNoPair) {      // inner nodes until leaves are queued
            const NodePair P = load_pair(S.tlas_pairs + pair);
            t.count(C_AABB, 2);
            bool hl = hit_aabb(V(P.a.x, P.a.y, P.a.z), V(P.a.w, P.b.x, P.b.y), ray, t.best.distance, ld);
            bool hr = hit_aabb(V(P.b.z, P.b.w, P.c.x), V(P.c.y, P.c.z, P.c.w), ray, t.best.distance, rd);
            bool lgo = hl, rgo = hr;
            if (hl && P.d.y) { q0_first = P.d.x; q0_count = P.d.y; leaves = 1; lgo = false; }
            if (hr && P.d.w) {
                if (leaves) { q1_first = P.d.z; q1_count = P.d.w; }
                else { q0_first = P.d.z; q0_count = P.d.w; }
                leaves++;
                rgo = false;
            }
            if (lgo) {
                u32t near_pair = P.d.x, far_pair = P.d.z;
                if (rgo) {
                    if (!any_hit && ld > rd) { near_pair = P.d.z; far_pair = P.d.x; }
                    if (sp >= kStack) {           // the queued leaves still run, then the walk ends
                        t.status |= S_STACK_OVERFLOW;
                        pair = kNoPair;
                        continue;
                    }
                    t.push(false, sp++, far_pair);
                }
                pair = near_pair;
            } else if (rgo) {
                pair = P.d.z;
            } else {
                pair = sp ? t.at(false, --sp) : kNoPair;
            }
        }
        if (!leaves) break;
#pragma unroll 1
        for (;;) {
            if (hit_primitives(t, S, ray, S.tlas_leaf_ids, q0_first, q0_count, any_hit, ssb, x, y)) {
                found = true;
                if (any_hit) return true;
            }
            if (--leaves == 0) break;
            q0_first = q1_first;
            q0_count = q1_count;
        }
        if (pair == kNoPair) break;
    }
    return found;
}

// ---- closest_hit/surface.h, lights.h ------------------------------------------------------------
template <bool CNT, int SHS>
__device__ v3 shade_from_lights(TState<CNT, SHS> &t, const SceneDev &S, Shaded &s, RayD &ray, v3 color) {   // surface.h:9
    // The reference writes each light into trace->closest_hit (:14-17) and the shadow ray's walk
    // reads it there (the occluder must be nearer than the light) or overwrites it with an
    // occluder: the walk's record t.best plays that part, and closest_hit's position and distances
    // are left as the last light's walk left them, because the emissive-quad test reads them (:55).
    Best &b = t.best;
    for (u32t i = 0; i < S.n_lights; i++) {
        const Light &light = S.lights[i];
        b.position = from(light.position_or_direction);
        s.light_direction = b.position - s.position;
        b.distance_squared = sqlen(s.light_direction);
        b.distance = sqrtf(b.distance_squared);
        s.light_direction = vscale(s.light_direction, 1.0f / b.distance);
        float NdotL = dot(s.normal, s.light_direction);
        if (NdotL <= 0) continue;
        float li = light.intensity / b.distance_squared;
        ray.origin = s.position;
        ray.direction = s.light_direction;
        t.count(C_SHADOW);
        if (trace_scene(t, S, ray, true, nullptr, 0, 0, false, false)) continue;       // inShadow trace.h:85
        color = vvfma(shade_point(s, NdotL), vscale(from(light.color), li), color);
    }
    if (S.n_lights) {
        t.closest.position = b.position;
        t.closest.distance_squared = b.distance_squared;
        t.closest.distance = b.distance;
    }
    return color;
}

template <bool CNT, int SHS>
__device__ bool shade_from_emissive_quads(TState<CNT, SHS> &t, const SceneDev &S, Shaded &s, RayD &ray, v3 &color) {  // surface.h:37
    Hit hit;                                    // the reference's trace->current_hit, scratch here
    bool found = false;
    for (u32t e = 0; e < S.n_emissive; e++) {
        const u32t qi = S.emissive_quads[e];
        const PrimDev Q = S.prims[qi];
        const Primitive &quad = S.prims_raw[qi];
        const Material &em = S.materials[prim_material(Q)];
        v3 Ro, Rd;
        to_object(s.viewing_origin, s.viewing_direction, Q, Ro, Rd);
        if (hit_quad(hit, Ro, Rd, prim_flags(Q))) {
            hit.position = pos_to_world(hit.position, Q);
            hit.distance_squared = sqlen(hit.position - s.viewing_origin);
            if (hit.distance_squared < t.closest.distance_squared) {
                hit.object_id = qi;
                hit.object_type = PrimitiveType_Quad;
                hit.material_id = prim_material(Q);
                t.closest = hit;
                found = true;
            }
        }
        v3 qn = qrot(V(0, 1, 0), prim_rot(Q));
        v3 qpos = V(Q.pos_bits.x, Q.pos_bits.y, Q.pos_bits.z);
        s.light_direction = ray.direction = qpos - s.position;
        if (dot(qn, s.light_direction) >= 0) continue;
        float ei = dot(s.normal, area_light_vector(quad, s.position, s.quad_vertices));
        if (ei > 0) {
            bool skip = true;
            for (int j = 0; j < 4; j++)
                if (dot(s.normal, s.quad_vertices[j] - s.position) >= 0) { skip = false; break; }
            if (skip) continue;
            float shaded_light = 1;
            if (qi != s.prim_index) {
                for (u32t k = 0; k < S.n_occluders; k++) {
                    const u32t oi = S.occluders[k];
                    const PrimDev O = S.prims[oi];
                    if (oi == qi || dot(qn, V(O.pos_bits.x, O.pos_bits.y, O.pos_bits.z) - qpos) <= 0) continue;
                    v3 oRo, oRd;
                    to_object(s.position, s.light_direction, O, oRo, oRd);
                    oRo = vsfma(oRd, kTraceOffset, oRo);
                    float d = 1;
                    if (prim_type(O) == PrimitiveType_Sphere) {
                        if (hit_sphere(hit, oRo, oRd, prim_flags(O)))
                            d -= (1.0f - sqrtf(hit.distance_squared)) / (hit.distance * ei * 3);
                    } else {
                        if (hit_quad(hit, oRo, oRd, prim_flags(O))) {
                            hit.position.y = 0;
                            hit.position.x = hit.position.x < 0 ? -hit.position.x : hit.position.x;
                            hit.position.z = hit.position.z < 0 ? -hit.position.z : hit.position.z;
                            if (hit.position.x > hit.position.z) {
                                hit.position.y = hit.position.z;
                                hit.position.z = hit.position.x;
                                hit.position.x = hit.position.y;
                                hit.position.y = 0;
                            }
                            d -= (1.0f - hit.position.z) / (hit.distance * ei);
                        }
                    }
                    if (d < shaded_light) shaded_light = d;
                }
            }
            if (shaded_light > 0) {
                float NdotL = dot01(s.normal, s.light_direction);
                if (NdotL) color = vvfma(shade_point(s, NdotL), vscale(from(em.emission), ei * shaded_light), color);
            }
        }
    }
    if (found) t.closest.distance = sqrtf(t.closest.distance_squared);
    return found;
}

__device__ __forceinline__ float volume_density(const SphereHitD &h) {   // lights.h:7
    float t1 = h.t_near > 0 ? h.t_near : 0;
    float t2 = h.t_far < h.furthest ? h.t_far : h.furthest;
    return (h.c * t1 - h.b * t1 * t1 + t1 * t1 * t1 / 3.0f - (
            h.c * t2 - h.b * t2 * t2 + t2 * t2 * t2 / 3.0f)) * (3.0f / 4.0f);
}
template <bool CNT, int SHS>
__device__ bool shade_lights(TState<CNT, SHS> &t, const SceneDev &S, v3 Ro, v3 Rd, float max_distance, v3 &color) {  // lights.h:17
    bool hit_light = false;
    SphereHitD &sh = t.sphere;
    sh.closest_distance = INFINITY;
    for (u32t i = 0; i < S.n_lights; i++) {
        const Light &light = S.lights[i];
        float size = light.intensity * (1.0f / 16.0f);
        float oor = 8.0f / size;
        sh.furthest = max_distance * oor;
        if (hit_sphere_simple(Ro, Rd, from(light.position_or_direction), oor, sh)) {
            float distance = sh.t_far - size * 8;
            float density = powf(volume_density(sh), 8) * 8;
            if (distance < sh.closest_distance) sh.closest_distance = distance;
            color = vsfma(from(light.color), density, color);
            hit_light = true;
        }
    }
    return hit_light;
}

template <bool CNT, int SHS>
__device__ __forceinline__ void apply_textures(TState<CNT, SHS> &t, const SceneDev &S, Shaded &s, Hit &hit, const Material &M,
                                               float &du, float &dv, bool first) {
    s.u = hit.u * M.uv_repeat.x;
    s.v = hit.v * M.uv_repeat.y;
    hit.uv_area /= M.uv_repeat.x / M.uv_repeat.y;
    float d = duv_ray_cone(hit.NdotV, hit.cone_width, hit.area, hit.uv_area);
    du = d;
    if (first) dv = d;              // surface.h:162 sets u and v; the bounce path (:230) only u
    if (M.use & ALBEDO_MAP) s.albedo = sample_texture(t, S, M.texture_ids[0], s.u, s.v, du, dv);
    if ((M.use & NORMAL_MAP) && M.texture_count > 1) {
        q4 rot = normal_rotation(sample_normal(t, S, M.texture_ids[1], s.u, s.v, du, dv));
        hit.normal = qrot(hit.normal, rot);
    }
}

// ---- the frame kernels -----------------------------------------------------------------------
// computeSSB render/SSB.h:5 for one primitive; the result is folded with IS_VISIBLE into one rect
// (an invisible primitive gets an empty rect) so that the primary-ray cull is a single test.
__device__ bool compute_ssb(int4 &b, v3 pos, float r, float fl, const ViewDev &v) {
    b.x = v.grid_w + 1; b.z = v.grid_w + 1; b.y = v.grid_h + 1; b.w = v.grid_h + 1;
    if (pos.z <= -r) return false;
    float x = pos.x, y = pos.y, z = pos.z, left, right, top, bottom, factor;
    if (z <= r) {
        float h = fabsf(z) / fl;
        top = y + r;
        bottom = y - r;
        if (h < bottom || top < -h) return false;
        float w = h * v.width_over_height;
        right = x + r;
        left = x - r;
        if (w < left || right < -w) return false;
        b.x = -w < left ? (int)(uint16_t)(v.f_width * (left + w) / (2 * w)) : 0;
        b.z = right < w ? (int)(uint16_t)(v.f_width * (right + w) / (2 * w)) : (int)v.grid_w;
        b.y = top < h ? (int)(uint16_t)(v.f_height * (h - top) / (2 * h)) : 0;
        b.w = -h < bottom ? (int)(uint16_t)(v.f_height * (h - bottom) / (2 * h)) : (int)v.grid_h;
        return true;
    }
    float den = z * z - r * r;
    factor = fl / den;
    float yz = y * z;
    float sqr = y * y + den;
    sqr = r * sqrtf(sqr);
    bottom = factor * (yz - sqr);
    top = factor * (yz + sqr);
    if (bottom < 1 && top > -1) {
        factor *= v.height_over_width;
        float xz = x * z;
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
            b.x = (int)(uint16_t)(v.h_width * left);
            b.z = (int)(uint16_t)(v.h_width * right);
            b.w = (int)(uint16_t)(v.h_height * bottom);
            b.y = (int)(uint16_t)(v.h_height * top);
            return true;
        }
    }
    return false;
}

// updatePrimitiveSSB render/SSB.h:137 for primitive i of one view
__device__ __forceinline__ void ssb_one(const SceneDev &S, const ViewDev &v, int4 *ssb, u32t i) {
    const Primitive p = S.prims_raw[i];
    v3 view = vmat3(from(p.position) - v.cam_pos, v.cam_rot_matrix_inv);
    float radius;
    v3 sc = from(p.scale);
    switch (p.type) {
        case PrimitiveType_Quad: case PrimitiveType_Box: radius = len(sc); break;
        case PrimitiveType_Tetrahedron: { float m = sc.x; if (sc.y > m) m = sc.y; if (sc.z > m) m = sc.z; radius = m * kSqrt2; } break;
        case PrimitiveType_Sphere: { float m = sc.x; if (sc.y > m) m = sc.y; if (sc.z > m) m = sc.z; radius = m; } break;
        case PrimitiveType_Mesh: {
            const MeshDev &M = S.meshes[p.id];
            float mn = len(vmul(sc, V(M.mesh_aabb[0], M.mesh_aabb[1], M.mesh_aabb[2])));
            float mx = len(vmul(sc, V(M.mesh_aabb[3], M.mesh_aabb[4], M.mesh_aabb[5])));
            radius = mx > mn ? mx : mn;
        } break;
        default: {
            // updatePrimitiveSSB returns without touching other types: keep the uploaded values
            const bool vis = p.flags & IS_VISIBLE;
            ssb[i] = vis ? make_int4(p.screen_bounds.min.x, p.screen_bounds.min.y, p.screen_bounds.max.x, p.screen_bounds.max.y)
                         : make_int4(1, 1, 0, 0);
            return;
        }
    }
    int4 b;
    bool vis = compute_ssb(b, view, radius, v.focal_length, v);
    ssb[i] = vis ? b : make_int4(1, 1, 0, 0);
}
__global__ void ssb_kernel(SceneDev S, ViewDev v, int4 *ssb) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S.n_prims) ssb_one(S, v, ssb, i);
}

// The reference walks each row of the QCAA grid by repeated addition (raytracer.h:156-170):
// row y starts at start + down added y times, pixel x at that plus right added x times.  That
// sequence is kept exactly: one thread per row walks it and stores every kSegment-th value
// ("segment starts", 3 MB at 1080p instead of a 25 MB direction table); the trace kernel adds
// `right` the remaining x % kSegment times itself.  The starts are stored segment-major (segment k
// of every row, row after row), so that the threads of a warp, one per row, write one contiguous
// run per segment, and a warp tile's four rows read 48 contiguous bytes.
__device__ __forceinline__ void row_segments_one(const ViewDev &v, float *seg, u32t row) {
    v3 cur = v.pp_start;
    for (u32t y = 0; y < row; y++) cur = cur + v.pp_down;
    const u32t nseg = (v.grid_w + kSegment - 1) / kSegment;
    for (u32t k = 0; k < nseg; k++) {
        float *out = seg + ((size_t)k * v.grid_h + row) * 3;
        out[0] = cur.x;
        out[1] = cur.y;
        out[2] = cur.z;
        for (int i = 0; i < kSegment; i++) cur = cur + v.pp_right;
    }
}
__global__ void row_segments_kernel(ViewDev v, float *seg) {
    const u32t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row < v.grid_h) row_segments_one(v, seg, row);
}

__device__ __forceinline__ v3 grid_direction(const ViewDev &v, const float *seg, u32t x, u32t y) {
    const float *s = seg + ((size_t)(x / kSegment) * v.grid_h + y) * 3;
    v3 cur = V(__ldg(s), __ldg(s + 1), __ldg(s + 2));
    for (u32t i = 0; i < x % kSegment; i++) cur = cur + v.pp_right;
    return cur;
}

// rayTrace render/raytracer.h:81 for one QCAA grid point, writing the FloatPixel the reference's
// setPixel leaves after beginDrawing's clear (viewport.h:88): hit -> (color, 1, z), miss ->
// (black, 0, +inf).
// park (optional): at each bounce, a warp whose lanes still tracing number fewer than
// park->threshold parks those lanes' paths in the queue (returns false: the point is not finished,
// nothing is written); resume (optional): a parked path, continued from its bounce ray.  A path
// runs the same steps whether it is parked or not, so the outputs and counters do not change.
template <bool CNT, int SHS>
__device__ __forceinline__ bool trace_point(TState<CNT, SHS> &t, const SceneDev &S, const ViewDev &v, const int4 *ssb,
                                            const float *dirs, u32t x, u32t y, FloatPixel *out, u32t *prim_ids,
                                            const ParkQueue *park = nullptr,
                                            u32t view_index = 0, const ParkedRay *resume = nullptr) {
    const size_t idx = (size_t)y * v.grid_w + x;
    const v3 Ro = v.cam_pos, Rd = norm(grid_direction(v, dirs, x, y));
    RayD ray;
    t.depth = v.depth;
    t.closest.distance = t.closest.distance_squared = INFINITY;
    t.closest.cone_width = 0;
    t.best.distance = t.best.distance_squared = INFINITY;
    v3 color = splat(0);
    bool lights_shaded = false, hit_found = false;
    float closest_distance = INFINITY, z = INFINITY;
    Hit &hit = t.closest;
    // shadeSurface's state (surface.h:146)
    Shaded s;
    const Material *M = nullptr;
    float du = 0, dv = 0, NdotRd = 0, ior = 0, max_distance = 0;
    v3 throughput = splat(1);
    u32t bounces = 0;                                       // shadeSurface's `depth`
    bool primary = true;
    if (resume) {                                           // a parked path, at its bounce ray
        const ParkedRay &P = *resume;
        ray.origin = V(P.origin_r.x, P.origin_r.y, P.origin_r.z);
        ray.direction = V(P.direction_g.x, P.direction_g.y, P.direction_g.z);
        color = V(P.origin_r.w, P.direction_g.w, P.throughput_b.w);
        throughput = V(P.throughput_b.x, P.throughput_b.y, P.throughput_b.z);
        du = P.carry.x;
        dv = P.carry.y;
        max_distance = P.carry.z;
        closest_distance = P.carry.w;
        z = P.depth.x;
        bounces = P.where.w >> 2;
        lights_shaded = (P.where.w >> 1) & 1u;
        hit_found = P.where.w & 1u;
        primary = false;
    } else {
        ray.origin = Ro;
        ray.direction = Rd;
        ray.rcp = rcp(ray.direction);
        pre_prep(ray);      // only the walk reads the prepared fields; every bounce ray prepares its own
        t.count(C_PRIMARY);
    }
    // The primary ray and every bounce ray of shadeSurface's loop share this one trace site, so the
    // kernel carries one inlined copy of the walk for both (shadow rays keep theirs).
    for (;;) {
        const bool found = trace_scene(t, S, ray, false, primary ? ssb : nullptr, (int)x, (int)y, primary,
                                       primary && !v.primary_tlas);
        if (found) finalize_hit(t, S, ray, primary ? v.cone_angle : 0.0f);
        if (primary) {                                      // rayTrace after the hit test (raytracer.h:89)
            primary = false;
            hit_found = found;
            if (prim_ids) __stcs(prim_ids + idx, found ? hit.object_id : 0xFFFFFFFFu);
            closest_distance = found ? hit.distance : INFINITY;
            if (!found) break;
            z = qrot(hit.position - v.cam_pos, v.cam_rot_inv).z;
            if (v.mode != RenderMode_Beauty) {
                switch (v.mode) {
                    case RenderMode_Depth: color = splat(4 / hit.distance); break;
                    case RenderMode_Normals: {
                        const Material &NM = S.materials[hit.material_id];
                        if (NM.texture_count > 1 && (NM.use & NORMAL_MAP)) {
                            float u = hit.u * NM.uv_repeat.x, vv = hit.v * NM.uv_repeat.y;
                            hit.uv_area /= NM.uv_repeat.x / NM.uv_repeat.y;
                            float ndu = duv_ray_cone(hit.NdotV, hit.cone_width, hit.area, hit.uv_area);
                            q4 rot = normal_rotation(sample_normal(t, S, NM.texture_ids[1], u, vv, ndu, 0.0f));
                            hit.normal = qrot(hit.normal, rot);
                        }
                        color = V(0.5f * (hit.normal.x + 1), 0.5f * (hit.normal.y + 1), 0.5f * (hit.normal.z + 1));
                    } break;
                    case RenderMode_UVs: color = V(0.5f * hit.u, 0.5f * hit.v, 0.5f); break;
                }
                break;
            }
            // shadeSurface (surface.h:146) up to its bounce loop
            M = S.materials + hit.material_id;
            t.count(C_SHADE);
            if (M->is & EMISSIVE) {
                if (!hit.from_behind) color = from(M->emission);
                break;
            }
            s.viewing_origin = ray.origin;
            s.viewing_direction = ray.direction;
            s.prim_index = hit.object_id;
            s.material = M;
            s.albedo = from(M->albedo);
            s.reflected_direction = splat(0);
            if (M->use && M->texture_count) apply_textures(t, S, s, hit, *M, du, dv, true);
            max_distance = hit.distance;
            bounces = t.depth;
        } else {                                            // traceRay returned (surface.h:214-239)
            if (!found) break;
            t.count(C_SHADE);
            s.prim_index = hit.object_id;
            s.material = M = S.materials + hit.material_id;
            s.albedo = from(M->albedo);
            if (M->use && M->texture_count) apply_textures(t, S, s, hit, *M, du, dv, false);
            if (hit.object_type == PrimitiveType_Quad && (M->is & EMISSIVE)) {
                color = hit.from_behind ? splat(0) : from(M->emission);
                break;
            }
            if (M->brdf != BRDF_CookTorrance) throughput = vmul(throughput, from(M->reflectivity));
            s.viewing_origin = ray.origin;
            s.viewing_direction = ray.direction;
        }
        // one iteration of shadeSurface's bounce loop
        if (!bounces) break;
        s.position = ray.origin = hit.position;
        s.normal = hit.from_behind ? neg(hit.normal) : hit.normal;
        ior = hit.from_behind ? s.material->n2_over_n1 : s.material->n1_over_n2;
        const bool is_ref = (M->is & REFLECTIVE) || (M->is & REFRACTIVE);
        if (is_ref || M->brdf == BRDF_Phong) {
            NdotRd = -clamp01(-dot(s.normal, s.viewing_direction));      // invDotVec3 common.h:97
            s.reflected_direction = vsfma(s.normal, -2.0f * NdotRd, s.viewing_direction);  // reflectWithDot :101
        }
        v3 cur = is_ref ? splat(0) : from(S.ambient);
        if (S.lights) cur = shade_from_lights(t, S, s, ray, cur);
        if (S.n_emissive)
            if (shade_from_emissive_quads(t, S, s, ray, cur)) max_distance = hit.distance;
        color = vvfma(cur, throughput, color);
        if (S.lights && shade_lights(t, S, s.viewing_origin, s.viewing_direction, max_distance, color))
            lights_shaded = true;
        if (!(is_ref && --bounces)) break;
        if (M->is & REFLECTIVE) ray.direction = s.reflected_direction;
        else {                                                         // refract common.h:105
            v3 Vv = s.viewing_direction, N = s.normal;
            float c = ior * ior * (1 - (NdotRd * NdotRd));
            if (c > 1) ray.direction = splat(0);
            else {
                Vv = vscale(Vv, ior);
                Vv = vsfma(N, ior * -NdotRd - sqrtf(1 - c), Vv);
                ray.direction = norm(Vv);
            }
            if (ray.direction.x == 0 && ray.direction.y == 0 && ray.direction.z == 0)
                ray.direction = s.reflected_direction;
        }
        t.count(C_BOUNCE);
        t.closest.distance = t.closest.distance_squared = INFINITY;           // traceRay trace.h:89
        t.best.distance = t.best.distance_squared = INFINITY;
        if (park && park->threshold) {
            // warp-vote compaction: the lanes at this bounce are the warp's lanes still tracing
            const unsigned mask = __activemask();
            const u32t n = __popc(mask);
            if (n < park->threshold) {
                const u32t lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
                u32t base = 0;
                if (lane == leader) base = atomicAdd(park->reserved, n);
                base = __shfl_sync(mask, base, leader);
                const u32t slot = base + __popc(mask & ((1u << lane) - 1u));
                if (base + n <= park->capacity) {
                    ParkedRay &P = park->rays[slot];
                    P.origin_r = make_float4(ray.origin.x, ray.origin.y, ray.origin.z, color.x);
                    P.direction_g = make_float4(ray.direction.x, ray.direction.y, ray.direction.z, color.y);
                    P.throughput_b = make_float4(throughput.x, throughput.y, throughput.z, color.z);
                    P.carry = make_float4(du, dv, max_distance, closest_distance);
                    P.where = make_uint4(x, y, view_index, (bounces << 2) | ((u32t)lights_shaded << 1) | (u32t)hit_found);
                    P.depth = make_float4(z, 0.0f, 0.0f, 0.0f);
                    return false;
                }
                // the queue is full: these paths go on here; slots of the refused range that lie
                // inside the queue are marked empty for the drain
                if (slot < park->capacity) park->rays[slot].where = make_uint4(0, 0, kEmptySlot, 0);
            }
        }
    }
    if (v.mode == RenderMode_Beauty && S.lights && !lights_shaded) {
        if (shade_lights(t, S, Ro, Rd, closest_distance, color)) {
            hit_found = true;
            z = t.sphere.closest_distance;
        }
    }
    float4 c01;
    double depth;
    if (hit_found) {
        if (v.mode == RenderMode_Beauty) {
            color.x = tone_mapped(color.x);
            color.y = tone_mapped(color.y);
            color.z = tone_mapped(color.z);
        }
        color = vscale(color, 255.0f);
        color = vmul(color, color);
        c01 = make_float4(color.x, color.y, color.z, 1.0f);
        depth = (double)z;
    } else {
        c01 = make_float4(0, 0, 0, 0);
        depth = (double)INFINITY;
    }
    // streaming stores: the grid is written once and read back by a copy or the resolve, so its
    // lines go first from L2 rather than the scene's nodes (0.5 % off the 1080p mesh frame)
    float2 *o = reinterpret_cast<float2 *>(out + idx);
    __stcs(o, make_float2(c01.x, c01.y));
    __stcs(o + 1, make_float2(c01.z, c01.w));
    __stcs(reinterpret_cast<double *>(o) + 2, depth);
    return true;
}

template <bool CNT, int SHS>
__device__ __forceinline__ void flush_counters(TState<CNT, SHS> &t, unsigned *status, unsigned long long *counters) {
    if (t.status) atomicOr(status, t.status);
    if (CNT) {
        const u32t lane = threadIdx.x & 31;
        for (int k = 0; k < C_COUNT; k++) {
            unsigned long long s = t.cnt[k];
            for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, off);
            if (lane == 0 && s) atomicAdd(counters + k, s);
        }
    }
}

// Resident 128-thread blocks per SM the register allocation must allow.  Eight (64 registers, more
// spills) beat the compiler's own choice of 128 registers (four blocks) on the 1080p mesh frame
// (2.38 vs 2.62 ms), and six and seven blocks (2.42, 2.40 ms) there, on the 64-view mixed batch and
// on the served stream; 5 blocks measured 2.52 ms, 2 blocks 5.6 ms.
// The per-frame trace kernel with device outputs runs nine blocks (56 registers): 2.101 ms against
// 2.110 at eight and 2.176 at ten on the 1080p mesh frame.  A frame whose float grid is copied to
// the host while it is traced runs with fewer blocks (more registers, fewer spills): its spill
// traffic and the copies slow each other, and on the 1080p mesh frame six blocks measured 2.19 ms
// alone but 798-803 Mrays/s end to end against 776 at eight.
#ifndef ST_TRACE_MIN_BLOCKS
#define ST_TRACE_MIN_BLOCKS 8
#endif
#ifndef ST_TRACE_DEVICE_MIN_BLOCKS
#define ST_TRACE_DEVICE_MIN_BLOCKS 9
#endif
#ifndef ST_TRACE_OVERLAP_MIN_BLOCKS
#define ST_TRACE_OVERLAP_MIN_BLOCKS 6
#endif
#define ST_TRACE_BOUNDS __launch_bounds__(128, ST_TRACE_MIN_BLOCKS)
template <bool CNT, int MINB>
__global__ void __launch_bounds__(128, MINB) trace_kernel(SceneDev S, ViewDev v, const int4 *ssb, const float *dirs,
                                                          FloatPixel *out, u32t *prim_ids, unsigned *status,
                                                          unsigned long long *counters, u32t bx_first) {
    const u32t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // A block covers 8x16 grid points: four 8x4 warp tiles stacked vertically.  Blocks are numbered
    // down the columns, starting at block column bx_first: blocks start in launch order, so this
    // decides which part of the frame is in flight at once (down the columns measured 3 % faster on
    // the 1080p mesh frame than along the rows).
    const u32t x = (blockIdx.y + bx_first) * 8 + (lane & 7);
    const u32t y = blockIdx.x * 16 + warp * 4 + (lane >> 3);
    TState<CNT, 0> t;
    t.status = 0;
    if (CNT) for (int k = 0; k < C_COUNT; k++) t.cnt[k] = 0;
    if (x < v.grid_w && y < v.grid_h) trace_point(t, S, v, ssb, dirs, x, y, out, prim_ids);
    flush_counters(t, status, counters);
}

// ---- picking: manipulateSelection viewport/manipulation.h:55-123 ---------------------------------
// One thread: the ray of setRayFromCoords (shaders/common.h:170) through pixel (x, y), hitPrimitives
// over the TLAS leaf list with the visibility cull at (x, y), then every light's glow sphere
// (radius intensity/128, hitSphereSimple sphere.h:44); out: found, type, id, position, distance,
// camera-space z.
__global__ void pick_kernel(SceneDev S, ViewDev v, const int4 *ssb, int x, int y, PickDev *out) {
    if (threadIdx.x || blockIdx.x) return;
    TState<false> t;
    t.status = 0;
    t.closest.distance = t.closest.distance_squared = INFINITY;       // MAX_DISTANCE base.h:164
    t.closest.cone_width = 0;
    t.best.distance = t.best.distance_squared = INFINITY;
    RayD ray;
    ray.origin = v.cam_pos;
    ray.direction = norm(vsfma(v.pp_down, (float)y, vsfma(v.pp_right, (float)x, v.pp_start)));
    ray.rcp = rcp(ray.direction);
    bool found = hit_primitives(t, S, ray, S.tlas_leaf_ids, 0, S.n_prims, false, ssb, (int)(uint16_t)x,
                                (int)(uint16_t)y);
    if (found) finalize_hit(t, S, ray, 0.0f);
    Hit &hit = t.closest;
    for (u32t i = 0; S.lights && i < S.n_lights; i++) {
        const Light &L = S.lights[i];
        const float radius = L.intensity * (1.0f / (8.0f * 16.0f));
        t.sphere.furthest = hit.distance / radius;
        if (hit_sphere_simple(ray.origin, ray.direction, from(L.position_or_direction), 1.0f / radius, t.sphere)) {
            hit.distance = t.sphere.t_near * radius;
            hit.position = vsfma(ray.direction, hit.distance, ray.origin);
            hit.object_type = PrimitiveType_Light;
            hit.object_id = i;
            found = true;
        }
    }
    PickDev r;
    r.found = found;
    r.object_type = found ? hit.object_type : 0;
    r.object_id = found ? hit.object_id : 0;
    r.position[0] = found ? hit.position.x : 0;
    r.position[1] = found ? hit.position.y : 0;
    r.position[2] = found ? hit.position.z : 0;
    r.distance = found ? hit.distance : 0;
    r.object_distance = found ? vmat3(hit.position - ray.origin, v.cam_rot_matrix_inv).z : 0;
    *out = r;
}

// ---- batched views: one persistent launch over the tiles of many views ------------------------
// Every view is cut into tiles of tile_w x tile_h grid points (one warp per tile), and the tiles
// into groups of four that cover about 8x16 grid points (the per-frame kernel's block), numbered
// down the view's columns of groups.  A block takes `chunk` groups at a time from one global
// counter, its four warps one tile of each, so a block traces one compact region as the
// per-frame kernel's blocks do, views of different sizes, scenes and bounce counts share the
// launch, and no block idles while work is left.  (Measured on 64 views: warps taking tiles on
// their own 45.4 ms, groups numbered along the rows 43.0 ms.)
template <bool CNT, int TW, int TH, int SHS>
__global__ void ST_TRACE_BOUNDS batch_kernel(const BatchView *views, u32t n_views, u32t total_tiles, u32t chunk,
                                                    u32t *tile_counter, unsigned *status, unsigned long long *counters,
                                                    ParkQueue park) {
    static_assert(TW * TH == 32, "one warp per tile");
    constexpr u32t GW = group_tiles_w(TW), GH = 4 / GW;
    const u32t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ u32t stack_columns[SHS > 0 ? 2 * SHS * kTraceBlock : 1];
    __shared__ u32t block_first;
    TState<CNT, SHS> t;
    t.sh = stack_columns + threadIdx.x;
    t.status = 0;
    if (CNT) for (int k = 0; k < C_COUNT; k++) t.cnt[k] = 0;
    u32t vi = 0;       // a block's groups come in increasing order, so its view index only grows
    for (;;) {
        if (threadIdx.x == 0) block_first = atomicAdd(tile_counter, 4 * chunk);
        __syncthreads();
        const u32t first = block_first;
        __syncthreads();
        if (first >= total_tiles) break;
        const u32t last = min(first + 4 * chunk, total_tiles);
        for (u32t tile = first + warp; tile < last; tile += 4) {
            while (vi + 1 < n_views && views[vi + 1].tile_begin <= tile) vi++;
            const BatchView &B = views[vi];
            const u32t local = tile - B.tile_begin;
            const u32t group = local >> 2, q = local & 3;
            const u32t tx = (group / B.groups_y) * GW + q % GW, ty = (group % B.groups_y) * GH + q / GW;
            const u32t x = tx * TW + (lane % TW), y = ty * TH + (lane / TW);
            if (x < B.view.grid_w && y < B.view.grid_h)
                trace_point(t, B.scene, B.view, B.ssb, B.dirs, x, y, B.out, B.prim_ids, &park, vi);
        }
    }
    flush_counters(t, status, counters);
}

// The paths batch_kernel parked, continued from their bounce rays to the end and written to their
// views' outputs: a persistent grid whose warps take 32 queue slots at a time.
template <bool CNT, int SHS>
__global__ void ST_TRACE_BOUNDS drain_kernel(const BatchView *views, ParkQueue park, unsigned *status,
                                                    unsigned long long *counters) {
    const u32t lane = threadIdx.x & 31;
    __shared__ u32t stack_columns[SHS > 0 ? 2 * SHS * kTraceBlock : 1];
    TState<CNT, SHS> t;
    t.sh = stack_columns + threadIdx.x;
    t.status = 0;
    if (CNT) for (int k = 0; k < C_COUNT; k++) t.cnt[k] = 0;
    const u32t n = min(*park.reserved, park.capacity);
    u32t drained = 0;
    for (;;) {
        u32t first = 0;
        if (lane == 0) first = atomicAdd(park.taken, 32u);
        first = __shfl_sync(0xFFFFFFFFu, first, 0);
        if (first >= n) break;
        const u32t i = first + lane;
        if (i < n) {
            const ParkedRay P = park.rays[i];
            if (P.where.z != kEmptySlot) {
                const BatchView &B = views[P.where.z];
                trace_point(t, B.scene, B.view, B.ssb, B.dirs, P.where.x, P.where.y, B.out, nullptr, nullptr, 0, &P);
                drained++;
            }
        }
    }
    for (int off = 16; off; off >>= 1) drained += __shfl_down_sync(0xFFFFFFFFu, drained, off);
    if (lane == 0 && drained) atomicAdd(park.drained, drained);
    flush_counters(t, status, counters);
}

// drawViewportToWindowContent viewport/viewport.h:12 (QCAA branch): the 2x2 corners' colour times
// opacity, averaged, square-rooted in double, truncated to u8; all-infinite corners -> background.
__device__ __forceinline__ void resolve_one(const FloatPixel *in, u32t grid_w, u32t width, uint32_t *out, u32t x, u32t y) {
    const FloatPixel TL = in[(size_t)y * grid_w + x], TR = in[(size_t)y * grid_w + x + 1];
    const FloatPixel BL = in[(size_t)(y + 1) * grid_w + x], BR = in[(size_t)(y + 1) * grid_w + x + 1];
    uint32_t px;
    if (BL.depth == INFINITY && BR.depth == INFINITY && TL.depth == INFINITY && TR.depth == INFINITY) {
        px = 0xFF000000u;
    } else {
        v3 c = vscale(vsfma(from(TL.color), TL.opacity, vsfma(from(TR.color), TR.opacity,
                      vsfma(from(BL.color), BL.opacity, vscale(from(BR.color), BR.opacity)))), 0.25f);
        unsigned R = (unsigned char)(c.x > (255 * 255) ? 255.0 : sqrt((double)c.x));
        unsigned G = (unsigned char)(c.y > (255 * 255) ? 255.0 : sqrt((double)c.y));
        unsigned B = (unsigned char)(c.z > (255 * 255) ? 255.0 : sqrt((double)c.z));
        px = B | (G << 8) | (R << 16) | 0xFF000000u;
    }
    out[(size_t)y * width + x] = px;
}
// Pixel columns [x0, x1) of the frame (pixel x reads grid columns x and x + 1), one thread per
// pixel along the rows of the range, so that a narrow range leaves no block mostly idle.
__global__ void resolve_kernel(const FloatPixel *in, u32t grid_w, u32t width, u32t height, uint32_t *out, u32t x0,
                               u32t x1) {
    const u32t n = x1 - x0;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const u32t y = (u32t)(i / n), x = x0 + (u32t)(i % n);
    if (y < height) resolve_one(in, grid_w, width, out, x, y);
}

// ---- a batch's per-view set-up and resolve, driven by the view table (one launch each) ----------
__global__ void batch_ssb_kernel(const BatchTable T, u32t n_views) {
    const u32t vi = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (vi >= n_views) return;
    const BatchView &B = T.v[vi];
    if (i < B.scene.n_prims) ssb_one(B.scene, B.view, const_cast<int4 *>(B.ssb), i);
}
__global__ void batch_rows_kernel(const BatchTable T, u32t n_views) {
    const u32t vi = blockIdx.y, row = blockIdx.x * blockDim.x + threadIdx.x;
    if (vi >= n_views) return;
    const BatchView &B = T.v[vi];
    if (row < B.view.grid_h) row_segments_one(B.view, const_cast<float *>(B.dirs), row);
}
__global__ void batch_resolve_kernel(const BatchTable T, u32t n_views) {
    const u32t vi = blockIdx.z, x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (vi >= n_views) return;
    const BatchView &B = T.v[vi];
    if (B.out_u8 && x + 1 < B.view.grid_w && y + 1 < B.view.grid_h)
        resolve_one(B.out, B.view.grid_w, B.view.grid_w - 1, B.out_u8, x, y);
}

// ---- launchers -------------------------------------------------------------------------------
void launch_ssb(const SceneDev &S, const ViewDev &v, int4 *ssb, cudaStream_t st) {
    if (!S.n_prims) return;
    ssb_kernel<<<(S.n_prims + 127) / 128, 128, 0, st>>>(S, v, ssb);
}
void launch_ray_rows(const ViewDev &v, float *dirs, cudaStream_t st) {
    row_segments_kernel<<<(v.grid_h + 63) / 64, 64, 0, st>>>(v, dirs);
}
void launch_trace(const SceneDev &S, const ViewDev &v, const int4 *ssb, const float *dirs, FloatPixel *out,
                  u32t *prim_ids, unsigned *status, unsigned long long *counters, bool count, cudaStream_t st,
                  u32t bx_first, u32t bx_count, bool overlapped) {
    const u32t bw = (v.grid_w + 7) / 8, bh = (v.grid_h + 15) / 16;
    if (bx_first >= bw) return;
    if (!bx_count || bx_first + bx_count > bw) bx_count = bw - bx_first;
    const dim3 grid(bh, bx_count);
    constexpr int A = ST_TRACE_DEVICE_MIN_BLOCKS, B = ST_TRACE_OVERLAP_MIN_BLOCKS;
    if (count && overlapped)
        trace_kernel<true, B><<<grid, 128, 0, st>>>(S, v, ssb, dirs, out, prim_ids, status, counters, bx_first);
    else if (count)
        trace_kernel<true, A><<<grid, 128, 0, st>>>(S, v, ssb, dirs, out, prim_ids, status, counters, bx_first);
    else if (overlapped)
        trace_kernel<false, B><<<grid, 128, 0, st>>>(S, v, ssb, dirs, out, prim_ids, status, counters, bx_first);
    else
        trace_kernel<false, A><<<grid, 128, 0, st>>>(S, v, ssb, dirs, out, prim_ids, status, counters, bx_first);
}
int launch_batch(const BatchView *views, u32t n_views, u32t total_tiles, int variant, u32t chunk, u32t grid_blocks,
                 u32t *tile_counter, unsigned *status, unsigned long long *counters, bool count, cudaStream_t st,
                 const ParkQueue &park) {
#define ST_BATCH(TW, TH, SHS) (count ? (batch_kernel<true, TW, TH, SHS><<<grid_blocks, 128, 0, st>>>(views, n_views, total_tiles, chunk, tile_counter, status, counters, park), 0) \
                                     : (batch_kernel<false, TW, TH, SHS><<<grid_blocks, 128, 0, st>>>(views, n_views, total_tiles, chunk, tile_counter, status, counters, park), 0))
#define ST_BATCH_STACKS(TW, TH) (variant_stack(variant) ? ST_BATCH(TW, TH, kSharedStackEntries) : ST_BATCH(TW, TH, 0))
    if (variant < 0 || variant >= BATCH_VARIANTS) return -1;
    switch (variant_tile(variant)) {
        case TILE_8x4: return ST_BATCH_STACKS(8, 4);
        case TILE_16x2: return ST_BATCH_STACKS(16, 2);
        case TILE_32x1: return ST_BATCH_STACKS(32, 1);
        case TILE_4x8: return ST_BATCH_STACKS(4, 8);
    }
#undef ST_BATCH_STACKS
#undef ST_BATCH
    return -1;
}
int launch_drain(const BatchView *views, const ParkQueue &park, int variant, u32t grid_blocks, unsigned *status,
                 unsigned long long *counters, bool count, cudaStream_t st) {
    if (variant < 0 || variant >= BATCH_VARIANTS) return -1;
    const bool shared_stacks = variant_stack(variant) != 0;
    if (count) {
        if (shared_stacks) drain_kernel<true, kSharedStackEntries><<<grid_blocks, 128, 0, st>>>(views, park, status, counters);
        else drain_kernel<true, 0><<<grid_blocks, 128, 0, st>>>(views, park, status, counters);
    } else {
        if (shared_stacks) drain_kernel<false, kSharedStackEntries><<<grid_blocks, 128, 0, st>>>(views, park, status, counters);
        else drain_kernel<false, 0><<<grid_blocks, 128, 0, st>>>(views, park, status, counters);
    }
    return 0;
}
int batch_blocks_per_sm(int variant) {
    int n = 0;
#define ST_OCC(TW, TH) (variant_stack(variant) \
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<false, TW, TH, kSharedStackEntries>, 128, 0) \
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<false, TW, TH, 0>, 128, 0))
    switch (variant_tile(variant)) {
        case TILE_16x2: ST_OCC(16, 2); break;
        case TILE_32x1: ST_OCC(32, 1); break;
        case TILE_4x8: ST_OCC(4, 8); break;
        default: ST_OCC(8, 4); break;
    }
#undef ST_OCC
    return n > 0 ? n : 1;
}
void tile_dims(int variant, u32t &tw, u32t &th) {
    switch (variant_tile(variant)) {
        case TILE_16x2: tw = 16; th = 2; return;
        case TILE_32x1: tw = 32; th = 1; return;
        case TILE_4x8: tw = 4; th = 8; return;
        default: tw = 8; th = 4; return;
    }
}
void launch_pick(const SceneDev &S, const ViewDev &v, const int4 *ssb, int x, int y, PickDev *out, cudaStream_t st) {
    pick_kernel<<<1, 32, 0, st>>>(S, v, ssb, x, y, out);
}
void launch_batch_setup(const BatchTable &T, u32t n_views, u32t max_prims, u32t max_rows, cudaStream_t st) {
    if (max_prims) batch_ssb_kernel<<<dim3((max_prims + 127) / 128, n_views), 128, 0, st>>>(T, n_views);
    batch_rows_kernel<<<dim3((max_rows + 63) / 64, n_views), 64, 0, st>>>(T, n_views);
}
void launch_batch_resolve(const BatchTable &T, u32t n_views, u32t max_width, u32t max_height, cudaStream_t st) {
    batch_resolve_kernel<<<dim3((max_width + 127) / 128, max_height, n_views), 128, 0, st>>>(T, n_views);
}
void launch_resolve(const FloatPixel *in, u32t grid_w, u32t width, u32t height, uint32_t *out, cudaStream_t st,
                    u32t x0, u32t x1) {
    if (x1 > width) x1 = width;
    if (x0 >= x1 || !height) return;
    const size_t pixels = (size_t)(x1 - x0) * height;
    resolve_kernel<<<(unsigned)((pixels + 255) / 256), 256, 0, st>>>(in, grid_w, width, height, out, x0, x1);
}

}  // namespace st
