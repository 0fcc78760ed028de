// st_overlay.cu — the debug overlays drawBVH (render/raytracer.h:46) and drawSSB (render/SSB.h:175)
// drawn on the device into the traced float grid, before the QCAA resolve.
//
// The reference draws box edges one after another with an anti-aliased line rasteriser
// (shapes/line.h:46) that blends every pixel it touches into the frame (setPixel, core/types.h:422);
// blending is order-dependent, so the device keeps the reference's drawing order exactly:
//
//   boxes      one per TLAS node, per implicit primitive of a leaf, per outlined BLAS node of a
//              leaf's mesh instance (nodes of depth <= 5, drawMeshAccelerationStructure
//              raytracer.h:33), numbered in the reference's visiting order through a scan of
//              per-node box counts;
//   edges      12 per box in BoxEdgeSides order, then 4 screen-space lines per primitive (drawSSB);
//              one thread per edge clips and projects it (cullAndClipEdge/projectEdge, edge.h:8,83)
//              and walks the rasteriser's columns twice: once to count the pixels it plots, once to
//              write them as fragments at the scanned offsets, so the fragment index is the
//              reference's global plotting order;
//   blend      fragments are radix-sorted by pixel (stable, so each pixel's fragments stay in
//              plotting order) and one thread per pixel applies setPixel in that order.
//
// The rasteriser's per-column values are kept as the reference computes them: the column offset is
// accumulated by repeated addition (gap += grad), 1/z by repeated f64 addition, and float -> int
// casts follow x86's truncating convert (NaN and out-of-range values give INT_MIN).
#include <algorithm>
#include <climits>
#include "st_kernels.h"

namespace st {

namespace {

// The unit box of initBox (core/init.h:279) in BoxCorners order (core/types.h:86), and the edges of
// setBoxEdgesFromVertices (core/init.h:250) in BoxEdgeSides order (core/types.h:102).
__constant__ float kCorner[8][3] = {{-1, 1, 1}, {1, 1, 1}, {-1, -1, 1}, {1, -1, 1},
                                    {-1, 1, -1}, {1, 1, -1}, {-1, -1, -1}, {1, -1, -1}};
__constant__ unsigned char kEdge[12][2] = {{0, 1}, {2, 3}, {2, 0}, {3, 1}, {4, 5}, {6, 7},
                                           {6, 4}, {7, 5}, {2, 6}, {0, 4}, {3, 7}, {1, 5}};

// Color() (core/base.h:577) of the overlay colours, squared as drawLine/drawHLine square them
// (mulVec3(color, color), line.h:16,62): index 1 White, 2 Grey, 3 Red, 4 Green, 5 Blue, 6 Cyan,
// 7 Magenta, 8 Yellow.
__device__ __forceinline__ v3 overlay_color_sq(u32t id) {
    const float M = 255.0f, H = 255.0f / 2.0f;
    v3 c = V(0, 0, 0);
    switch (id) {
        case 1: c = V(M, M, M); break;
        case 2: c = V(H, H, H); break;
        case 3: c = V(M, 0, 0); break;
        case 4: c = V(0, M, 0); break;
        case 5: c = V(0, 0, M); break;
        case 6: c = V(0, M, M); break;
        case 7: c = V(M, 0, M); break;
        case 8: c = V(M, M, 0); break;
    }
    return vmul(c, c);
}

__device__ __forceinline__ u32t type_color(unsigned type) {
    switch (type) {
        case PrimitiveType_Box: return 6;
        case PrimitiveType_Quad: return 1;
        case PrimitiveType_Sphere: return 8;
        case PrimitiveType_Tetrahedron: return 7;
        default: return 0;
    }
}

struct BoxRec {
    v3 v[8];          // corners in view space
    u32t color;       // overlay colour id
    float opacity;
    u32t line_width;
    u32t pad;
};

struct Frag {
    double depth;
    float opacity;
    u32t color;
};

__device__ __forceinline__ int trunc_i32(float v) { return (v >= -2147483648.0f && v < 2147483648.0f) ? (int)v : INT_MIN; }
__device__ __forceinline__ float frac_of(float v) { return v - floorf(v); }
__device__ __forceinline__ float one_minus_frac_of(float v) { return 1 - frac_of(v); }
__device__ __forceinline__ bool in_range(int v, int end, int start) { return v >= start && v < end; }

// convertPositionToWorldSpace (scene/primitive.h:35) of a box primitive given as its fields
__device__ __forceinline__ v3 to_world(v3 p, unsigned flags, v3 pos, q4 rot, v3 scale) {
    if (flags & IS_SCALED) p = vmul(p, scale);
    if (flags & IS_ROTATED) p = qrot(p, rot);
    if (flags & IS_TRANSLATED) p = p + pos;
    return p;
}

// Boxes per TLAS node in drawBVH's order: the node itself, its leaf primitives' boxes, and the
// outlined BLAS nodes of its mesh instances.
__global__ void box_count_kernel(OverlayParams P, u32t *counts) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.node_count) return;
    const BVHNode n = P.nodes[i];
    u32t c = 1;
    for (u32t j = 0; j < n.child_count; j++) {
        const Primitive &p = P.prims[P.leaf_ids[n.first_child_id + j]];
        if (p.type == PrimitiveType_Mesh) c += p.id < P.n_meshes ? P.outline_range[p.id].y : 0;
        else if (type_color(p.type)) c += 1;
    }
    counts[i] = c;
}

// setBoxPrimitiveFromAABB (raytracer.h:18)
__device__ __forceinline__ void box_from_aabb(const float *a, unsigned &flags, v3 &pos, q4 &rot, v3 &scale) {
    const v3 mn = V(a[0], a[1], a[2]), mx = V(a[3], a[4], a[5]);
    rot.axis = V(0, 0, 0);
    rot.w = 1;
    pos = vscale(mn + mx, 0.5f);
    scale = vscale(mx - mn, 0.5f);
    flags = IS_TRANSLATED | IS_SCALED | IS_SCALED_NON_UNIFORMLY;
}

// One box: find its TLAS node by binary search over the scanned counts, then which of the node's
// boxes it is; write its corners in view space (transformBoxVerticesFromObjectToViewSpace, box.h:9).
__global__ void box_kernel(OverlayParams P, const u32t *offsets, const u32t *total, BoxRec *boxes, u32t n_boxes) {
    const u32t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_boxes) return;
    BoxRec r;
    r.color = 0;
    r.opacity = 1;
    r.line_width = 1;
    r.pad = 0;
    unsigned flags = 0;
    v3 pos = V(0, 0, 0), scale = V(1, 1, 1);
    q4 rot;
    rot.axis = V(0, 0, 0);
    rot.w = 1;
    bool valid = b < *total;
    if (valid) {
        u32t lo = 0, hi = P.node_count - 1;    // last node with offsets[node] <= b
        while (lo < hi) {
            const u32t mid = (lo + hi + 1) >> 1;
            if (offsets[mid] <= b) lo = mid; else hi = mid - 1;
        }
        const BVHNode n = P.nodes[lo];
        u32t k = b - offsets[lo];
        bool done = false;
        for (u32t j = 0; j < n.child_count && !done; j++) {
            const Primitive &p = P.prims[P.leaf_ids[n.first_child_id + j]];
            if (p.type == PrimitiveType_Mesh) {
                const uint2 rg = p.id < P.n_meshes ? P.outline_range[p.id] : make_uint2(0, 0);
                if (k < rg.y) {
                    // setBoxPrimitiveFromPrimitiveAndAABB (raytracer.h:25)
                    const OutlineBox &o = P.outlines[rg.x + k];
                    box_from_aabb(o.aabb, flags, pos, rot, scale);
                    scale = vmul(scale, from(p.scale));
                    rot.axis = from(p.rotation.axis);
                    rot.w = p.rotation.amount;
                    flags |= IS_ROTATED;
                    q4 prot;
                    prot.axis = from(p.rotation.axis);
                    prot.w = p.rotation.amount;
                    pos = to_world(pos, p.flags, from(p.position), prot, from(p.scale));
                    r.color = o.color;
                    r.opacity = 0.125f;
                    r.line_width = 0;
                    done = true;
                } else k -= rg.y;
            } else if (type_color(p.type)) {
                if (k == 0) {
                    flags = p.flags;
                    pos = from(p.position);
                    rot.axis = from(p.rotation.axis);
                    rot.w = p.rotation.amount;
                    scale = from(p.scale);
                    r.color = type_color(p.type);
                    done = true;
                } else k -= 1;
            }
        }
        if (!done) {
            box_from_aabb(&n.aabb.min.x, flags, pos, rot, scale);
            r.color = n.child_count ? 1u : (lo ? 2u : 5u);
        }
    }
    for (int c = 0; c < 8; c++) {
        const v3 w = to_world(V(kCorner[c][0], kCorner[c][1], kCorner[c][2]), flags, pos, rot, scale);
        r.v[c] = qrot(w - P.cam_pos, P.cam_rot_inv);
    }
    if (!valid) r.color = 0;   // a box past the device total draws nothing
    boxes[b] = r;
}

// lerpVec3 (vec3.h:265)
__device__ __forceinline__ v3 lerp3(v3 from, v3 to, float by) { return vsfma(to - from, by, from); }

// cullAndClipEdge (edge.h:8)
__device__ bool clip_edge(v3 &pa, v3 &pb, const OverlayParams &P) {
    v3 A = pa, B = pb, N = V(0, 0, 0);
    float d = P.near_plane;
    unsigned out = (A.z < d) | ((B.z < d) << 1);
    if (out) {
        if (out == 3) return false;
        if (out & 1) A = lerp3(A, B, (d - A.z) / (B.z - A.z));
        else         B = lerp3(B, A, (d - B.z) / (A.z - B.z));
    }
    d = P.far_plane;
    out = (A.z > d) | ((B.z > d) << 1);
    if (out) {
        if (out == 3) return false;
        if (out & 1) A = lerp3(A, B, (A.z - d) / (A.z - B.z));
        else         B = lerp3(B, A, (B.z - d) / (B.z - A.z));
    }
    for (int plane = 0; plane < 4; plane++) {
        if (plane == 0) N = V(P.focal_length, 0, P.width_over_height);   // left
        else if (plane == 1) N.x = -N.x;                                   // right
        else if (plane == 2) N = V(0, P.focal_length, 1);                  // bottom
        else N.y = -N.y;                                                   // top
        const float na = dot(N, A), nb = dot(N, B);
        out = (na < 0) | ((nb < 0) << 1);
        if (out) {
            if (out == 3) return false;
            if (out & 1) A = lerp3(A, B, na / (na - nb));
            else         B = lerp3(B, A, nb / (nb - na));
        }
    }
    pa = A;
    pb = B;
    return true;
}

// mulVec4Mat4 (vec4.h:96) of (p, 1), then the perspective divide (projectEdge, edge.h:90-95)
__device__ __forceinline__ v3 project_point(v3 p, const float *m) {
    const float x = p.x * m[0] + p.y * m[4] + p.z * m[8] + 1.0f * m[12];
    const float y = p.x * m[1] + p.y * m[5] + p.z * m[9] + 1.0f * m[13];
    const float z = p.x * m[2] + p.y * m[6] + p.z * m[10] + 1.0f * m[14];
    const float w = p.x * m[3] + p.y * m[7] + p.z * m[11] + 1.0f * m[15];
    return vscale(V(x, y, z), 1.0f / w);
}

// Where a line's pixels go: counted, or written as fragments in plotting order.
struct CountSink {
    u32t n = 0;
    __device__ void set_color(u32t) {}
    __device__ void plot(int, int, double, float) { n++; }
};
struct EmitSink {
    const OverlayParams *P;
    u32t *keys, *vals;
    Frag *frags;
    u32t pos, end, color;
    __device__ void set_color(u32t c) { color = c; }
    __device__ void plot(int x, int y, double z, float opacity) {
        if (pos >= end) return;   // never more than the counting walk found
        // setPixelByCoords (core/types.h:453): pixels + stride * y + x; a pixel outside the grid (a
        // viewport position that is not 0) gets the key grid_pixels and is not blended, instead of
        // being written past the buffer
        const long long idx = (long long)P->stride * y + x;
        keys[pos] = (idx >= 0 && idx < (long long)P->grid_pixels) ? (u32t)idx : P->grid_pixels;
        vals[pos] = pos;
        Frag f;
        f.depth = z;
        f.opacity = opacity;
        f.color = color;
        frags[pos] = f;
        pos++;
    }
};

// Longest run of columns or rows a line may walk.  Edges clipped to the view frustum project inside
// the frame, so real lines stay far below it; a line whose endpoints are not finite (a near plane
// at or behind the camera) or whose run exceeds it is not drawn (the reference would walk up to
// 2^32 columns).
constexpr long long kMaxRun = 1 << 20;

// drawLine (shapes/line.h:46)
template <class Sink>
__device__ void draw_line(const OverlayParams &P, float x1, float y1, double z1, float x2, float y2, double z2,
                          float opacity, u32t line_width, Sink &sink) {
    if (x1 < 0 && y1 < 0 && x2 < 0 && y2 < 0) return;
    if (!isfinite(x1) || !isfinite(y1) || !isfinite(x2) || !isfinite(y2)) return;
    const int x_left = P.pos_x, y_top = P.pos_y, w = P.width + x_left, h = P.height + y_top;
    x1 += (float)x_left; x2 += (float)x_left;
    y1 += (float)y_top;  y2 += (float)y_top;
    double tmp, z_range, range_remap, z = 0, z_curr = 0, z_step = 0;
    const float dx = x2 - x1, dy = y2 - y1;
    float gap, grad, first_offset, last_offset, fx, fy, lx, ly;
    int x, y, sx, sy, ex, ey;
    const bool has_depth = z1 || z2;
    if (fabsf(dx) > fabsf(dy)) {
        if (x2 < x1) { tmp = x2; x2 = x1; x1 = (float)tmp; tmp = y2; y2 = y1; y1 = (float)tmp; tmp = z2; z2 = z1; z1 = tmp; }
        grad = dy / dx;
        fx = roundf(x1); lx = roundf(x2);
        first_offset = fx - x1; last_offset = lx - x2;
        fy = y1 + grad * first_offset; ly = y2 + grad * last_offset;
        sx = trunc_i32(fx); sy = trunc_i32(fy); ex = trunc_i32(lx); ey = trunc_i32(ly);
        if ((long long)ex - sx > kMaxRun) return;
        x = sx; y = sy;
        gap = one_minus_frac_of(x1 + 0.5f);
        if (in_range(x, w, x_left)) {
            if (in_range(y, h, y_top)) sink.plot(x, y, z1, one_minus_frac_of(fy) * gap * opacity);
            for (u32t i = 0; i < line_width; i++) { y++; if (in_range(y, h, y_top)) sink.plot(x, y, z1, opacity); }
            y++;
            if (in_range(y, h, y_top)) sink.plot(x, y, z1, frac_of(fy) * gap * opacity);
        }
        x = ex; y = ey;
        gap = frac_of(x2 + 0.5f);
        if (in_range(x, w, x_left)) {
            if (in_range(y, h, y_top)) sink.plot(x, y, z2, one_minus_frac_of(ly) * gap * opacity);
            for (u32t i = 0; i < line_width; i++) { y++; if (in_range(y, h, y_top)) sink.plot(x, y, z2, opacity); }
            y++;
            if (in_range(y, h, y_top)) sink.plot(x, y, z2, frac_of(ly) * gap * opacity);
        }
        if (has_depth) {
            z1 = 1.0 / z1; z2 = 1.0 / z2;
            z_range = z2 - z1;
            range_remap = z_range / (double)(x2 - x1);
            z1 += range_remap * (double)(first_offset + 1);
            z2 += range_remap * (double)(last_offset - 1);
            z_range = z2 - z1;
            z_step = z_range / (double)(lx - fx - 1);
            z_curr = z1;
        } else z = 0;
        gap = fy + grad;
        for (x = sx + 1; x < ex; x++) {
            if (in_range(x, w, x_left)) {
                if (has_depth) z = 1.0 / z_curr;
                y = trunc_i32(gap);
                if (in_range(y, h, y_top)) sink.plot(x, y, z, one_minus_frac_of(gap) * opacity);
                for (u32t i = 0; i < line_width; i++) { y++; if (in_range(y, h, y_top)) sink.plot(x, y, z, opacity); }
                y++;
                if (in_range(y, h, y_top)) sink.plot(x, y, z, frac_of(gap) * opacity);
            }
            gap += grad;
            if (has_depth) z_curr += z_step;
        }
    } else {
        if (y2 < y1) { tmp = x2; x2 = x1; x1 = (float)tmp; tmp = y2; y2 = y1; y1 = (float)tmp; tmp = z2; z2 = z1; z1 = tmp; }
        grad = dx / dy;
        fy = roundf(y1); ly = roundf(y2);
        first_offset = y1 - fy; last_offset = ly - y2;
        fx = x1 + grad * first_offset; lx = x2 + grad * last_offset;
        sy = trunc_i32(fy); sx = trunc_i32(fx); ey = trunc_i32(ly); ex = trunc_i32(lx);
        if ((long long)ey - sy > kMaxRun) return;
        x = sx; y = sy;
        gap = one_minus_frac_of(y1 + 0.5f);
        if (in_range(y, h, y_top)) {
            if (in_range(x, w, x_left)) sink.plot(x, y, z1, one_minus_frac_of(fx) * gap * opacity);
            for (u32t i = 0; i < line_width; i++) { x++; if (in_range(x, w, x_left)) sink.plot(x, y, z1, opacity); }
            x++;
            if (in_range(x, w, x_left)) sink.plot(x, y, z1, frac_of(fx) * gap * opacity);
        }
        x = ex; y = ey;
        gap = frac_of(y2 + 0.5f);
        if (in_range(y, h, y_top)) {
            if (in_range(x, w, x_left)) sink.plot(x, y, z2, one_minus_frac_of(lx) * gap * opacity);
            for (u32t i = 0; i < line_width; i++) { x++; if (in_range(x, w, x_left)) sink.plot(x, y, z2, opacity); }
            x++;
            if (in_range(x, w, x_left)) sink.plot(x, y, z2, frac_of(lx) * gap * opacity);
        }
        if (has_depth) {
            z1 = 1.0 / z1; z2 = 1.0 / z2;
            z_range = z2 - z1;
            range_remap = z_range / (double)(y2 - y1);
            z1 += range_remap * (double)(first_offset + 1);
            z2 += range_remap * (double)(last_offset - 1);
            z_range = z2 - z1;
            z_step = z_range / (double)(ly - fy - 1);
            z_curr = z1;
        } else z = 0;
        gap = fx + grad;
        for (y = sy + 1; y < ey; y++) {
            if (in_range(y, h, y_top)) {
                if (has_depth) z = 1.0 / z_curr;
                x = trunc_i32(gap);
                if (in_range(x, w, x_left)) sink.plot(x, y, z, one_minus_frac_of(gap) * opacity);
                for (u32t i = 0; i < line_width; i++) { x++; if (in_range(x, w, x_left)) sink.plot(x, y, z, opacity); }
                x++;
                if (in_range(x, w, x_left)) sink.plot(x, y, z, frac_of(gap) * opacity);
            }
            gap += grad;
            if (has_depth) z_curr += z_step;
        }
    }
}

// drawHLine / drawVLine (shapes/line.h:5,22) with subRange (core/base.h:373): one screen-space line
// of drawSSB, k = 0/1 the rows min.y/max.y, k = 2/3 the columns min.x/max.x.
template <class Sink>
__device__ void draw_ssb_line(const OverlayParams &P, int4 b, int k, Sink &sink) {
    const bool horizontal = k < 2;
    int from = horizontal ? b.x : b.y, to = horizontal ? b.z : b.w;
    int at = k == 0 ? b.y : k == 1 ? b.w : k == 2 ? b.x : b.z;
    const int along0 = horizontal ? P.pos_x : P.pos_y, across0 = horizontal ? P.pos_y : P.pos_x;
    const int along_end = (horizontal ? (int)P.width : (int)P.height) + along0;
    const int across_end = (horizontal ? (int)P.height : (int)P.width) + across0;
    from += along0; to += along0; at += across0;
    if (!in_range(at, across_end, across0)) return;
    int first = from, last = to;
    if (to < from) { first = to; last = from; }
    first = first > along0 ? first : along0;
    last = (last < along_end ? last : along_end) - 1;
    for (int s = first; s <= last; s++) {
        if (horizontal) sink.plot(s, at, 0.0, 1.0f);
        else sink.plot(at, s, 0.0, 1.0f);
    }
}

// One edge (a box edge, or a drawSSB line after all box edges) through the given sink.
template <class Sink>
__device__ void walk_edge(const OverlayParams &P, const BoxRec *boxes, u32t n_boxes, const int4 *ssb, u32t e,
                          Sink &sink) {
    if (e < 12 * n_boxes) {
        const BoxRec &r = boxes[e / 12];
        if (!r.color) return;
        sink.set_color(r.color);
        v3 A = r.v[kEdge[e % 12][0]], B = r.v[kEdge[e % 12][1]];
        if (!clip_edge(A, B, P)) return;
        const float az = A.z, bz = B.z;
        v3 a = project_point(A, P.proj), c = project_point(B, P.proj);
        a.x += 1; a.x *= P.h_width;
        c.x += 1; c.x *= P.h_width;
        a.y += 1; a.y *= P.h_height;
        c.y += 1; c.y *= P.h_height;
        a.y = P.f_height - a.y;
        c.y = P.f_height - c.y;
        draw_line(P, a.x, a.y, (double)az, c.x, c.y, (double)bz, r.opacity, r.line_width, sink);
        return;
    }
    const u32t s = e - 12 * n_boxes, i = s >> 2;
    if (i >= P.n_prims) return;
    const int4 b = ssb[i];
    if (b.x == 1 && b.y == 1 && b.z == 0 && b.w == 0) return;    // not visible (ssb_kernel's empty rect)
    const Primitive &p = P.prims[i];
    const u32t color = p.type == PrimitiveType_Mesh ? 3u : type_color(p.type);
    if (!color) return;
    sink.set_color(color);
    draw_ssb_line(P, b, (int)(s & 3), sink);
}

__global__ void edge_count_kernel(OverlayParams P, const BoxRec *boxes, u32t n_boxes, const int4 *ssb, u32t n_edges,
                                  u32t *counts, unsigned long long *total64) {
    const u32t e = blockIdx.x * blockDim.x + threadIdx.x;
    CountSink sink;
    if (e < n_edges) {
        walk_edge(P, boxes, n_boxes, ssb, e, sink);
        counts[e] = sink.n;
    }
    // the exact total in 64 bits, so that the host can refuse a fragment count the 32-bit scan
    // cannot hold
    unsigned long long v = sink.n;
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(total64, v);
}

__global__ void edge_emit_kernel(OverlayParams P, const BoxRec *boxes, u32t n_boxes, const int4 *ssb, u32t n_edges,
                                 const u32t *offsets, const u32t *counts, u32t *keys, u32t *vals, Frag *frags) {
    const u32t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_edges) return;
    EmitSink sink;
    sink.P = &P;
    sink.keys = keys;
    sink.vals = vals;
    sink.frags = frags;
    sink.pos = offsets[e];
    sink.end = offsets[e] + counts[e];
    sink.color = 0;
    walk_edge(P, boxes, n_boxes, ssb, e, sink);
}

// setPixel (core/types.h:422)
__device__ __forceinline__ void set_pixel(FloatPixel &px, v3 color, float opacity, double depth) {
    FloatPixel np;
    np.opacity = opacity;
    np.color.x = color.x; np.color.y = color.y; np.color.z = color.z;
    np.depth = depth;
    if (!(opacity == 1 && depth == 0)) {
        FloatPixel bg, fg;
        const FloatPixel old = px;
        if (old.depth < np.depth) { bg = np; fg = old; } else { bg = old; fg = np; }
        if (fg.opacity != 1) {
            const float omf = 1.0f - fg.opacity;
            opacity = fg.opacity + bg.opacity * omf;
            const float oo = opacity ? 1.0f / opacity : 1;
            const float bf = bg.opacity * oo * omf;
            const float ff = fg.opacity * oo;
            px.color.x = fg.color.x * ff + bg.color.x * bf;
            px.color.y = fg.color.y * ff + bg.color.y * bf;
            px.color.z = fg.color.z * ff + bg.color.z * bf;
            px.opacity = opacity;
            px.depth = fg.depth;
        } else px = fg;
    } else px = np;
}

// One thread per run of equal pixel keys (sorted, so each run is in plotting order).
__global__ void blend_kernel(const u32t *keys, const u32t *vals, const Frag *frags, u32t n, u32t grid_pixels,
                             FloatPixel *grid, FloatPixel *grid_host) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32t key = keys[i];
    if (key >= grid_pixels || (i > 0 && keys[i - 1] == key)) return;
    FloatPixel px = grid[key];
    for (u32t j = i; j < n && keys[j] == key; j++) {
        const Frag f = frags[vals[j]];
        set_pixel(px, overlay_color_sq(f.color), f.opacity, f.depth);
    }
    grid[key] = px;
    if (grid_host) grid_host[key] = px;
}

}  // namespace

// Scratch layout shared by overlay_count and overlay_draw.
struct OverlayCarve {
    u32t *node_counts, *node_offsets, *sums, *totals, *edge_counts, *edge_offsets, *edge_sums;
    BoxRec *boxes;
    u32t n_boxes, n_edges;
};
static size_t carve(OverlayCarve &c, const OverlayParams &P, u32t n_boxes, void *base) {
    char *cur = static_cast<char *>(base);
    auto take = [&](size_t b) { char *p = cur; cur += (b + 255) / 256 * 256; return p; };
    c.n_boxes = n_boxes;
    c.n_edges = 12 * n_boxes + 4 * P.n_prims;
    const size_t nodes = std::max(P.node_count, 1u), edges = std::max(c.n_edges, 1u);
    c.node_counts = reinterpret_cast<u32t *>(take(4 * nodes));
    c.node_offsets = reinterpret_cast<u32t *>(take(4 * nodes));
    c.sums = reinterpret_cast<u32t *>(take(4 * (nodes / 1024 + 2)));
    c.totals = reinterpret_cast<u32t *>(take(32));   // node total, fragment total, 64-bit fragment total at +8
    c.boxes = reinterpret_cast<BoxRec *>(take(sizeof(BoxRec) * (size_t)std::max(n_boxes, 1u)));
    c.edge_counts = reinterpret_cast<u32t *>(take(4 * edges));
    c.edge_offsets = reinterpret_cast<u32t *>(take(4 * edges));
    c.edge_sums = reinterpret_cast<u32t *>(take(4 * (edges / 1024 + 2)));
    return (size_t)(cur - static_cast<char *>(base));
}

size_t overlay_scratch_bytes(const OverlayParams &P, u32t n_boxes) {
    OverlayCarve c;
    return carve(c, P, n_boxes, nullptr) + 256;
}

size_t overlay_fragment_bytes(u32t n_frags) {
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    return al(4 * (size_t)n_frags) * 4 + al(sizeof(Frag) * (size_t)n_frags) + al(radix_sort_scratch_bytes(n_frags)) + 256;
}

cudaError_t overlay_count(const OverlayParams &P, const int4 *ssb, u32t n_boxes, void *scratch, u32t *n_frags,
                          cudaStream_t st) {
    const u32t T = 256;
    OverlayCarve c;
    carve(c, P, n_boxes, scratch);
    *n_frags = 0;
    if (n_boxes) {
        box_count_kernel<<<(P.node_count + T - 1) / T, T, 0, st>>>(P, c.node_counts);
        scan_exclusive_u32(c.node_counts, c.node_offsets, P.node_count, c.sums, c.totals, st);
        box_kernel<<<(n_boxes + T - 1) / T, T, 0, st>>>(P, c.node_offsets, c.totals, c.boxes, n_boxes);
    }
    if (!c.n_edges) return cudaGetLastError();
    unsigned long long *total64 = reinterpret_cast<unsigned long long *>(c.totals + 2);
    cudaError_t e = cudaMemsetAsync(total64, 0, sizeof(*total64), st);
    if (e != cudaSuccess) return e;
    edge_count_kernel<<<(c.n_edges + T - 1) / T, T, 0, st>>>(P, c.boxes, n_boxes, ssb, c.n_edges, c.edge_counts, total64);
    scan_exclusive_u32(c.edge_counts, c.edge_offsets, c.n_edges, c.edge_sums, c.totals + 1, st);
    unsigned long long total = 0;
    e = cudaMemcpyAsync(&total, total64, sizeof(total), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (total > 0x7FFFFFFFull) return cudaErrorMemoryAllocation;   // more pixels than one pass can sort
    *n_frags = (u32t)total;
    return cudaSuccess;
}

cudaError_t overlay_draw(const OverlayParams &P, const int4 *ssb, u32t n_boxes, void *scratch, u32t n_frags,
                         void *frag_buf, FloatPixel *grid, FloatPixel *grid_host, cudaStream_t st) {
    const u32t T = 256;
    if (!n_frags) return cudaSuccess;
    OverlayCarve c;
    carve(c, P, n_boxes, scratch);
    char *cur = static_cast<char *>(frag_buf);
    auto take = [&](size_t b) { char *p = cur; cur += (b + 255) / 256 * 256; return p; };
    u32t *k0 = reinterpret_cast<u32t *>(take(4 * (size_t)n_frags));
    u32t *v0 = reinterpret_cast<u32t *>(take(4 * (size_t)n_frags));
    u32t *k1 = reinterpret_cast<u32t *>(take(4 * (size_t)n_frags));
    u32t *v1 = reinterpret_cast<u32t *>(take(4 * (size_t)n_frags));
    Frag *frags = reinterpret_cast<Frag *>(take(sizeof(Frag) * (size_t)n_frags));
    void *sort_scratch = take(radix_sort_scratch_bytes(n_frags));
    edge_emit_kernel<<<(c.n_edges + T - 1) / T, T, 0, st>>>(P, c.boxes, n_boxes, ssb, c.n_edges, c.edge_offsets,
                                                           c.edge_counts, k0, v0, frags);
    // keys are pixel indices, or grid_pixels for a pixel outside the grid: sort on the bytes that
    // grid_pixels spans
    int passes = 0;
    for (u32t top = P.grid_pixels; top; top >>= 8) passes++;
    const int in_alt = radix_sort_pairs(k0, v0, k1, v1, n_frags, passes, sort_scratch, st);
    blend_kernel<<<(n_frags + T - 1) / T, T, 0, st>>>(in_alt ? k1 : k0, in_alt ? v1 : v0, frags, n_frags, P.grid_pixels,
                                                      grid, grid_host);
    return cudaGetLastError();
}

}  // namespace st
