// st_bvh.cu — device BVH builds: the 30-bit Morton LBVH (TLAS and BLAS), refit, and the conversions
// into the traversal layouts.
//
// LBVH30 (no reference counterpart; builder_bottom_up.h is dead code):
//   boxes      TLAS: the 8-corner world box of each primitive's local box (AABB.h:44,
//              primitive.h:53); BLAS: each triangle's box with EPS padding on flat axes
//              (builder_top_down.h:283-318)
//   bounds     union of the item boxes under the IEEE total order (-0 < +0), so every union here
//              is independent of the order it is formed in
//   code       10 bits per axis of the box centre (min+max)*0.5, scaled by 1024/extent and clamped
//              to [0,1023]; x in the highest bit of each triple
//   sort       stable LSD radix sort of (code, index): 4 passes of 8 bits, one block per 2048-key
//              tile, ranks made stable with warp match + per-warp prefix counts
//   topology   Karras 2012 over the 64-bit keys code<<32 | index (all distinct)
//   collapse   internal nodes covering <= max_leaf items become leaves; kept nodes are ranked in
//              index order and kept node r's children occupy output slots 1+2r, 2+2r, which is the
//              reference's BVHNode layout (root 0, sibling pairs, builder_top_down.h:172-174)
#include <cstdio>
#include "st_kernels.h"

namespace st {

__device__ __forceinline__ unsigned ord_bits(float f) {
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ord(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// ---- item boxes ---------------------------------------------------------------------------------
__device__ __forceinline__ v3 prim_to_world(v3 pos, const Primitive &p) {   // convertPositionToWorldSpace primitive.h:30
    if (p.flags & IS_SCALED) pos = vmul(pos, from(p.scale));
    if (p.flags & IS_ROTATED) { q4 q; q.axis = from(p.rotation.axis); q.w = p.rotation.amount; pos = qrot(pos, q); }
    if (p.flags & IS_TRANSLATED) pos = pos + from(p.position);
    return pos;
}

__global__ void prim_aabbs_kernel(const Primitive *prims, const MeshDev *meshes, u32t n, float *aabbs) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Primitive p = prims[i];
    float lo[3], hi[3];
    if (p.type == PrimitiveType_Mesh) {
        const MeshDev &m = meshes[p.id];
        for (int a = 0; a < 3; a++) { lo[a] = m.mesh_aabb[a]; hi[a] = m.mesh_aabb[3 + a]; }
    } else {
        const float e = p.type == PrimitiveType_Tetrahedron ? (1.73205080757f / 3) : 1.0f;
        for (int a = 0; a < 3; a++) { lo[a] = -e; hi[a] = e; }
    }
    // transformAABB AABB.h:44: the 8 corners in the reference's order, strict comparisons
    float x = +INFINITY, y = +INFINITY, z = +INFINITY, X = -INFINITY, Y = -INFINITY, Z = -INFINITY;
#pragma unroll
    for (int c = 0; c < 8; c++) {
        v3 q = prim_to_world(V((c & 4) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 1) ? hi[2] : lo[2]), p);
        if (q.x > X) X = q.x;
        if (q.y > Y) Y = q.y;
        if (q.z > Z) Z = q.z;
        if (q.x < x) x = q.x;
        if (q.y < y) y = q.y;
        if (q.z < z) z = q.z;
    }
    float *o = aabbs + 6 * (size_t)i;
    o[0] = x; o[1] = y; o[2] = z; o[3] = X; o[4] = Y; o[5] = Z;
}

__global__ void tri_aabbs_kernel(const vec3 *pos, const uint32_t *idx, u32t n, float *aabbs) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const vec3 v1 = pos[idx[3 * i]], v2 = pos[idx[3 * i + 1]], v3_ = pos[idx[3 * i + 2]];
    float mn[3], mx[3];
    const float a1[3] = {v1.x, v1.y, v1.z}, a2[3] = {v2.x, v2.y, v2.z}, a3[3] = {v3_.x, v3_.y, v3_.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        mn[a] = a2[a] < a3[a] ? a2[a] : a3[a];
        mx[a] = a2[a] > a3[a] ? a2[a] : a3[a];
        mn[a] = mn[a] < a1[a] ? mn[a] : a1[a];
        mx[a] = mx[a] > a1[a] ? mx[a] : a1[a];
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float d = mx[a] - mn[a];
        if (d < 0) d = -d;
        if (d < 0.0001f) { mn[a] -= 0.0001f; mx[a] += 0.0001f; }
    }
    float *o = aabbs + 6 * (size_t)i;
    o[0] = mn[0]; o[1] = mn[1]; o[2] = mn[2]; o[3] = mx[0]; o[4] = mx[1]; o[5] = mx[2];
}

// ---- Morton codes ------------------------------------------------------------------------------
__global__ void bounds_init_kernel(unsigned *b) {
    if (threadIdx.x < 3) b[threadIdx.x] = 0xFFFFFFFFu;
    else if (threadIdx.x < 6) b[threadIdx.x] = 0u;
}
__global__ void bounds_kernel(const float *aabbs, u32t n, unsigned *b) {
    unsigned lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0, 0, 0};
    for (u32t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float *a = aabbs + 6 * (size_t)i;
        for (int k = 0; k < 3; k++) {
            lo[k] = min(lo[k], ord_bits(a[k]));
            hi[k] = max(hi[k], ord_bits(a[3 + k]));
        }
    }
    for (int k = 0; k < 3; k++) {
        for (int off = 16; off; off >>= 1) {
            lo[k] = min(lo[k], __shfl_down_sync(0xFFFFFFFFu, lo[k], off));
            hi[k] = max(hi[k], __shfl_down_sync(0xFFFFFFFFu, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++) { atomicMin(b + k, lo[k]); atomicMax(b + 3 + k, hi[k]); }
}
__device__ __forceinline__ u32t spread10(u32t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ u32t quantize(float c, float lo, float scale) {
    float t = (c - lo) * scale;
    if (!(t > 0.0f)) return 0;
    if (t >= 1023.0f) return 1023;
    return (u32t)t;
}
__global__ void morton_kernel(const float *aabbs, u32t n, const unsigned *b, u32t *codes, u32t *order) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u32t q[3];
    const float *a = aabbs + 6 * (size_t)i;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        float lo = from_ord(b[k]), hi = from_ord(b[3 + k]);
        float ext = hi - lo;
        float scale = ext > 0.0f ? 1024.0f / ext : 0.0f;
        float c = (a[k] + a[3 + k]) * 0.5f;
        q[k] = quantize(c, lo, scale);
    }
    codes[i] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    order[i] = i;
}

// ---- exclusive scan (3 phases) -----------------------------------------------------------------
constexpr int SCAN_BLOCK = 1024;  // elements per block (256 threads x 4)
__device__ __forceinline__ u32t block_exclusive_scan_256(u32t v, u32t *smem, u32t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32t x = v;
    for (int off = 1; off < 32; off <<= 1) {
        u32t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        u32t w = lane < 8 ? smem[lane] : 0;
        for (int off = 1; off < 8; off <<= 1) {
            u32t y = __shfl_up_sync(0xFFFFFFFFu, w, off);
            if (lane >= off) w += y;
        }
        if (lane < 8) smem[lane] = w;
    }
    __syncthreads();
    total = smem[7];
    u32t base = warp ? smem[warp - 1] : 0;
    u32t r = base + x - v;
    __syncthreads();
    return r;
}
__global__ void scan_reduce_kernel(const u32t *in, u32t n, u32t *sums) {
    __shared__ u32t sm[8];
    u32t s = 0;
    u32t base = blockIdx.x * SCAN_BLOCK + threadIdx.x * 4;
    for (int k = 0; k < 4; k++) if (base + k < n) s += in[base + k];
    u32t total;
    block_exclusive_scan_256(s, sm, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void scan_top_kernel(u32t *sums, u32t nb, u32t *total_out) {
    __shared__ u32t sm[8];
    u32t carry = 0;
    for (u32t c = 0; c < nb; c += 256) {
        u32t i = c + threadIdx.x;
        u32t v = i < nb ? sums[i] : 0;
        u32t total;
        u32t ex = block_exclusive_scan_256(v, sm, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}
__global__ void scan_down_kernel(const u32t *in, u32t *out, u32t n, const u32t *sums) {
    __shared__ u32t sm[8];
    u32t base = blockIdx.x * SCAN_BLOCK + threadIdx.x * 4;
    u32t v[4], s = 0;
    for (int k = 0; k < 4; k++) { v[k] = base + k < n ? in[base + k] : 0; s += v[k]; }
    u32t total;
    u32t ex = block_exclusive_scan_256(s, sm, total) + sums[blockIdx.x];
    for (int k = 0; k < 4; k++) { if (base + k < n) out[base + k] = ex; ex += v[k]; }
}
void scan_exclusive_u32(const u32t *in, u32t *out, u32t n, u32t *sums, u32t *total, cudaStream_t st) {
    u32t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    scan_reduce_kernel<<<nb, 256, 0, st>>>(in, n, sums);
    scan_top_kernel<<<1, 256, 0, st>>>(sums, nb, total);
    scan_down_kernel<<<nb, 256, 0, st>>>(in, out, n, sums);
}

// ---- stable LSD radix sort of (code, value) -------------------------------------------------------
constexpr int RS_THREADS = 256, RS_ITEMS = 8, RS_TILE = RS_THREADS * RS_ITEMS;
__global__ void rs_hist_kernel(const u32t *keys, u32t n, int shift, u32t *hist, u32t nblocks) {
    __shared__ u32t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    for (int r = 0; r < RS_ITEMS; r++) {
        u32t idx = blockIdx.x * RS_TILE + r * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}
__global__ void rs_scatter_kernel(const u32t *kin, const u32t *vin, u32t *kout, u32t *vout, u32t n, int shift,
                                  const u32t *offsets, u32t nblocks) {
    __shared__ u32t base[256];
    __shared__ u32t wcnt[RS_THREADS / 32][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    base[tid] = offsets[tid * nblocks + blockIdx.x];
    __syncthreads();
    for (int r = 0; r < RS_ITEMS; r++) {
        u32t idx = blockIdx.x * RS_TILE + r * RS_THREADS + tid;
        bool valid = idx < n;
        u32t key = valid ? kin[idx] : 0, val = valid ? vin[idx] : 0;
        u32t d = valid ? (key >> shift) & 255u : 256u;
        for (int k = lane; k < 256; k += 32) wcnt[warp][k] = 0;
        __syncwarp();
        u32t peers = __match_any_sync(0xFFFFFFFFu, d);
        u32t below = peers & ((1u << lane) - 1u);
        if (valid && below == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        {
            u32t run = base[tid];
            for (int w = 0; w < RS_THREADS / 32; w++) { u32t c = wcnt[w][tid]; wcnt[w][tid] = run; run += c; }
            base[tid] = run;
        }
        __syncthreads();
        if (valid) {
            u32t pos = wcnt[warp][d] + __popc(below);
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
    }
}

size_t radix_sort_scratch_bytes(u32t n) {
    const size_t nblocks = (n + RS_TILE - 1) / RS_TILE;
    const size_t hist = 256 * nblocks;
    return sizeof(u32t) * (hist + (hist + SCAN_BLOCK - 1) / SCAN_BLOCK + 64);
}
int radix_sort_pairs(u32t *k0, u32t *v0, u32t *k1, u32t *v1, u32t n, int passes, void *scratch, cudaStream_t st) {
    const u32t nblocks = (n + RS_TILE - 1) / RS_TILE;
    u32t *hist = static_cast<u32t *>(scratch), *sums = hist + (size_t)256 * nblocks;
    u32t *kin = k0, *vin = v0, *kout = k1, *vout = v1;
    for (int pass = 0; pass < passes; pass++) {
        rs_hist_kernel<<<nblocks, RS_THREADS, 0, st>>>(kin, n, 8 * pass, hist, nblocks);
        scan_exclusive_u32(hist, hist, 256 * nblocks, sums, nullptr, st);
        rs_scatter_kernel<<<nblocks, RS_THREADS, 0, st>>>(kin, vin, kout, vout, n, 8 * pass, hist, nblocks);
        u32t *tk = kin; kin = kout; kout = tk;
        u32t *tv = vin; vin = vout; vout = tv;
    }
    return passes & 1;
}

// ---- Karras topology ------------------------------------------------------------------------------
__device__ __forceinline__ int delta(const u32t *codes, const u32t *order, u32t n, int i, int j) {
    if (j < 0 || j >= (int)n) return -1;
    unsigned long long a = ((unsigned long long)codes[i] << 32) | order[i];
    unsigned long long b = ((unsigned long long)codes[j] << 32) | order[j];
    return __clzll(a ^ b);
}
__global__ void karras_kernel(const u32t *codes, const u32t *order, u32t n, u32t *first, u32t *last, u32t *lchild,
                              u32t *rchild, u32t *parent, u32t *leaf_parent) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int)n - 1) return;
    int d = (delta(codes, order, n, i, i + 1) - delta(codes, order, n, i, i - 1)) > 0 ? 1 : -1;
    int dmin = delta(codes, order, n, i, i - d);
    int lmax = 2;
    while (delta(codes, order, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(codes, order, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(codes, order, n, i, j);
    int s = 0;
    for (int t = (l + 1) / 2;; t = (t + 1) / 2) {
        if (delta(codes, order, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    int g = i + s * d + (d < 0 ? -1 : 0);
    int lo = min(i, j), hi = max(i, j);
    first[i] = lo;
    last[i] = hi;
    u32t lc = (lo == g) ? (0x80000000u | (u32t)g) : (u32t)g;
    u32t rc = (hi == g + 1) ? (0x80000000u | (u32t)(g + 1)) : (u32t)(g + 1);
    lchild[i] = lc;
    rchild[i] = rc;
    if (lc & 0x80000000u) leaf_parent[lc & 0x7FFFFFFFu] = i; else parent[lc] = i;
    if (rc & 0x80000000u) leaf_parent[rc & 0x7FFFFFFFu] = i; else parent[rc] = i;
    if (i == 0) parent[0] = 0xFFFFFFFFu;
}
__global__ void keep_flags_kernel(const u32t *first, const u32t *last, u32t ni, u32t max_leaf, u32t *flags) {
    u32t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ni) flags[k] = (last[k] - first[k] + 1 > max_leaf) ? 1u : 0u;
}

// bottom-up boxes of every internal node (first arrival stops, second combines)
__device__ __forceinline__ void item_box(const float *aabbs, u32t item, unsigned b[6]) {
    const float *a = aabbs + 6 * (size_t)item;
    for (int k = 0; k < 6; k++) b[k] = ord_bits(a[k]);
}
__device__ __forceinline__ void child_box(u32t ch, const float *aabbs, const u32t *order, const unsigned *kbox, unsigned b[6]) {
    if (ch & 0x80000000u) item_box(aabbs, order[ch & 0x7FFFFFFFu], b);
    else for (int k = 0; k < 6; k++) b[k] = __ldcg(kbox + 6 * (size_t)ch + k);
}
__global__ void karras_boxes_kernel(const float *aabbs, const u32t *order, u32t n, const u32t *lchild, const u32t *rchild,
                                    const u32t *parent, const u32t *leaf_parent, u32t *arrivals, unsigned *kbox) {
    u32t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    u32t p = leaf_parent[j];
    while (p != 0xFFFFFFFFu) {
        __threadfence();
        if (atomicAdd(arrivals + p, 1u) == 0) return;
        __threadfence();
        unsigned a[6], b[6];
        child_box(lchild[p], aabbs, order, kbox, a);
        child_box(rchild[p], aabbs, order, kbox, b);
        unsigned *o = kbox + 6 * (size_t)p;
        for (int k = 0; k < 3; k++) { __stcg(o + k, min(a[k], b[k])); __stcg(o + 3 + k, max(a[3 + k], b[3 + k])); }
        p = parent[p];
    }
}
__device__ __forceinline__ void write_node(BVHNode &o, const unsigned b[6], u32t first, u32t count, u32t depth) {
    o.aabb.min.x = from_ord(b[0]); o.aabb.min.y = from_ord(b[1]); o.aabb.min.z = from_ord(b[2]);
    o.aabb.max.x = from_ord(b[3]); o.aabb.max.y = from_ord(b[4]); o.aabb.max.z = from_ord(b[5]);
    o.first_child_id = first;
    o.child_count = (uint16_t)count;
    o.depth = (uint16_t)depth;
}
__global__ void layout_kernel(const float *aabbs, const u32t *order, u32t ni, const u32t *first, const u32t *last,
                              const u32t *lchild, const u32t *rchild, const u32t *parent, const u32t *flags,
                              const u32t *rank, const unsigned *kbox, BVHNode *out, u32t *height) {
    u32t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ni || !flags[k]) return;
    u32t dep = 0;
    for (u32t p = parent[k]; p != 0xFFFFFFFFu; p = parent[p]) dep++;
    if (k == 0) {
        unsigned b[6];
        for (int q = 0; q < 6; q++) b[q] = kbox[q];
        write_node(out[0], b, 1 + 2 * rank[0], 0, 0);
    }
    const u32t kids[2] = {lchild[k], rchild[k]};
    for (int c = 0; c < 2; c++) {
        const u32t ch = kids[c];
        unsigned b[6];
        BVHNode &o = out[1 + 2 * rank[k] + c];
        if (ch & 0x80000000u) {
            u32t f = ch & 0x7FFFFFFFu;
            item_box(aabbs, order[f], b);
            write_node(o, b, f, 1, dep + 1);
        } else {
            for (int q = 0; q < 6; q++) b[q] = kbox[6 * (size_t)ch + q];
            if (flags[ch]) write_node(o, b, 1 + 2 * rank[ch], 0, dep + 1);
            else write_node(o, b, first[ch], last[ch] - first[ch] + 1, dep + 1);
        }
    }
    atomicMax(height, dep + 1);
}
__global__ void single_leaf_kernel(const float *aabbs, const u32t *order, u32t n, BVHNode *out) {
    unsigned b[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0, 0, 0};
    for (u32t i = 0; i < n; i++) {
        unsigned c[6];
        item_box(aabbs, order[i], c);
        for (int k = 0; k < 3; k++) { b[k] = min(b[k], c[k]); b[3 + k] = max(b[3 + k], c[3 + k]); }
    }
    write_node(out[0], b, 0, n, 0);
}

__global__ void codes_by_item_kernel(const u32t *sorted_codes, const u32t *order, u32t n, u32t *out) {
    u32t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[order[k]] = sorted_codes[k];
}
void launch_codes_by_item(const LbvhScratch &s, u32t n, u32t *out, cudaStream_t st) {
    if (n) codes_by_item_kernel<<<(n + 255) / 256, 256, 0, st>>>(s.codes, s.order, n, out);
}

cudaError_t lbvh_reserve(LbvhScratch &s, u32t n) {
    if (n <= s.capacity) return cudaSuccess;
    lbvh_release(s);
    u32t cap = n < 1024 ? 1024 : n;
    u32t nblocks = (cap + RS_TILE - 1) / RS_TILE;
    size_t hist = (size_t)256 * nblocks + 2 * ((cap + SCAN_BLOCK - 1) / SCAN_BLOCK) + 64;
    cudaError_t e = cudaSuccess;
#define ST_ALLOC(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    ST_ALLOC(s.aabbs, sizeof(float) * 6 * cap);
    ST_ALLOC(s.bounds, sizeof(unsigned) * 8);
    ST_ALLOC(s.codes, sizeof(u32t) * cap);
    ST_ALLOC(s.codes_alt, sizeof(u32t) * cap);
    ST_ALLOC(s.order, sizeof(u32t) * cap);
    ST_ALLOC(s.order_alt, sizeof(u32t) * cap);
    ST_ALLOC(s.hist, sizeof(u32t) * hist * 2);
    ST_ALLOC(s.first, sizeof(u32t) * cap);
    ST_ALLOC(s.last, sizeof(u32t) * cap);
    ST_ALLOC(s.lchild, sizeof(u32t) * cap);
    ST_ALLOC(s.rchild, sizeof(u32t) * cap);
    ST_ALLOC(s.parent, sizeof(u32t) * cap);
    ST_ALLOC(s.leaf_parent, sizeof(u32t) * cap);
    ST_ALLOC(s.rank, sizeof(u32t) * cap);
    ST_ALLOC(s.flags, sizeof(u32t) * cap);
    ST_ALLOC(s.kbox, sizeof(unsigned) * 6 * cap);
    ST_ALLOC(s.info, sizeof(u32t) * 4);
#undef ST_ALLOC
    if (e != cudaSuccess) { lbvh_release(s); return e; }
    s.capacity = cap;
    return cudaSuccess;
}
static_assert(RS_TILE == 2048 && SCAN_BLOCK == 1024, "lbvh_scratch_bytes assumes these tile sizes");
void lbvh_carve(LbvhScratch &s, void *base, u32t cap) {
    char *p = static_cast<char *>(base);
    auto take = [&](size_t bytes) { char *q = p; p += lbvh_align(bytes); return q; };
    const u32t nblocks = (cap + RS_TILE - 1) / RS_TILE;
    const size_t hist = (size_t)256 * nblocks + 2 * ((cap + SCAN_BLOCK - 1) / SCAN_BLOCK) + 64;
    s = LbvhScratch();
    s.bounds = reinterpret_cast<unsigned *>(take(sizeof(unsigned) * 8));
    u32t **arrays[] = {&s.codes, &s.codes_alt, &s.order, &s.order_alt, &s.first, &s.last, &s.lchild, &s.rchild,
                       &s.parent, &s.leaf_parent, &s.rank, &s.flags};
    for (u32t **a : arrays) *a = reinterpret_cast<u32t *>(take(sizeof(u32t) * (size_t)cap));
    s.kbox = reinterpret_cast<unsigned *>(take(sizeof(unsigned) * 6 * (size_t)cap));
    s.info = reinterpret_cast<u32t *>(take(sizeof(u32t) * 4));
    s.hist = reinterpret_cast<u32t *>(take(sizeof(u32t) * hist * 2));
    s.capacity = cap;
}

void lbvh_release(LbvhScratch &s) {
    void *ptrs[] = {s.aabbs, s.bounds, s.codes, s.codes_alt, s.order, s.order_alt, s.hist, s.first, s.last, s.lchild,
                    s.rchild, s.parent, s.leaf_parent, s.rank, s.flags, s.kbox, s.info};
    for (void *p : ptrs) if (p) cudaFree(p);
    s = LbvhScratch();
}

cudaError_t lbvh_build(LbvhScratch &s, u32t n, u32t max_leaf, BVHNode *out_nodes, u32t *out_order, u32t info[2],
                       cudaStream_t st) {
    if (n == 0) { info[0] = 0; info[1] = 0; return cudaSuccess; }
    u32t h[3];
    lbvh_enqueue(s, n, max_leaf, out_nodes, out_order, h, st);
    cudaError_t e = cudaStreamSynchronize(st);
    info[0] = 1 + 2 * h[2];
    info[1] = h[1];
    return e;
}

void lbvh_enqueue(LbvhScratch &s, u32t n, u32t max_leaf, BVHNode *out_nodes, u32t *out_order, u32t *counts,
                  cudaStream_t st) {
    const u32t T = 256;
    bounds_init_kernel<<<1, 32, 0, st>>>(s.bounds);
    bounds_kernel<<<min((n + T - 1) / T, 1184u), T, 0, st>>>(s.aabbs, n, s.bounds);
    morton_kernel<<<(n + T - 1) / T, T, 0, st>>>(s.aabbs, n, s.bounds, s.codes, s.order);
    // radix sort, 4 passes; the result lands back in codes/order
    const u32t nblocks = (n + RS_TILE - 1) / RS_TILE;
    u32t *hist = s.hist, *sums = s.hist + (size_t)256 * nblocks;
    u32t *kin = s.codes, *vin = s.order, *kout = s.codes_alt, *vout = s.order_alt;
    for (int pass = 0; pass < 4; pass++) {
        rs_hist_kernel<<<nblocks, RS_THREADS, 0, st>>>(kin, n, 8 * pass, hist, nblocks);
        scan_exclusive_u32(hist, hist, 256 * nblocks, sums, nullptr, st);
        rs_scatter_kernel<<<nblocks, RS_THREADS, 0, st>>>(kin, vin, kout, vout, n, 8 * pass, hist, nblocks);
        u32t *tk = kin; kin = kout; kout = tk;
        u32t *tv = vin; vin = vout; vout = tv;
    }
    // after an even number of passes kin/vin are codes/order again
    if (n <= max_leaf) {
        single_leaf_kernel<<<1, 1, 0, st>>>(s.aabbs, s.order, n, out_nodes);
        cudaMemcpyAsync(out_order, s.order, sizeof(u32t) * n, cudaMemcpyDeviceToDevice, st);
        counts[0] = 0;                     // one node (1 + 2 * 0 kept internal nodes), height 1
        counts[1] = 1;
        counts[2] = 0;
        return;
    }
    const u32t ni = n - 1;
    karras_kernel<<<(ni + T - 1) / T, T, 0, st>>>(s.codes, s.order, n, s.first, s.last, s.lchild, s.rchild, s.parent,
                                                  s.leaf_parent);
    keep_flags_kernel<<<(ni + T - 1) / T, T, 0, st>>>(s.first, s.last, ni, max_leaf, s.flags);
    scan_exclusive_u32(s.flags, s.rank, ni, s.hist, s.info + 2, st);
    // arrivals reuse codes_alt (free after the sort)
    cudaMemsetAsync(s.codes_alt, 0, sizeof(u32t) * ni, st);
    karras_boxes_kernel<<<(n + T - 1) / T, T, 0, st>>>(s.aabbs, s.order, n, s.lchild, s.rchild, s.parent, s.leaf_parent,
                                                       s.codes_alt, s.kbox);
    cudaMemsetAsync(s.info + 1, 0, sizeof(u32t), st);
    layout_kernel<<<(ni + T - 1) / T, T, 0, st>>>(s.aabbs, s.order, ni, s.first, s.last, s.lchild, s.rchild, s.parent,
                                                  s.flags, s.rank, s.kbox, out_nodes, s.info + 1);
    cudaMemcpyAsync(out_order, s.order, sizeof(u32t) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(counts, s.info, sizeof(u32t) * 3, cudaMemcpyDeviceToHost, st);
}

// ---- refit of a reference-layout BVH ------------------------------------------------------------
__global__ void refit_parents_kernel(const BVHNode *nodes, u32t count, u32t *parent) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (i == 0) parent[0] = 0xFFFFFFFFu;
    const BVHNode nd = nodes[i];
    if (!nd.child_count && nd.first_child_id + 1 < count) {
        parent[nd.first_child_id] = i;
        parent[nd.first_child_id + 1] = i;
    }
}
__global__ void refit_kernel(BVHNode *nodes, u32t count, const u32t *leaf_ids, const float *aabbs, const u32t *parent,
                             u32t *arrivals, unsigned *box) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BVHNode nd = nodes[i];
    if (!nd.child_count) return;          // internal nodes are combined by their children's walk
    unsigned b[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0, 0, 0};
    for (u32t k = 0; k < nd.child_count; k++) {
        unsigned c[6];
        item_box(aabbs, leaf_ids[nd.first_child_id + k], c);
        for (int q = 0; q < 3; q++) { b[q] = min(b[q], c[q]); b[3 + q] = max(b[3 + q], c[3 + q]); }
    }
    for (int q = 0; q < 6; q++) __stcg(box + 6 * (size_t)i + q, b[q]);
    write_node(nodes[i], b, nd.first_child_id, nd.child_count, nd.depth);
    u32t p = parent[i];
    while (p != 0xFFFFFFFFu) {
        __threadfence();
        if (atomicAdd(arrivals + p, 1u) == 0) return;
        __threadfence();
        const BVHNode pn = nodes[p];
        const unsigned *l = box + 6 * (size_t)pn.first_child_id, *r = l + 6;
        unsigned m[6];
        for (int q = 0; q < 3; q++) { m[q] = min(__ldcg(l + q), __ldcg(r + q)); m[3 + q] = max(__ldcg(l + 3 + q), __ldcg(r + 3 + q)); }
        for (int q = 0; q < 6; q++) __stcg(box + 6 * (size_t)p + q, m[q]);
        write_node(nodes[p], m, pn.first_child_id, 0, pn.depth);
        p = parent[p];
    }
}
cudaError_t refit_bvh(BVHNode *nodes, u32t node_count, const u32t *leaf_ids, const float *aabbs,
                      u32t *scratch_parent, u32t *scratch_flags, unsigned *scratch_box, cudaStream_t st) {
    if (!node_count) return cudaSuccess;
    const u32t T = 256;
    refit_parents_kernel<<<(node_count + T - 1) / T, T, 0, st>>>(nodes, node_count, scratch_parent);
    cudaMemsetAsync(scratch_flags, 0, sizeof(u32t) * node_count, st);
    refit_kernel<<<(node_count + T - 1) / T, T, 0, st>>>(nodes, node_count, leaf_ids, aabbs, scratch_parent,
                                                         scratch_flags, scratch_box);
    return cudaGetLastError();
}

// ---- BLAS triangle records: updateMeshBVH builder_top_down.h:330-363 -----------------------------
__global__ void tri_records_kernel(const vec3 *pos, const vec3 *nrm, const vec2 *uv, const uint32_t *pidx,
                                   const uint32_t *nidx, const uint32_t *uidx, int has_uvs, const u32t *order, u32t n,
                                   Triangle *out, u32t *inverse) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32t t = order[i];
    inverse[t] = i;
    const v3 v1 = from(pos[pidx[3 * t]]), v2 = from(pos[pidx[3 * t + 1]]), v3_ = from(pos[pidx[3 * t + 2]]);
    v3 X = v3_ - v1, Y = v2 - v1, Z = cross(X, Y);
    Triangle r;
    r.area_of_parallelogram = len(Z);
    Z = vscale(Z, 1.0f / r.area_of_parallelogram);
    // invMat3 math/mat3.h:97 of the rows X, Y, Z
    float d = 1.0f / (
        + X.x * (Y.y * Z.z - Z.y * Y.z)
        - Y.x * (X.y * Z.z - Z.y * X.z)
        + Z.x * (X.y * Y.z - Y.y * X.z));
    r.world_to_tangent.X.x = + (Y.y * Z.z - Z.y * Y.z) * d;
    r.world_to_tangent.Y.x = - (Y.x * Z.z - Z.x * Y.z) * d;
    r.world_to_tangent.Z.x = + (Y.x * Z.y - Z.x * Y.y) * d;
    r.world_to_tangent.X.y = - (X.y * Z.z - Z.y * X.z) * d;
    r.world_to_tangent.Y.y = + (X.x * Z.z - Z.x * X.z) * d;
    r.world_to_tangent.Z.y = - (X.x * Z.y - Z.x * X.y) * d;
    r.world_to_tangent.X.z = + (X.y * Y.z - Y.y * X.z) * d;
    r.world_to_tangent.Y.z = - (X.x * Y.z - Y.x * X.z) * d;
    r.world_to_tangent.Z.z = + (X.x * Y.y - Y.x * X.y) * d;
    r.normal.x = Z.x; r.normal.y = Z.y; r.normal.z = Z.z;
    r.position = pos[pidx[3 * t]];
    r.vertex_normals[0] = nrm[nidx[3 * t]];
    r.vertex_normals[1] = nrm[nidx[3 * t + 1]];
    r.vertex_normals[2] = nrm[nidx[3 * t + 2]];
    r.area_of_uv = 0;
    r.uvs[0].x = r.uvs[0].y = r.uvs[1].x = r.uvs[1].y = r.uvs[2].x = r.uvs[2].y = 0;
    if (has_uvs) {
        vec2 a = r.uvs[0] = uv[uidx[3 * t]];
        vec2 b = r.uvs[1] = uv[uidx[3 * t + 1]];
        vec2 c = r.uvs[2] = uv[uidx[3 * t + 2]];
        r.area_of_uv = fabsf((b.x - a.x) * (c.y - a.y) - (c.x - a.x) * (b.y - a.y));
    }
    out[i] = r;
}

// ---- conversions into the traversal layouts ---------------------------------------------------
__global__ void make_pairs_kernel(const BVHNode *nodes, u32t node_count, NodePair *pairs) {
    u32t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 + 2 * k >= node_count) return;
    const BVHNode L = nodes[1 + 2 * k], R = nodes[2 + 2 * k];
    NodePair p;
    p.a = make_float4(L.aabb.min.x, L.aabb.min.y, L.aabb.min.z, L.aabb.max.x);
    p.b = make_float4(L.aabb.max.y, L.aabb.max.z, R.aabb.min.x, R.aabb.min.y);
    p.c = make_float4(R.aabb.min.z, R.aabb.max.x, R.aabb.max.y, R.aabb.max.z);
    p.d = make_uint4(L.child_count ? L.first_child_id : (L.first_child_id - 1) >> 1, L.child_count,
                     R.child_count ? R.first_child_id : (R.first_child_id - 1) >> 1, R.child_count);
    pairs[k] = p;
}
__global__ void make_trihot_kernel(const Triangle *tris, u32t n, TriHot *hot) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Triangle t = tris[i];
    const mat3 &m = t.world_to_tangent;
    TriHot h;
    h.p = make_float4(t.position.x, t.position.y, t.position.z, t.normal.x);
    h.q = make_float4(t.normal.y, t.normal.z, m.X.x, m.X.y);
    h.r = make_float4(m.X.z, m.Y.x, m.Y.y, m.Y.z);
    h.s = make_float4(m.Z.x, m.Z.y, m.Z.z, 0.0f);
    hot[i] = h;
}
__device__ __forceinline__ PrimDev primdev_of(const Primitive &p) {
    PrimDev d;
    unsigned bits = (unsigned)p.flags | ((unsigned)p.type << 8) | ((unsigned)p.material_id << 16);
    d.pos_bits = make_float4(p.position.x, p.position.y, p.position.z, __uint_as_float(bits));
    d.rot = make_float4(p.rotation.axis.x, p.rotation.axis.y, p.rotation.axis.z, p.rotation.amount);
    d.scale_id = make_float4(p.scale.x, p.scale.y, p.scale.z, __uint_as_float(p.id));
    d.inv_scale = make_float4(1.0f / p.scale.x, 1.0f / p.scale.y, 1.0f / p.scale.z, 0.0f);
    return d;
}
__global__ void make_primdev_kernel(const Primitive *prims, u32t n, PrimDev *out) {
    u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = primdev_of(prims[i]);
}
// Moved primitives: record k replaces primitive ids[k] (raw record and its PrimDev).  Ids are
// distinct within one call (the host checks), so no two threads write the same slot.
__global__ void scatter_prims_kernel(const Primitive *recs, const u32t *ids, u32t count, Primitive *raw, PrimDev *dev) {
    u32t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const Primitive p = recs[k];
    raw[ids[k]] = p;
    dev[ids[k]] = primdev_of(p);
}

void launch_prim_aabbs(const Primitive *prims, const MeshDev *meshes, u32t n, float *aabbs, cudaStream_t st) {
    if (n) prim_aabbs_kernel<<<(n + 127) / 128, 128, 0, st>>>(prims, meshes, n, aabbs);
}
void launch_tri_aabbs(const vec3 *pos, const uint32_t *idx, u32t n, float *aabbs, cudaStream_t st) {
    if (n) tri_aabbs_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, idx, n, aabbs);
}
void launch_tri_records(const vec3 *pos, const vec3 *nrm, const vec2 *uv, const uint32_t *pidx, const uint32_t *nidx,
                        const uint32_t *uidx, int has_uvs, const u32t *order, u32t n, Triangle *out, u32t *inverse,
                        cudaStream_t st) {
    if (n) tri_records_kernel<<<(n + 255) / 256, 256, 0, st>>>(pos, nrm, uv, pidx, nidx, uidx, has_uvs, order, n, out, inverse);
}
void launch_make_pairs(const BVHNode *nodes, u32t node_count, NodePair *pairs, cudaStream_t st) {
    u32t np = node_count > 1 ? (node_count - 1) / 2 : 0;
    if (np) make_pairs_kernel<<<(np + 255) / 256, 256, 0, st>>>(nodes, node_count, pairs);
}
void launch_make_trihot(const Triangle *tris, u32t n, TriHot *hot, cudaStream_t st) {
    if (n) make_trihot_kernel<<<(n + 255) / 256, 256, 0, st>>>(tris, n, hot);
}
void launch_make_primdev(const Primitive *prims, u32t n, PrimDev *out, cudaStream_t st) {
    if (n) make_primdev_kernel<<<(n + 127) / 128, 128, 0, st>>>(prims, n, out);
}
void launch_scatter_prims(const Primitive *recs, const u32t *ids, u32t count, Primitive *raw, PrimDev *dev,
                          cudaStream_t st) {
    if (count) scatter_prims_kernel<<<(count + 127) / 128, 128, 0, st>>>(recs, ids, count, raw, dev);
}

}  // namespace st
