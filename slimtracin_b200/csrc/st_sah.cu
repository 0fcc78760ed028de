// st_sah.cu — device binned-SAH BVH build (TLAS "binned SAH" mode, and BLAS on request).
//
// Breadth-first, one level per step, the same specification as the CPU oracle's orc_binned_sah:
//   centroid (min+max)*0.5; a node's box and centroid box are unions under the IEEE total order;
//   per axis with centroid extent e > 0, bin = clamp((c - lo) * (32 / e)) in [0, 31];
//   a split after bin k costs halfArea(L)*nL + halfArea(R)*nR (AABB.h:39), empty sides skipped,
//   the lowest cost wins with ties to the lower axis then the lower k; with no candidate the range
//   is split at its middle; the partition is stable; the split nodes of a level get child pairs in
//   level order (pair p -> slots 1+2p, 2+2p); depth = level; height = deepest leaf.
// Large tasks (> kSmall items) are binned by many blocks into global bins; small tasks are done by
// one block each in shared memory.  Bin counts are integers and boxes are min/max of ordered bits,
// so the result does not depend on the order the atomics land in.
#include <cstdio>
#include "st_kernels.h"

namespace st {

constexpr int kBins = 32;
constexpr int kSmall = 2048;           // items a single block partitions in shared memory
constexpr int kChunk = 2048;           // items per block when binning / partitioning a large task
constexpr int kBinWords = 13;          // count + box(6) + centroid box(6)

struct SahTask {
    u32t begin, end, slot, pad;
    unsigned box[6], cbox[6];          // ordered bits
};

__device__ __forceinline__ unsigned ob(float f) {
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fo(unsigned k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k); }
__device__ __forceinline__ u32t bin_of(float c, float lo, float scale) {
    float t = (c - lo) * scale;
    if (!(t > 0.0f)) return 0;
    if (t >= (float)(kBins - 1)) return kBins - 1;
    return (u32t)t;
}
__device__ __forceinline__ float half_area_bits(const unsigned *b) {
    float ex = fo(b[3]) - fo(b[0]), ey = fo(b[4]) - fo(b[1]), ez = fo(b[5]) - fo(b[2]);
    return ex * ey + ey * ez + ez * ex;
}
__device__ __forceinline__ void empty6(unsigned *b) {
    b[0] = b[1] = b[2] = 0xFFFFFFFFu;
    b[3] = b[4] = b[5] = 0u;
}
__device__ __forceinline__ void grow6(unsigned *b, const unsigned *c) {
    for (int q = 0; q < 3; q++) { b[q] = min(b[q], c[q]); b[3 + q] = max(b[3 + q], c[3 + q]); }
}
__device__ __forceinline__ void atomic_grow6(unsigned *b, const unsigned *c) {
    for (int q = 0; q < 3; q++) { atomicMin(b + q, c[q]); atomicMax(b + 3 + q, c[3 + q]); }
}

// ---- set-up: centroids and the root task ----------------------------------------------------
__global__ void sah_setup_kernel(const float *aabbs, u32t n, float *cent, u32t *ids, unsigned *root) {
    unsigned b[6], c[6];
    empty6(b);
    empty6(c);
    for (u32t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float *a = aabbs + 6 * (size_t)i;
        unsigned it[6], ct[6];
        for (int q = 0; q < 3; q++) {
            float cc = (a[q] + a[3 + q]) * 0.5f;
            cent[3 * (size_t)i + q] = cc;
            ct[q] = ct[3 + q] = ob(cc);
        }
        for (int q = 0; q < 6; q++) it[q] = ob(a[q]);
        grow6(b, it);
        grow6(c, ct);
        ids[i] = i;
    }
    for (int q = 0; q < 3; q++)
        for (int off = 16; off; off >>= 1) {
            b[q] = min(b[q], __shfl_down_sync(0xFFFFFFFFu, b[q], off));
            b[3 + q] = max(b[3 + q], __shfl_down_sync(0xFFFFFFFFu, b[3 + q], off));
            c[q] = min(c[q], __shfl_down_sync(0xFFFFFFFFu, c[q], off));
            c[3 + q] = max(c[3 + q], __shfl_down_sync(0xFFFFFFFFu, c[3 + q], off));
        }
    if ((threadIdx.x & 31) == 0) {
        atomic_grow6(root, b);
        atomic_grow6(root + 6, c);
    }
}
__global__ void sah_root_init_kernel(unsigned *root) {
    if (threadIdx.x == 0) { empty6(root); empty6(root + 6); }
}
__global__ void sah_root_task_kernel(const unsigned *root, u32t n, SahTask *tasks) {
    SahTask t;
    t.begin = 0;
    t.end = n;
    t.slot = 0;
    t.pad = 0;
    for (int q = 0; q < 6; q++) { t.box[q] = root[q]; t.cbox[q] = root[6 + q]; }
    tasks[0] = t;
}

// ---- per level: classification -------------------------------------------------------------
// flags: [0,nt) split, [nt,2nt) large, [2nt,3nt) chunks of large tasks
__global__ void sah_classify_kernel(const SahTask *tasks, u32t nt, u32t max_leaf, u32t *flags) {
    u32t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    u32t cnt = tasks[t].end - tasks[t].begin;
    bool split = cnt > max_leaf;
    bool large = cnt > (u32t)kSmall;
    flags[t] = split;
    flags[nt + t] = large;
    flags[2 * nt + t] = large ? (cnt + kChunk - 1) / kChunk : 0;
}
// scanned: [0,nt) pair index within the level, [nt,2nt) large rank, [2nt,3nt) chunk offset
__global__ void sah_large_list_kernel(const SahTask *tasks, u32t nt, const u32t *flags, const u32t *scanned,
                                      u32t *large_tasks, u32t *chunk_task) {
    u32t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt || !flags[nt + t]) return;
    u32t r = scanned[nt + t];
    large_tasks[r] = t;
    u32t off = scanned[2 * nt + t], c = flags[2 * nt + t];
    for (u32t k = 0; k < c; k++) chunk_task[off + k] = r;
}

// ---- large tasks: global binning ------------------------------------------------------------
__device__ __forceinline__ void task_axes(const SahTask &T, float lo[3], float scale[3], bool valid[3]) {
    for (int a = 0; a < 3; a++) {
        float l = fo(T.cbox[a]), h = fo(T.cbox[3 + a]);
        float e = h - l;
        valid[a] = e > 0.0f;
        lo[a] = l;
        scale[a] = valid[a] ? (float)kBins / e : 0.0f;
    }
}
__global__ void sah_bin_large_kernel(const SahTask *tasks, const u32t *large_tasks, const u32t *chunk_task,
                                     const u32t *chunk_offsets, const u32t *ids, const float *aabbs, const float *cent,
                                     unsigned *gbins) {
    __shared__ unsigned sb[3 * kBins * kBinWords];
    const u32t r = chunk_task[blockIdx.x];
    const SahTask T = tasks[large_tasks[r]];
    const u32t chunk = blockIdx.x - chunk_offsets[large_tasks[r]];
    for (int k = threadIdx.x; k < 3 * kBins; k += blockDim.x) {
        unsigned *b = sb + k * kBinWords;
        b[0] = 0;
        empty6(b + 1);
        empty6(b + 7);
    }
    __syncthreads();
    float lo[3], scale[3];
    bool valid[3];
    task_axes(T, lo, scale, valid);
    const u32t first = T.begin + chunk * kChunk, last = min(T.end, first + kChunk);
    for (u32t k = first + threadIdx.x; k < last; k += blockDim.x) {
        const u32t i = ids[k];
        unsigned it[6], ct[6];
        for (int q = 0; q < 6; q++) it[q] = ob(aabbs[6 * (size_t)i + q]);
        for (int q = 0; q < 3; q++) ct[q] = ct[3 + q] = ob(cent[3 * (size_t)i + q]);
        for (int a = 0; a < 3; a++) {
            if (!valid[a]) continue;
            unsigned *b = sb + (a * kBins + bin_of(cent[3 * (size_t)i + a], lo[a], scale[a])) * kBinWords;
            atomicAdd(b, 1u);
            atomic_grow6(b + 1, it);
            atomic_grow6(b + 7, ct);
        }
    }
    __syncthreads();
    unsigned *g = gbins + (size_t)r * 3 * kBins * kBinWords;
    for (int k = threadIdx.x; k < 3 * kBins; k += blockDim.x) {
        const unsigned *b = sb + k * kBinWords;
        if (!b[0]) continue;
        unsigned *d = g + k * kBinWords;
        atomicAdd(d, b[0]);
        atomic_grow6(d + 1, b + 1);
        atomic_grow6(d + 7, b + 7);
    }
}
__global__ void sah_clear_bins_kernel(unsigned *gbins, u32t nlarge) {
    u32t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlarge * 3 * kBins) return;
    unsigned *b = gbins + (size_t)k * kBinWords;
    b[0] = 0;
    empty6(b + 1);
    empty6(b + 7);
}

// Sweep the bins of one task (one warp; lanes 0..2 take one axis each).  Writes the decision
// (axis, k; axis -1 = middle split) and, for a binned split, the children's boxes and left count.
__device__ void sweep(const unsigned *bins, const bool valid[3], int lane, int &best_axis, int &best_k, float &best_cost) {
    float cost_a = INFINITY;
    int k_a = -1;
    if (lane < 3 && valid[lane]) {
        const unsigned *B = bins + lane * kBins * kBinWords;
        unsigned R[kBins][6];
        u32t nR[kBins];
        unsigned acc[6];
        empty6(acc);
        u32t an = 0;
        for (int b = kBins - 1; b >= 1; b--) {
            grow6(acc, B + b * kBinWords + 1);
            an += B[b * kBinWords];
            for (int q = 0; q < 6; q++) R[b][q] = acc[q];
            nR[b] = an;
        }
        empty6(acc);
        an = 0;
        for (int k = 0; k < kBins - 1; k++) {
            grow6(acc, B + k * kBinWords + 1);
            an += B[k * kBinWords];
            if (!an || !nR[k + 1]) continue;
            float cost = half_area_bits(acc) * (float)an + half_area_bits(R[k + 1]) * (float)nR[k + 1];
            if (cost < cost_a) { cost_a = cost; k_a = k; }
        }
    }
    float c0 = __shfl_sync(0xFFFFFFFFu, cost_a, 0), c1 = __shfl_sync(0xFFFFFFFFu, cost_a, 1), c2 = __shfl_sync(0xFFFFFFFFu, cost_a, 2);
    int k0 = __shfl_sync(0xFFFFFFFFu, k_a, 0), k1 = __shfl_sync(0xFFFFFFFFu, k_a, 1), k2 = __shfl_sync(0xFFFFFFFFu, k_a, 2);
    best_axis = -1;
    best_k = -1;
    best_cost = INFINITY;
    if (k0 >= 0 && c0 < best_cost) { best_cost = c0; best_axis = 0; best_k = k0; }
    if (k1 >= 0 && c1 < best_cost) { best_cost = c1; best_axis = 1; best_k = k1; }
    if (k2 >= 0 && c2 < best_cost) { best_cost = c2; best_axis = 2; best_k = k2; }
}

struct SahDecision { int axis, k; u32t nleft; unsigned lbox[6], lcbox[6], rbox[6], rcbox[6]; };

__device__ void side_boxes(const unsigned *bins, int axis, int k, SahDecision &d) {
    empty6(d.lbox); empty6(d.lcbox); empty6(d.rbox); empty6(d.rcbox);
    d.nleft = 0;
    const unsigned *B = bins + axis * kBins * kBinWords;
    for (int b = 0; b < kBins; b++) {
        if (b <= k) { grow6(d.lbox, B + b * kBinWords + 1); grow6(d.lcbox, B + b * kBinWords + 7); d.nleft += B[b * kBinWords]; }
        else { grow6(d.rbox, B + b * kBinWords + 1); grow6(d.rcbox, B + b * kBinWords + 7); }
    }
}

// one warp per large task
__global__ void sah_split_large_kernel(const SahTask *tasks, const u32t *large_tasks, u32t nlarge, const unsigned *gbins,
                                       SahDecision *dec) {
    const u32t r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (r >= nlarge) return;
    const int lane = threadIdx.x & 31;
    const SahTask T = tasks[large_tasks[r]];
    float lo[3], scale[3];
    bool valid[3];
    task_axes(T, lo, scale, valid);
    const unsigned *bins = gbins + (size_t)r * 3 * kBins * kBinWords;
    int axis, k;
    float cost;
    sweep(bins, valid, lane, axis, k, cost);
    if (lane == 0) {
        SahDecision d;
        d.axis = axis;
        d.k = k;
        if (axis >= 0) side_boxes(bins, axis, k, d);
        else {
            d.nleft = (T.end - T.begin) / 2;
            empty6(d.lbox); empty6(d.lcbox); empty6(d.rbox); empty6(d.rcbox);
        }
        dec[r] = d;
    }
}

// middle split of a large task: children's boxes from the items (rare: all centroids equal)
__global__ void sah_middle_boxes_kernel(const SahTask *tasks, const u32t *large_tasks, const u32t *chunk_task,
                                        const u32t *chunk_offsets, const u32t *ids, const float *aabbs,
                                        const float *cent, SahDecision *dec) {
    const u32t r = chunk_task[blockIdx.x];
    SahDecision &d = dec[r];
    if (d.axis >= 0) return;
    const SahTask T = tasks[large_tasks[r]];
    const u32t chunk = blockIdx.x - chunk_offsets[large_tasks[r]];
    const u32t mid = T.begin + d.nleft;
    const u32t first = T.begin + chunk * kChunk, last = min(T.end, first + kChunk);
    for (u32t k = first + threadIdx.x; k < last; k += blockDim.x) {
        const u32t i = ids[k];
        unsigned it[6], ct[6];
        for (int q = 0; q < 6; q++) it[q] = ob(aabbs[6 * (size_t)i + q]);
        for (int q = 0; q < 3; q++) ct[q] = ct[3 + q] = ob(cent[3 * (size_t)i + q]);
        if (k < mid) { atomic_grow6(d.lbox, it); atomic_grow6(d.lcbox, ct); }
        else { atomic_grow6(d.rbox, it); atomic_grow6(d.rcbox, ct); }
    }
}

// stable partition of large tasks: per-chunk left counts, a per-task scan over its chunks, scatter
__device__ __forceinline__ bool goes_left(const SahDecision &d, const float lo[3], const float scale[3], const float *cent,
                                          u32t i, u32t pos, u32t mid) {
    if (d.axis < 0) return pos < mid;
    return bin_of(cent[3 * (size_t)i + d.axis], lo[d.axis], scale[d.axis]) <= (u32t)d.k;
}
__global__ void sah_count_left_kernel(const SahTask *tasks, const u32t *large_tasks, const u32t *chunk_task,
                                      const u32t *chunk_offsets, const u32t *ids, const float *cent,
                                      const SahDecision *dec, u32t *chunk_left) {
    __shared__ u32t total;
    const u32t r = chunk_task[blockIdx.x];
    const SahTask T = tasks[large_tasks[r]];
    const SahDecision d = dec[r];
    const u32t chunk = blockIdx.x - chunk_offsets[large_tasks[r]];
    float lo[3], scale[3];
    bool valid[3];
    task_axes(T, lo, scale, valid);
    if (threadIdx.x == 0) total = 0;
    __syncthreads();
    const u32t first = T.begin + chunk * kChunk, last = min(T.end, first + kChunk);
    u32t c = 0;
    for (u32t k = first + threadIdx.x; k < last; k += blockDim.x)
        c += goes_left(d, lo, scale, cent, ids[k], k, T.begin + d.nleft);
    for (int off = 16; off; off >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&total, c);
    __syncthreads();
    if (threadIdx.x == 0) chunk_left[blockIdx.x] = total;
}
__global__ void sah_chunk_scan_kernel(const u32t *large_tasks, u32t nlarge, const u32t *chunk_offsets, const u32t *flags,
                                      u32t nt, u32t *chunk_left) {
    u32t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nlarge) return;
    u32t t = large_tasks[r];
    u32t off = chunk_offsets[t], c = flags[2 * nt + t], run = 0;
    for (u32t k = 0; k < c; k++) { u32t v = chunk_left[off + k]; chunk_left[off + k] = run; run += v; }
}
__global__ void sah_scatter_kernel(const SahTask *tasks, const u32t *large_tasks, const u32t *chunk_task,
                                   const u32t *chunk_offsets, const u32t *ids, const float *cent, const SahDecision *dec,
                                   const u32t *chunk_left, u32t *tmp) {
    __shared__ u32t warp_sums[8];
    __shared__ u32t carry;
    const u32t r = chunk_task[blockIdx.x];
    const SahTask T = tasks[large_tasks[r]];
    const SahDecision d = dec[r];
    const u32t chunk = blockIdx.x - chunk_offsets[large_tasks[r]];
    float lo[3], scale[3];
    bool valid[3];
    task_axes(T, lo, scale, valid);
    const u32t first = T.begin + chunk * kChunk, last = min(T.end, first + kChunk);
    const u32t left_before = chunk_left[blockIdx.x];
    const u32t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (u32t base = first; base < last; base += blockDim.x) {
        const u32t k = base + threadIdx.x;
        const bool in = k < last;
        const u32t i = in ? ids[k] : 0;
        const bool l = in && goes_left(d, lo, scale, cent, i, k, T.begin + d.nleft);
        const unsigned ball = __ballot_sync(0xFFFFFFFFu, l);
        if (lane == 0) warp_sums[warp] = __popc(ball);
        __syncthreads();
        u32t before = carry;
        for (u32t w = 0; w < warp; w++) before += warp_sums[w];
        before += __popc(ball & ((1u << lane) - 1u));
        if (in) {
            const u32t lrank = left_before + before;                   // left items before k in the task
            const u32t pos_in_task = k - T.begin;
            const u32t dst = l ? T.begin + lrank : T.begin + d.nleft + (pos_in_task - lrank);
            tmp[dst] = i;
        }
        __syncthreads();
        if (threadIdx.x == 0) { u32t s = 0; for (u32t w = 0; w < blockDim.x / 32; w++) s += warp_sums[w]; carry += s; }
        __syncthreads();
    }
}
__global__ void sah_copy_back_kernel(const SahTask *tasks, const u32t *large_tasks, const u32t *chunk_task,
                                     const u32t *chunk_offsets, const u32t *tmp, u32t *ids) {
    const u32t r = chunk_task[blockIdx.x];
    const SahTask T = tasks[large_tasks[r]];
    const u32t chunk = blockIdx.x - chunk_offsets[large_tasks[r]];
    const u32t first = T.begin + chunk * kChunk, last = min(T.end, first + kChunk);
    for (u32t k = first + threadIdx.x; k < last; k += blockDim.x) ids[k] = tmp[k];
}

// ---- small tasks: one block does binning, sweep and the stable partition in shared memory ----
__global__ void sah_small_kernel(const SahTask *tasks, u32t nt, const u32t *flags, u32t *ids, const float *aabbs,
                                 const float *cent, SahDecision *small_dec) {
    const u32t t = blockIdx.x;
    if (t >= nt) return;
    const SahTask T = tasks[t];
    const u32t cnt = T.end - T.begin;
    if (!flags[t] || flags[nt + t]) return;                  // leaves and large tasks are elsewhere
    __shared__ unsigned sb[3 * kBins * kBinWords];
    __shared__ u32t sids[kSmall], stmp[kSmall];
    __shared__ SahDecision sd;
    __shared__ u32t warp_sums[8];
    for (int k = threadIdx.x; k < 3 * kBins; k += blockDim.x) {
        unsigned *b = sb + k * kBinWords;
        b[0] = 0;
        empty6(b + 1);
        empty6(b + 7);
    }
    for (u32t k = threadIdx.x; k < cnt; k += blockDim.x) sids[k] = ids[T.begin + k];
    __syncthreads();
    float lo[3], scale[3];
    bool valid[3];
    task_axes(T, lo, scale, valid);
    for (u32t k = threadIdx.x; k < cnt; k += blockDim.x) {
        const u32t i = sids[k];
        unsigned it[6], ct[6];
        for (int q = 0; q < 6; q++) it[q] = ob(aabbs[6 * (size_t)i + q]);
        for (int q = 0; q < 3; q++) ct[q] = ct[3 + q] = ob(cent[3 * (size_t)i + q]);
        for (int a = 0; a < 3; a++) {
            if (!valid[a]) continue;
            unsigned *b = sb + (a * kBins + bin_of(cent[3 * (size_t)i + a], lo[a], scale[a])) * kBinWords;
            atomicAdd(b, 1u);
            atomic_grow6(b + 1, it);
            atomic_grow6(b + 7, ct);
        }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        int axis, k;
        float cost;
        sweep(sb, valid, threadIdx.x, axis, k, cost);
        if (threadIdx.x == 0) {
            sd.axis = axis;
            sd.k = k;
            if (axis >= 0) side_boxes(sb, axis, k, sd);
            else {
                sd.nleft = cnt / 2;
                empty6(sd.lbox); empty6(sd.lcbox); empty6(sd.rbox); empty6(sd.rcbox);
            }
        }
    }
    __syncthreads();
    if (sd.axis < 0) {  // middle split: boxes from the items
        for (u32t k = threadIdx.x; k < cnt; k += blockDim.x) {
            const u32t i = sids[k];
            unsigned it[6], ct[6];
            for (int q = 0; q < 6; q++) it[q] = ob(aabbs[6 * (size_t)i + q]);
            for (int q = 0; q < 3; q++) ct[q] = ct[3 + q] = ob(cent[3 * (size_t)i + q]);
            if (k < sd.nleft) { atomic_grow6(sd.lbox, it); atomic_grow6(sd.lcbox, ct); }
            else { atomic_grow6(sd.rbox, it); atomic_grow6(sd.rcbox, ct); }
        }
    }
    // stable partition through shared memory
    const u32t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32t carry = 0;
    for (u32t base = 0; base < cnt; base += blockDim.x) {
        const u32t k = base + threadIdx.x;
        const bool in = k < cnt;
        const u32t i = in ? sids[k] : 0;
        const bool l = in && (sd.axis < 0 ? k < sd.nleft
                                          : bin_of(cent[3 * (size_t)i + sd.axis], lo[sd.axis], scale[sd.axis]) <= (u32t)sd.k);
        const unsigned ball = __ballot_sync(0xFFFFFFFFu, l);
        if (lane == 0) warp_sums[warp] = __popc(ball);
        __syncthreads();
        u32t before = carry;
        for (u32t w = 0; w < warp; w++) before += warp_sums[w];
        before += __popc(ball & ((1u << lane) - 1u));
        if (in) stmp[l ? before : sd.nleft + (k - before)] = i;
        u32t s = 0;
        for (u32t w = 0; w < blockDim.x / 32; w++) s += warp_sums[w];
        __syncthreads();
        carry += s;
    }
    __syncthreads();
    for (u32t k = threadIdx.x; k < cnt; k += blockDim.x) ids[T.begin + k] = stmp[k];
    if (threadIdx.x == 0) small_dec[t] = sd;
}

// ---- per level: write nodes and the next level's tasks -------------------------------------------
__global__ void sah_emit_kernel(const SahTask *tasks, u32t nt, const u32t *flags, const u32t *scanned,
                                const SahDecision *large_dec, const SahDecision *small_dec, u32t pairs_before,
                                u32t level, BVHNode *nodes, SahTask *next, u32t *height) {
    u32t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const SahTask T = tasks[t];
    BVHNode &o = nodes[T.slot];
    o.aabb.min.x = fo(T.box[0]); o.aabb.min.y = fo(T.box[1]); o.aabb.min.z = fo(T.box[2]);
    o.aabb.max.x = fo(T.box[3]); o.aabb.max.y = fo(T.box[4]); o.aabb.max.z = fo(T.box[5]);
    o.depth = (uint16_t)level;
    if (!flags[t]) {
        o.first_child_id = T.begin;
        o.child_count = (uint16_t)(T.end - T.begin);
        atomicMax(height, level);
        return;
    }
    const SahDecision &d = flags[nt + t] ? large_dec[scanned[nt + t]] : small_dec[t];
    const u32t p = scanned[t];
    o.first_child_id = 1 + 2 * (pairs_before + p);
    o.child_count = 0;
    SahTask L, R;
    L.begin = T.begin; L.end = T.begin + d.nleft; L.slot = 1 + 2 * (pairs_before + p); L.pad = 0;
    R.begin = L.end; R.end = T.end; R.slot = L.slot + 1; R.pad = 0;
    for (int q = 0; q < 6; q++) { L.box[q] = d.lbox[q]; L.cbox[q] = d.lcbox[q]; R.box[q] = d.rbox[q]; R.cbox[q] = d.rcbox[q]; }
    next[2 * p] = L;
    next[2 * p + 1] = R;
}

// ---- host driver ------------------------------------------------------------------------------
struct SahScratch {
    size_t n = 0;
    char *base = nullptr;
};

void scan_exclusive_u32(const u32t *in, u32t *out, u32t n, u32t *sums, u32t *total, cudaStream_t st);

namespace {
struct SahLayout {
    size_t o_cent, o_tmp, o_ta, o_tb, o_flags, o_scan, o_sums, o_large, o_ctask, o_cleft, o_bins, o_ldec, o_sdec, o_misc;
    size_t bytes = 0;
};
// scratch: centroids, tmp ids, two task lists, flags/scans (3n each), large lists, bins, decisions
SahLayout sah_layout(u32t n) {
    SahLayout L;
    const size_t nb = n;
    const u32t max_large = (u32t)(n / kSmall + 2);
    const size_t max_chunks = n / kChunk + max_large + 2;
    auto add = [&](size_t b) { size_t off = L.bytes; L.bytes += (b + 255) & ~(size_t)255; return off; };
    L.o_cent = add(sizeof(float) * 3 * nb); L.o_tmp = add(sizeof(u32t) * nb);
    L.o_ta = add(sizeof(SahTask) * nb); L.o_tb = add(sizeof(SahTask) * nb);
    L.o_flags = add(sizeof(u32t) * 3 * nb + 64); L.o_scan = add(sizeof(u32t) * 3 * nb + 64);
    L.o_sums = add(sizeof(u32t) * (3 * nb / 1024 + 64));
    L.o_large = add(sizeof(u32t) * max_large); L.o_ctask = add(sizeof(u32t) * max_chunks);
    L.o_cleft = add(sizeof(u32t) * max_chunks);
    L.o_bins = add(sizeof(unsigned) * (size_t)max_large * 3 * kBins * kBinWords);
    L.o_ldec = add(sizeof(SahDecision) * max_large); L.o_sdec = add(sizeof(SahDecision) * nb);
    L.o_misc = add(sizeof(u32t) * 64);
    return L;
}
}  // namespace

size_t sah_scratch_bytes(u32t n) { return sah_layout(n).bytes; }

cudaError_t sah_build(const float *aabbs, u32t n, u32t max_leaf, BVHNode *out_nodes, u32t *out_order, u32t info[2],
                      cudaStream_t st, void *scratch, size_t scratch_bytes) {
    if (n == 0) { info[0] = info[1] = 0; return cudaSuccess; }
    const SahLayout Lo = sah_layout(n);
    const size_t o_cent = Lo.o_cent, o_tmp = Lo.o_tmp, o_ta = Lo.o_ta, o_tb = Lo.o_tb, o_flags = Lo.o_flags,
                 o_scan = Lo.o_scan, o_sums = Lo.o_sums, o_large = Lo.o_large, o_ctask = Lo.o_ctask,
                 o_cleft = Lo.o_cleft, o_bins = Lo.o_bins, o_ldec = Lo.o_ldec, o_sdec = Lo.o_sdec, o_misc = Lo.o_misc;
    // the caller's scratch when it is large enough, else a stream-ordered allocation
    char *base = nullptr;
    const bool own = !(scratch && scratch_bytes >= Lo.bytes);
    cudaError_t e = cudaSuccess;
    if (own) e = cudaMallocAsync((void **)&base, Lo.bytes, st);
    else base = static_cast<char *>(scratch);
    if (e != cudaSuccess) return e;
    float *cent = (float *)(base + o_cent);
    u32t *tmp = (u32t *)(base + o_tmp);
    SahTask *cur = (SahTask *)(base + o_ta), *next = (SahTask *)(base + o_tb);
    u32t *flags = (u32t *)(base + o_flags), *scanned = (u32t *)(base + o_scan), *sums = (u32t *)(base + o_sums);
    u32t *large = (u32t *)(base + o_large), *ctask = (u32t *)(base + o_ctask), *cleft = (u32t *)(base + o_cleft);
    unsigned *bins = (unsigned *)(base + o_bins);
    SahDecision *ldec = (SahDecision *)(base + o_ldec), *sdec = (SahDecision *)(base + o_sdec);
    u32t *misc = (u32t *)(base + o_misc);   // [0..12) root bits, [16..20) totals, [20] height
    u32t *ids = out_order;

    sah_root_init_kernel<<<1, 32, 0, st>>>(misc);
    sah_setup_kernel<<<min((n + 255) / 256, 1184u), 256, 0, st>>>(aabbs, n, cent, ids, misc);
    sah_root_task_kernel<<<1, 1, 0, st>>>(misc, n, cur);
    cudaMemsetAsync(misc + 20, 0, sizeof(u32t), st);
    u32t nt = 1, pairs = 0, level = 0;
    while (nt) {
        const u32t T = 256;
        sah_classify_kernel<<<(nt + T - 1) / T, T, 0, st>>>(cur, nt, max_leaf, flags);
        scan_exclusive_u32(flags, scanned, nt, sums, misc + 16, st);
        scan_exclusive_u32(flags + nt, scanned + nt, nt, sums, misc + 17, st);
        scan_exclusive_u32(flags + 2 * nt, scanned + 2 * nt, nt, sums, misc + 18, st);
        u32t tot[3];
        cudaMemcpyAsync(tot, misc + 16, sizeof(tot), cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) break;
        const u32t nsplit = tot[0], nlarge = tot[1], nchunks = tot[2];
        if (nlarge) {
            sah_large_list_kernel<<<(nt + T - 1) / T, T, 0, st>>>(cur, nt, flags, scanned, large, ctask);
            sah_clear_bins_kernel<<<(nlarge * 3 * kBins + T - 1) / T, T, 0, st>>>(bins, nlarge);
            sah_bin_large_kernel<<<nchunks, 256, 0, st>>>(cur, large, ctask, scanned + 2 * nt, ids, aabbs, cent, bins);
            sah_split_large_kernel<<<(nlarge + 3) / 4, 128, 0, st>>>(cur, large, nlarge, bins, ldec);
            sah_middle_boxes_kernel<<<nchunks, 256, 0, st>>>(cur, large, ctask, scanned + 2 * nt, ids, aabbs, cent, ldec);
            sah_count_left_kernel<<<nchunks, 256, 0, st>>>(cur, large, ctask, scanned + 2 * nt, ids, cent, ldec, cleft);
            sah_chunk_scan_kernel<<<(nlarge + T - 1) / T, T, 0, st>>>(large, nlarge, scanned + 2 * nt, flags, nt, cleft);
            sah_scatter_kernel<<<nchunks, 256, 0, st>>>(cur, large, ctask, scanned + 2 * nt, ids, cent, ldec, cleft, tmp);
            sah_copy_back_kernel<<<nchunks, 256, 0, st>>>(cur, large, ctask, scanned + 2 * nt, tmp, ids);
        }
        sah_small_kernel<<<nt, 256, 0, st>>>(cur, nt, flags, ids, aabbs, cent, sdec);
        sah_emit_kernel<<<(nt + T - 1) / T, T, 0, st>>>(cur, nt, flags, scanned, ldec, sdec, pairs, level, out_nodes, next,
                                                       misc + 20);
        pairs += nsplit;
        nt = 2 * nsplit;
        SahTask *sw = cur; cur = next; next = sw;
        level++;
    }
    u32t h = 0;
    if (e == cudaSuccess) {
        cudaMemcpyAsync(&h, misc + 20, sizeof(u32t), cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
    }
    if (own) cudaFreeAsync(base, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    info[0] = 1 + 2 * pairs;
    info[1] = h < 1 ? 1 : h;
    return e != cudaSuccess ? e : e2;
}

}  // namespace st
