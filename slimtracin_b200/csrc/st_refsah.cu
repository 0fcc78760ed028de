// st_refsah.cu — the reference's top-down SAH build (buildBVH, builder_top_down.h:204-263) on the
// device, node for node: ST_BVH_REF_SAH, for hosts whose images must follow the reference's TLAS
// topology (any-hit traversal order decides which occluder a shadow ray meets first).
//
// The reference builds depth first from an explicit stack, taking the right child first
// (:229-262); each split (splitBVHNode :168) sorts the node's items on every axis by aabb.max with
// its own quicksort (Lomuto partition, pivot last, :66-123 — not stable, so the order of equal keys
// is the algorithm's), sweeps the merged boxes from both ends (:125-166) and takes the first
// cheapest split (strict comparisons) of the first cheapest axis.  A split only reads and writes
// its own range of the item array, so the splits of one tree level are independent: here they run
// level by level, one block per node and one thread per axis, each thread running the reference's
// quicksort and sweeps as written.  Node numbers and leaf slots follow from the tree's shape: the
// reference numbers the children of its k-th split 1 + 2k, 2 + 2k and appends leaves as it reaches
// them, and both orders are the right-first depth-first order, which a bottom-up count of internal
// nodes and a top-down pass reproduce.  The depth fields are the reference's stack indices.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "st_kernels.h"

namespace st {
namespace {

// One node of the build: the items [start, end) of the item array, its box (set by the parent's
// split), whether it was split, and its children in the task array.
struct RefTask {
    u32t start, end;
    float box[6];
    u32t split;                 // 1: an internal node
    u32t left, right;           // task indices of the children
    u32t left_count;
};

constexpr u32t kSmemItems = 4096;   // ranges up to this many items sort in shared memory

__device__ __forceinline__ void merge_box(float *m, const float *b) {   // mergeAABBs AABB.h:25
    m[0] = m[0] < b[0] ? m[0] : b[0];
    m[1] = m[1] < b[1] ? m[1] : b[1];
    m[2] = m[2] < b[2] ? m[2] : b[2];
    m[3] = m[3] > b[3] ? m[3] : b[3];
    m[4] = m[4] > b[4] ? m[4] : b[4];
    m[5] = m[5] > b[5] ? m[5] : b[5];
}
__device__ __forceinline__ float half_area(const float *a) {            // getSurfaceAreaOfAABB AABB.h:39
    const float ex = a[3] - a[0], ey = a[4] - a[1], ez = a[5] - a[2];
    return ex * ey + ey * ez + ez * ex;
}

// sortNodesByAxis (:92) with partitionNodesByAxis (:66) over ids[0..m) keyed by keys[] (moved along
// with the ids); stack holds at most `cap` entries.  Returns false if the stack would overflow
// (it cannot for cap >= m; checked all the same).
__device__ bool lomuto_sort(u32t *ids, float *keys, int m, int *stack, int cap) {
    // keys strictly increasing: every partition keeps the order (each item is swapped with itself
    // and the pivot stays last), so the result is the input
    bool increasing = true;
    for (int i = 1; i < m && increasing; i++) increasing = keys[i - 1] < keys[i];
    if (increasing) return true;
    int top = -1;
    stack[++top] = 0;
    stack[++top] = m - 1;
    while (top >= 0) {
        const int end = stack[top--];
        const int start = stack[top--];
        const float pivot = keys[end];
        int p = start;
        for (int i = start; i < end; i++) {
            if (keys[i] < pivot) {
                const u32t ti = ids[i]; ids[i] = ids[p]; ids[p] = ti;
                const float tk = keys[i]; keys[i] = keys[p]; keys[p] = tk;
                p++;
            }
        }
        { const u32t ti = ids[end]; ids[end] = ids[p]; ids[p] = ti; }
        { const float tk = keys[end]; keys[end] = keys[p]; keys[p] = tk; }
        if (top + 5 > cap) return false;
        if (p - 1 > start) { stack[++top] = start; stack[++top] = p - 1; }
        if (p + 1 < end) { stack[++top] = p + 1; stack[++top] = end; }
    }
    return true;
}

// One level of splits: block b splits task first + b if it holds more than max_leaf items.  Thread
// a < 3 sorts a copy of the range on axis a and sweeps it (partitionBVHNodeIDs :125); thread 0 then
// picks the axis (:186-194), writes the chosen order back and appends the two children.
__global__ void refsah_level_kernel(const float *__restrict__ boxes, u32t *ids, RefTask *tasks, u32t first,
                                    u32t count, u32t max_leaf, u32t *sorted3, float *keys3, int *stack3,
                                    float *lsa3, float *rsa3, u32t n, u32t *task_count, unsigned *error) {
    extern __shared__ unsigned char smem[];
    __shared__ float s_best[3];
    __shared__ u32t s_left[3];
    const u32t ti = first + blockIdx.x;
    if (blockIdx.x >= count) return;
    RefTask &T = tasks[ti];
    const u32t m = T.end - T.start;
    if (m <= max_leaf) return;                                    // a leaf
    const u32t a = threadIdx.x;
    if (a < 3) {
        const bool in_smem = m <= kSmemItems;
        u32t *sid = in_smem ? reinterpret_cast<u32t *>(smem) + a * m : sorted3 + (size_t)a * n + T.start;
        float *skey = in_smem ? reinterpret_cast<float *>(smem + 3 * sizeof(u32t) * m) + a * m
                              : keys3 + (size_t)a * n + T.start;
        for (u32t i = 0; i < m; i++) {
            const u32t id = ids[T.start + i];
            sid[i] = id;
            skey[i] = boxes[6 * id + 3 + a];                        // aabb.max[axis]
        }
        if (!lomuto_sort(sid, skey, (int)m, stack3 + (size_t)a * (n + 2) + T.start, (int)m + 2)) atomicOr(error, 1u);
        float *lsa = lsa3 + (size_t)a * n + T.start, *rsa = rsa3 + (size_t)a * n + T.start;
        float L[6], R[6];
        for (int k = 0; k < 6; k++) { L[k] = boxes[6 * sid[0] + k]; R[k] = boxes[6 * sid[m - 1] + k]; }
        for (u32t li = 0, ri = m - 1; li < m; li++, ri--) {
            if (li) {
                merge_box(L, boxes + 6 * sid[li]);
                merge_box(R, boxes + 6 * sid[ri]);
            }
            lsa[li] = half_area(L);
            rsa[ri] = half_area(R);
        }
        float best = INFINITY;
        u32t left_count = 1;
        for (u32t ci = 0, ni = 1, li = 1, ri = m - 1; ci < m - 1; ci++, ni++, li++, ri--) {
            const float cost = lsa[ci] * (float)li + rsa[ni] * (float)ri;
            if (best > cost) { best = cost; left_count = ni; }
        }
        s_best[a] = best;
        s_left[a] = left_count;
        if (in_smem) {                                           // keep the order for thread 0
            u32t *g = sorted3 + (size_t)a * n + T.start;
            for (u32t i = 0; i < m; i++) g[i] = sid[i];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int chosen = 0;
        float best = INFINITY;
        for (int k = 0; k < 3; k++)
            if (s_best[k] < best) { best = s_best[k]; chosen = k; }
        const u32t lc = s_left[chosen];
        const u32t *sid = sorted3 + (size_t)chosen * n + T.start;
        for (u32t i = 0; i < m; i++) ids[T.start + i] = sid[i];
        // the children's boxes: the chosen sweep's left box at lc - 1 and right box at lc, merged
        // in the sweep's own order (merging in another order could flip the sign of a zero)
        float L[6], R[6];
        for (int k = 0; k < 6; k++) { L[k] = boxes[6 * sid[0] + k]; R[k] = boxes[6 * sid[m - 1] + k]; }
        for (u32t i = 1; i < lc; i++) merge_box(L, boxes + 6 * sid[i]);
        for (u32t i = m - 2; i + 1 > lc; i--) merge_box(R, boxes + 6 * sid[i]);
        const u32t c = atomicAdd(task_count, 2u);
        RefTask &l = tasks[c], &r = tasks[c + 1];
        l.start = T.start; l.end = T.start + lc; r.start = T.start + lc; r.end = T.end;
        for (int k = 0; k < 6; k++) { l.box[k] = L[k]; r.box[k] = R[k]; }
        l.split = r.split = 0;
        T.split = 1;
        T.left = c;
        T.right = c + 1;
        T.left_count = lc;
    }
}

}  // namespace

// The reference's buildBVH over n item boxes (6 floats each, device memory), leaves of at most
// max_leaf items: nodes (2n BVHNodes, device), leaf_ids (n, device) as the reference writes them,
// info = {node_count, height}.  Synchronous on `st` (one host round trip per tree level).
cudaError_t refsah_build(const float *boxes, u32t n, u32t max_leaf, BVHNode *nodes, u32t *leaf_ids, u32t info[2],
                         cudaStream_t st) {
    if (n == 0) { info[0] = info[1] = 0; return cudaSuccess; }
    // host copy of the boxes: the numbering pass and the root leaf run on the host from the tasks
    std::vector<float> hboxes(6 * (size_t)n);
    cudaError_t e = cudaMemcpyAsync(hboxes.data(), boxes, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    std::vector<BVHNode> out(2 * (size_t)n);
    std::vector<u32t> out_leaf(n);
    memset(out.data(), 0, sizeof(BVHNode) * out.size());
    if (n <= max_leaf) {                                          // buildBVH :208-221
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
        float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (u32t i = 0; i < n; i++) {
            out_leaf[i] = i;
            const float *x = hboxes.data() + 6 * i;
            for (int k = 0; k < 3; k++) { b[k] = b[k] < x[k] ? b[k] : x[k]; b[3 + k] = b[3 + k] > x[3 + k] ? b[3 + k] : x[3 + k]; }
        }
        memcpy(&out[0].aabb, b, sizeof(b));
        out[0].child_count = (uint16_t)n;
        info[0] = 1;
        info[1] = 1;
        e = cudaMemcpyAsync(nodes, out.data(), sizeof(BVHNode), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(leaf_ids, out_leaf.data(), sizeof(u32t) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return e;
    }
    // scratch: item ids, tasks (at most 2n - 1), three axes of sorted ids, keys, sort stacks and sweeps
    const size_t b_ids = sizeof(u32t) * n, b_tasks = sizeof(RefTask) * 2 * (size_t)n, b_sorted = sizeof(u32t) * 3 * (size_t)n,
                 b_keys = sizeof(float) * 3 * (size_t)n, b_stack = sizeof(int) * 3 * ((size_t)n + 2),
                 b_sa = sizeof(float) * 3 * (size_t)n;
    char *base = nullptr;
    const size_t bytes = b_ids + b_tasks + b_sorted + b_keys + b_stack + 2 * b_sa + 64;
    if ((e = cudaMallocAsync((void **)&base, bytes, st)) != cudaSuccess) return e;
    u32t *d_ids = reinterpret_cast<u32t *>(base);
    RefTask *d_tasks = reinterpret_cast<RefTask *>(base + b_ids);
    u32t *d_sorted = reinterpret_cast<u32t *>(base + b_ids + b_tasks);
    float *d_keys = reinterpret_cast<float *>(base + b_ids + b_tasks + b_sorted);
    int *d_stack = reinterpret_cast<int *>(base + b_ids + b_tasks + b_sorted + b_keys);
    float *d_lsa = reinterpret_cast<float *>(base + b_ids + b_tasks + b_sorted + b_keys + b_stack);
    float *d_rsa = d_lsa + 3 * (size_t)n;
    u32t *d_misc = reinterpret_cast<u32t *>(d_rsa + 3 * (size_t)n);   // task count, error flag
    std::vector<u32t> iota(n);
    for (u32t i = 0; i < n; i++) iota[i] = i;
    RefTask root;
    memset(&root, 0, sizeof(root));
    root.start = 0;
    root.end = n;
    u32t misc[2] = {1, 0};
    e = cudaMemcpyAsync(d_ids, iota.data(), sizeof(u32t) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_tasks, &root, sizeof(root), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_misc, misc, sizeof(misc), cudaMemcpyHostToDevice, st);
    u32t first = 0, count = 1;
    const size_t smem = 3 * (sizeof(u32t) + sizeof(float)) * (size_t)std::min(n, kSmemItems);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(refsah_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    while (e == cudaSuccess && count) {
        refsah_level_kernel<<<count, 32, smem, st>>>(boxes, d_ids, d_tasks, first, count, max_leaf, d_sorted, d_keys,
                                                     d_stack, d_lsa, d_rsa, n, d_misc, d_misc + 1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(misc, d_misc, sizeof(misc), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && misc[1]) e = cudaErrorUnknown;
        const u32t total = misc[0];
        first += count;
        count = total - first;
    }
    std::vector<RefTask> tasks(first);
    std::vector<u32t> ids(n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tasks.data(), d_tasks, sizeof(RefTask) * first, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ids.data(), d_ids, sizeof(u32t) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(base, st);
    if (e != cudaSuccess) return e;
    // numbering (buildBVH :229-262): children appear after their parent in the task array, so one
    // backward sweep counts internal nodes per subtree and one forward sweep assigns, in the
    // reference's right-first depth-first order, split ranks (children's node ids), leaf slots and
    // stack indices
    const u32t nt = first;
    std::vector<u32t> internal(nt, 0), rank(nt, 0), slot(nt, 0), sidx(nt, 0), node_id(nt, 0);
    for (u32t i = nt; i-- > 0;)
        if (tasks[i].split) internal[i] = 1 + internal[tasks[i].left] + internal[tasks[i].right];
    u32t height = 1, splits = 0;
    for (u32t i = 0; i < nt; i++) {
        const RefTask &T = tasks[i];
        if (!T.split) continue;
        splits++;
        const u32t l = T.left, r = T.right;
        rank[r] = rank[i] + 1;
        rank[l] = rank[i] + 1 + internal[r];
        slot[r] = slot[i];
        slot[l] = slot[i] + (tasks[r].end - tasks[r].start);
        sidx[r] = sidx[i] + 1;
        sidx[l] = sidx[i];
        node_id[l] = 1 + 2 * rank[i];
        node_id[r] = 2 + 2 * rank[i];
        if (sidx[r] > height) height = sidx[r];
    }
    for (u32t i = 0; i < nt; i++) {
        const RefTask &T = tasks[i];
        BVHNode &N = out[node_id[i]];
        if (i) memcpy(&N.aabb, T.box, sizeof(T.box));
        if (T.split) {
            N.first_child_id = 1 + 2 * rank[i];
            N.child_count = 0;
        } else {
            N.first_child_id = slot[i];
            N.child_count = (uint16_t)(T.end - T.start);
            for (u32t k = 0; k < T.end - T.start; k++) out_leaf[slot[i] + k] = ids[T.start + k];
        }
    }
    // depth fields: a split writes its own stack index into both children (:251); a leaf then
    // writes its own (:237); the root keeps 0
    for (u32t i = 0; i < nt; i++) {
        const RefTask &T = tasks[i];
        if (!T.split) continue;
        out[node_id[T.left]].depth = out[node_id[T.right]].depth = (uint16_t)sidx[i];
    }
    for (u32t i = 0; i < nt; i++)
        if (!tasks[i].split && i) out[node_id[i]].depth = (uint16_t)sidx[i];
    out[0].depth = 0;
    // the root box: merge of its children's (:262)
    {
        const float *l = reinterpret_cast<const float *>(&out[1].aabb), *r = reinterpret_cast<const float *>(&out[2].aabb);
        float b[6];
        for (int k = 0; k < 3; k++) { b[k] = l[k] < r[k] ? l[k] : r[k]; b[3 + k] = l[3 + k] > r[3 + k] ? l[3 + k] : r[3 + k]; }
        memcpy(&out[0].aabb, b, sizeof(b));
    }
    info[0] = 1 + 2 * splits;
    info[1] = height;
    e = cudaMemcpyAsync(nodes, out.data(), sizeof(BVHNode) * info[0], cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(leaf_ids, out_leaf.data(), sizeof(u32t) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

}  // namespace st
