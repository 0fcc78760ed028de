// st_obj.cu — obj2mesh (obj2mesh.c:25) as a library path: a Wavefront OBJ parsed on the host's
// threads, its unique edges found on the device, its BLAS built on the device (st_update_mesh_bvh).
//
// Parsing keeps obj2mesh's reading of the file: fgets lines of at most 1023 characters, a line
// counted by its first two characters ("vn", "vt", "v ", "f "), the face layout taken from the
// first face line that has 0, 3 or 6 slashes, numbers read with the same sscanf formats (so every
// float is parsed by the C library exactly as the reference parses it), 1-based indices, the
// optional winding inversion swapping the second and third corner.
//
// The reference collects edges by searching its edge list for every triangle side (obj2mesh.c:
// 209-234), quadratic in the triangle count.  The device finds the same list — each undirected
// side once, ordered by where it first appears — with two stable radix sorts (by `to`, then by
// `from`) of (side, position) pairs, a first-of-run flag per position, and a scan over positions.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>
#include "st_kernels.h"

namespace st {

namespace {

// One fgets line of obj2mesh: [begin, begin + len) of the file, and what it holds.
struct ObjLine {
    size_t begin;
    uint32_t len;
    uint8_t kind;      // 0 other, 1 vertex, 2 normal, 3 uv, 4 face
};

bool read_file(const char *path, std::vector<char> &data) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (n < 0) { fclose(f); return false; }
    data.resize((size_t)n);
    const bool ok = n == 0 || fread(data.data(), 1, (size_t)n, f) == (size_t)n;
    fclose(f);
    return ok;
}

// Lines as fgets(line, 1024, file) returns them, classified as obj2mesh's counting loop
// (obj2mesh.c:45-66) classifies them, and the face layout (slashes in the first face line that has
// 0, 3 or 6 of them).
void scan_lines(const std::vector<char> &d, std::vector<ObjLine> &lines, ObjCounts &c) {
    size_t at = 0;
    const size_t n = d.size();
    c = ObjCounts();
    while (at < n) {
        const size_t limit = std::min(n, at + 1023);
        const void *nl = memchr(d.data() + at, '\n', limit - at);
        const size_t end = nl ? (size_t)(static_cast<const char *>(nl) - d.data()) + 1 : limit;
        ObjLine l;
        l.begin = at;
        l.len = (uint32_t)(end - at);
        l.kind = 0;
        const char a = l.len > 0 ? d[at] : 0, b = l.len > 1 ? d[at + 1] : 0;
        if (a == 'v' && b == 'n') { l.kind = 2; c.normals++; }
        else if (a == 'v' && b == 't') { l.kind = 3; c.uvs++; }
        else if (a == 'v' && b == ' ') { l.kind = 1; c.vertices++; }
        else if (a == 'f' && b == ' ') {
            l.kind = 4;
            c.triangles++;
            if (c.layout == 0) {
                int slashes = 0;
                for (size_t k = at; k < end; k++) slashes += d[k] == '/';
                if (slashes == 0) c.layout = 1;
                else if (slashes == 3) c.layout = 2;
                else if (slashes == 6) c.layout = 3;
            }
        }
        lines.push_back(l);
        at = end;
    }
}

__global__ void edge_keys_kernel(const uint32_t *ids, u32t n_sides, u32t *to_key, u32t *from_val, u32t *pos) {
    const u32t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_sides) return;
    const u32t t = p / 3, k = p % 3;
    u32t a = ids[3 * t + k], b = ids[3 * t + (k + 1) % 3];
    if (a > b) { const u32t s = a; a = b; b = s; }
    to_key[p] = b;
    from_val[p] = a;
    pos[p] = p;
}
__global__ void side_to_kernel(const uint32_t *ids, u32t n_sides, u32t *to_key) {
    const u32t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_sides) return;
    const u32t t = p / 3, k = p % 3;
    const u32t a = ids[3 * t + k], b = ids[3 * t + (k + 1) % 3];
    to_key[p] = a > b ? a : b;
}
__global__ void gather_kernel(const u32t *src, const u32t *idx, u32t n, u32t *dst) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
// After sorting by (from, to) with ties in position order, the first of each run is the side's
// first appearance: flag it at its position.
__global__ void first_flags_kernel(const u32t *from, const u32t *to, const u32t *pos, u32t n, u32t *flags) {
    const u32t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool head = i == 0 || from[i] != from[i - 1] || to[i] != to[i - 1];
    flags[pos[i]] = head ? 1u : 0u;
}
__global__ void emit_edges_kernel(const uint32_t *ids, u32t n_sides, const u32t *flags, const u32t *offsets,
                                  EdgeVertexIndices *edges) {
    const u32t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_sides || !flags[p]) return;
    const u32t t = p / 3, k = p % 3;
    u32t a = ids[3 * t + k], b = ids[3 * t + (k + 1) % 3];
    if (a > b) { const u32t s = a; a = b; b = s; }
    EdgeVertexIndices e;
    e.from = a;
    e.to = b;
    edges[offsets[p]] = e;
}

}  // namespace

int obj_count(const char *path, ObjCounts &c) {
    std::vector<char> data;
    if (!read_file(path, data)) return -1;
    std::vector<ObjLine> lines;
    scan_lines(data, lines, c);
    return 0;
}

int obj_parse(const char *path, bool invert_winding, const ObjCounts &expect, vec3 *positions, vec3 *normals, vec2 *uvs,
              uint32_t *position_ids, uint32_t *uv_ids, uint32_t *normal_ids) {
    std::vector<char> data;
    if (!read_file(path, data)) return -1;
    std::vector<ObjLine> lines;
    ObjCounts c;
    scan_lines(data, lines, c);
    if (c.vertices != expect.vertices || c.normals != expect.normals || c.uvs != expect.uvs ||
        c.triangles != expect.triangles || c.layout != expect.layout)
        return -1;
    // output slot of every line: the running count of its kind (the reference's pointer bumps)
    std::vector<uint32_t> slot(lines.size());
    uint32_t next[5] = {0, 0, 0, 0, 0};
    for (size_t i = 0; i < lines.size(); i++) slot[i] = next[lines[i].kind]++;
    const int v1 = 0, v2 = invert_winding ? 2 : 1, v3 = invert_winding ? 1 : 2;
    const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<int> bad(hw, 0);
    auto work = [&](unsigned w) {
        char line[1024];
        const size_t lo = lines.size() * w / hw, hi = lines.size() * (w + 1) / hw;
        for (size_t i = lo; i < hi; i++) {
            const ObjLine &l = lines[i];
            if (!l.kind) continue;
            memcpy(line, data.data() + l.begin, l.len);
            line[l.len] = 0;
            const uint32_t s = slot[i];
            if (l.kind == 1) {
                vec3 &p = positions[s];
                if (sscanf(line, "v %f %f %f", &p.x, &p.y, &p.z) != 3) bad[w] = 1;
            } else if (l.kind == 2) {
                vec3 &n = normals[s];
                if (sscanf(line, "vn %f %f %f", &n.x, &n.y, &n.z) != 3) bad[w] = 1;
            } else if (l.kind == 3) {
                vec2 &t = uvs[s];
                if (sscanf(line, "vt %f %f", &t.x, &t.y) != 2) bad[w] = 1;
            } else {
                int vi[3], ti[3], ni[3];
                if (sscanf(line, "f %d/%d/%d %d/%d/%d %d/%d/%d", &vi[v1], &ti[v1], &ni[v1], &vi[v2], &ti[v2], &ni[v2],
                           &vi[v3], &ti[v3], &ni[v3]) != 9) {
                    bad[w] = 1;
                    continue;
                }
                for (int k = 0; k < 3; k++) {
                    if (vi[k] < 1 || (uint32_t)vi[k] > c.vertices || ti[k] < 1 || (uint32_t)ti[k] > c.uvs || ni[k] < 1 ||
                        (uint32_t)ni[k] > c.normals)
                        bad[w] = 1;
                    position_ids[3 * (size_t)s + k] = (uint32_t)(vi[k] - 1);
                    uv_ids[3 * (size_t)s + k] = (uint32_t)(ti[k] - 1);
                    normal_ids[3 * (size_t)s + k] = (uint32_t)(ni[k] - 1);
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned w = 1; w < hw; w++) pool.emplace_back(work, w);
    work(0);
    for (auto &t : pool) t.join();
    for (int b : bad) if (b) return -2;
    return 0;
}

size_t unique_edges_scratch_bytes(u32t n_triangles) {
    const size_t n = 3 * (size_t)n_triangles, a = (4 * n + 255) / 256 * 256;
    return 9 * a + 4 * (n / 1024 + 2) + radix_sort_scratch_bytes((u32t)n) + 1024;
}

cudaError_t unique_edges(const uint32_t *dev_ids, u32t n_triangles, u32t n_vertices, void *scratch,
                         EdgeVertexIndices *dev_edges, u32t *n_edges, cudaStream_t st) {
    const u32t n = 3 * n_triangles, T = 256;
    *n_edges = 0;
    if (!n) return cudaSuccess;
    char *cur = static_cast<char *>(scratch);
    auto take = [&](size_t b) { char *p = cur; cur += (b + 255) / 256 * 256; return p; };
    u32t *k0 = reinterpret_cast<u32t *>(take(4 * (size_t)n)), *v0 = reinterpret_cast<u32t *>(take(4 * (size_t)n));
    u32t *k1 = reinterpret_cast<u32t *>(take(4 * (size_t)n)), *v1 = reinterpret_cast<u32t *>(take(4 * (size_t)n));
    u32t *from = reinterpret_cast<u32t *>(take(4 * (size_t)n)), *to = reinterpret_cast<u32t *>(take(4 * (size_t)n));
    u32t *flags = reinterpret_cast<u32t *>(take(4 * (size_t)n)), *offsets = reinterpret_cast<u32t *>(take(4 * (size_t)n));
    u32t *total = reinterpret_cast<u32t *>(take(16));
    u32t *sums = reinterpret_cast<u32t *>(take(4 * ((size_t)n / 1024 + 2)));
    void *sort_scratch = take(radix_sort_scratch_bytes(n));
    int passes = 0;
    for (u32t top = n_vertices ? n_vertices - 1 : 0; top; top >>= 8) passes++;
    passes = std::max(passes, 1);
    // to (key) with positions, from kept aside by position
    edge_keys_kernel<<<(n + T - 1) / T, T, 0, st>>>(dev_ids, n, k0, from, v0);
    int alt = radix_sort_pairs(k0, v0, k1, v1, n, passes, sort_scratch, st);
    u32t *pos = alt ? v1 : v0;                 // positions ordered by to
    u32t *spare_k = alt ? k0 : k1, *spare_v = alt ? v0 : v1;
    gather_kernel<<<(n + T - 1) / T, T, 0, st>>>(from, pos, n, spare_k);   // from, in that order
    // stable sort by from: ties keep the order by to, and within equal sides the position order
    u32t *a_k = spare_k, *a_v = pos, *b_k = alt ? k1 : k0, *b_v = spare_v;
    alt = radix_sort_pairs(a_k, a_v, b_k, b_v, n, passes, sort_scratch, st);
    u32t *sorted_from = alt ? b_k : a_k, *sorted_pos = alt ? b_v : a_v;
    // the `to` of each sorted entry, gathered through its position
    side_to_kernel<<<(n + T - 1) / T, T, 0, st>>>(dev_ids, n, flags);
    gather_kernel<<<(n + T - 1) / T, T, 0, st>>>(flags, sorted_pos, n, to);
    first_flags_kernel<<<(n + T - 1) / T, T, 0, st>>>(sorted_from, to, sorted_pos, n, flags);
    scan_exclusive_u32(flags, offsets, n, sums, total, st);
    emit_edges_kernel<<<(n + T - 1) / T, T, 0, st>>>(dev_ids, n, flags, offsets, dev_edges);
    cudaError_t e = cudaMemcpyAsync(n_edges, total, sizeof(u32t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

}  // namespace st
