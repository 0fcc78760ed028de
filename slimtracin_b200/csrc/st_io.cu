// st_io.cu — the reference's file formats as library calls (host code):
//   .mesh     loadMeshFromFile / saveMeshToFile / getMeshMemorySize   (scene/io.h:62-175)
//   .texture  loadTextureFromFile / getTextureMemorySize (scene/io.h:6-59) and the writer of
//             bmp2texture (bmp2texture.c:367-385)
//   .scene    loadSceneFromFile / saveSceneToFile                     (scene/io.h:178-213)
// The byte streams are the reference's: each struct or array written as it lies in memory, in the
// reference's order, with the 32-bit-u32 layout of include/slimtracin_types.h.  Unlike the
// reference's callbacks, every read is checked (a short file is an error, not a silent zero) and
// every destination is sized by the caller.
#include <cstdio>
#include <cstring>
#include <vector>
#include "slimtracin_b200.h"

namespace {

struct File {
    FILE *f = nullptr;
    File(const char *path, const char *mode) { f = path ? fopen(path, mode) : nullptr; }
    ~File() { if (f) fclose(f); }
    bool read(void *p, size_t n) { return n == 0 || fread(p, 1, n, f) == n; }
    bool write(const void *p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }
};

size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// The carve of a mesh file's arrays out of one caller block, in loadMeshFromFile's order.
struct MeshCarve {
    size_t positions, position_ids, edges, triangles, uvs, uv_ids, normals, normal_ids, nodes, leaf_ids, total;
};
MeshCarve mesh_carve(const Mesh &m) {
    MeshCarve c;
    size_t at = 0;
    auto take = [&](size_t b) { size_t o = at; at += align16(b); return o; };
    c.nodes = take(sizeof(BVHNode) * 2 * (size_t)m.triangle_count);   // initBVH: 2N nodes (core/init.h)
    c.leaf_ids = take(sizeof(u32) * (size_t)m.triangle_count);
    c.positions = take(sizeof(vec3) * (size_t)m.vertex_count);
    c.position_ids = take(sizeof(TriangleVertexIndices) * (size_t)m.triangle_count);
    c.edges = take(sizeof(EdgeVertexIndices) * (size_t)m.edge_count);
    c.triangles = take(sizeof(Triangle) * (size_t)m.triangle_count);
    c.uvs = take(sizeof(vec2) * (size_t)m.uvs_count);
    c.uv_ids = take(m.uvs_count ? sizeof(TriangleVertexIndices) * (size_t)m.triangle_count : 0);
    c.normals = take(sizeof(vec3) * (size_t)m.normals_count);
    c.normal_ids = take(m.normals_count ? sizeof(TriangleVertexIndices) * (size_t)m.triangle_count : 0);
    c.total = at;
    return c;
}

// The header of a .mesh file (scene/io.h:100-112): AABB, then vertex, triangle, edge, uv and
// normal counts, node count and height.
bool read_mesh_header(File &f, Mesh &m) {
    return f.read(&m.aabb, sizeof(AABB)) && f.read(&m.vertex_count, sizeof(u32)) &&
           f.read(&m.triangle_count, sizeof(u32)) && f.read(&m.edge_count, sizeof(u32)) &&
           f.read(&m.uvs_count, sizeof(u32)) && f.read(&m.normals_count, sizeof(u32)) &&
           f.read(&m.bvh.node_count, sizeof(u32)) && f.read(&m.bvh.height, sizeof(u32));
}

}  // namespace

extern "C" {

int64_t st_mesh_file_bytes(const char *path) {
    File f(path, "rb");
    if (!f.f) return -1;
    Mesh m;
    memset(&m, 0, sizeof(m));
    if (!read_mesh_header(f, m)) return -1;
    return (int64_t)mesh_carve(m).total;
}

int st_read_mesh_file(const char *path, Mesh *mesh, void *memory, uint64_t memory_bytes) {
    if (!path || !mesh || !memory) return ST_ERR_INVALID_ARG;
    File f(path, "rb");
    if (!f.f) return ST_ERR_IO;
    Mesh m;
    memset(&m, 0, sizeof(m));
    if (!read_mesh_header(f, m)) return ST_ERR_IO;
    if (m.bvh.node_count > 2 * (uint64_t)m.triangle_count) return ST_ERR_BAD_SCENE;
    const MeshCarve c = mesh_carve(m);
    if (c.total > memory_bytes) return ST_ERR_BUDGET;
    char *base = static_cast<char *>(memory);
    m.bvh.nodes = reinterpret_cast<BVHNode *>(base + c.nodes);
    m.bvh.leaf_ids = reinterpret_cast<u32 *>(base + c.leaf_ids);
    m.vertex_positions = reinterpret_cast<vec3 *>(base + c.positions);
    m.vertex_position_indices = reinterpret_cast<TriangleVertexIndices *>(base + c.position_ids);
    m.edge_vertex_indices = reinterpret_cast<EdgeVertexIndices *>(base + c.edges);
    m.triangles = reinterpret_cast<Triangle *>(base + c.triangles);
    m.vertex_uvs = m.uvs_count ? reinterpret_cast<vec2 *>(base + c.uvs) : nullptr;
    m.vertex_uvs_indices = m.uvs_count ? reinterpret_cast<TriangleVertexIndices *>(base + c.uv_ids) : nullptr;
    m.vertex_normals = m.normals_count ? reinterpret_cast<vec3 *>(base + c.normals) : nullptr;
    m.vertex_normal_indices = m.normals_count ? reinterpret_cast<TriangleVertexIndices *>(base + c.normal_ids) : nullptr;
    const size_t tri_ids = sizeof(TriangleVertexIndices) * (size_t)m.triangle_count;
    bool ok = f.read(m.vertex_positions, sizeof(vec3) * (size_t)m.vertex_count) &&
              f.read(m.vertex_position_indices, tri_ids) &&
              f.read(m.edge_vertex_indices, sizeof(EdgeVertexIndices) * (size_t)m.edge_count);
    if (ok && m.uvs_count) ok = f.read(m.vertex_uvs, sizeof(vec2) * (size_t)m.uvs_count) && f.read(m.vertex_uvs_indices, tri_ids);
    if (ok && m.normals_count)
        ok = f.read(m.vertex_normals, sizeof(vec3) * (size_t)m.normals_count) && f.read(m.vertex_normal_indices, tri_ids);
    ok = ok && f.read(m.triangles, sizeof(Triangle) * (size_t)m.triangle_count) &&
         f.read(m.bvh.nodes, sizeof(BVHNode) * (size_t)m.bvh.node_count) &&
         f.read(m.bvh.leaf_ids, sizeof(u32) * (size_t)m.triangle_count);
    if (!ok) return ST_ERR_IO;
    *mesh = m;
    return ST_OK;
}

int st_write_mesh_file(const char *path, const Mesh *mesh) {
    if (!path || !mesh) return ST_ERR_INVALID_ARG;
    const Mesh &m = *mesh;
    if ((m.vertex_count && !m.vertex_positions) || (m.triangle_count && (!m.vertex_position_indices || !m.triangles || !m.bvh.leaf_ids)) ||
        (m.edge_count && !m.edge_vertex_indices) || (m.uvs_count && (!m.vertex_uvs || !m.vertex_uvs_indices)) ||
        (m.normals_count && (!m.vertex_normals || !m.vertex_normal_indices)) || (m.bvh.node_count && !m.bvh.nodes))
        return ST_ERR_INVALID_ARG;
    File f(path, "wb");
    if (!f.f) return ST_ERR_IO;
    const size_t tri_ids = sizeof(TriangleVertexIndices) * (size_t)m.triangle_count;
    bool ok = f.write(&m.aabb, sizeof(AABB)) && f.write(&m.vertex_count, sizeof(u32)) &&
              f.write(&m.triangle_count, sizeof(u32)) && f.write(&m.edge_count, sizeof(u32)) &&
              f.write(&m.uvs_count, sizeof(u32)) && f.write(&m.normals_count, sizeof(u32)) &&
              f.write(&m.bvh.node_count, sizeof(u32)) && f.write(&m.bvh.height, sizeof(u32)) &&
              f.write(m.vertex_positions, sizeof(vec3) * (size_t)m.vertex_count) &&
              f.write(m.vertex_position_indices, tri_ids) &&
              f.write(m.edge_vertex_indices, sizeof(EdgeVertexIndices) * (size_t)m.edge_count);
    if (ok && m.uvs_count) ok = f.write(m.vertex_uvs, sizeof(vec2) * (size_t)m.uvs_count) && f.write(m.vertex_uvs_indices, tri_ids);
    if (ok && m.normals_count)
        ok = f.write(m.vertex_normals, sizeof(vec3) * (size_t)m.normals_count) && f.write(m.vertex_normal_indices, tri_ids);
    ok = ok && f.write(m.triangles, sizeof(Triangle) * (size_t)m.triangle_count) &&
         f.write(m.bvh.nodes, sizeof(BVHNode) * (size_t)m.bvh.node_count) &&
         f.write(m.bvh.leaf_ids, sizeof(u32) * (size_t)m.triangle_count);
    return ok ? ST_OK : ST_ERR_IO;
}

// .texture: width, height (u16), mipmap, wrap (bool), mip_count (u8), then per mip its width and
// height (u16) and (w+1)(h+1) TexelQuads.
int64_t st_texture_file_bytes(const char *path) {
    File f(path, "rb");
    if (!f.f) return -1;
    Texture t;
    memset(&t, 0, sizeof(t));
    if (!(f.read(&t.width, 2) && f.read(&t.height, 2) && f.read(&t.mipmap, 1) && f.read(&t.wrap, 1) &&
          f.read(&t.mip_count, 1)))
        return -1;
    size_t total = align16(sizeof(TextureMip) * t.mip_count);
    for (u8 i = 0; i < t.mip_count; i++) {
        u16 w, h;
        if (!(f.read(&w, 2) && f.read(&h, 2))) return -1;
        const size_t q = sizeof(TexelQuad) * ((size_t)w + 1) * ((size_t)h + 1);
        total += align16(q);
        if (fseek(f.f, (long)q, SEEK_CUR) != 0) return -1;
    }
    return (int64_t)total;
}

int st_read_texture_file(const char *path, Texture *texture, void *memory, uint64_t memory_bytes) {
    if (!path || !texture || !memory) return ST_ERR_INVALID_ARG;
    const int64_t need = st_texture_file_bytes(path);
    if (need < 0) return ST_ERR_IO;
    if ((uint64_t)need > memory_bytes) return ST_ERR_BUDGET;
    File f(path, "rb");
    if (!f.f) return ST_ERR_IO;
    Texture t;
    memset(&t, 0, sizeof(t));
    if (!(f.read(&t.width, 2) && f.read(&t.height, 2) && f.read(&t.mipmap, 1) && f.read(&t.wrap, 1) &&
          f.read(&t.mip_count, 1)))
        return ST_ERR_IO;
    char *base = static_cast<char *>(memory);
    t.mips = reinterpret_cast<TextureMip *>(base);
    size_t at = align16(sizeof(TextureMip) * t.mip_count);
    for (u8 i = 0; i < t.mip_count; i++) {
        TextureMip &mip = t.mips[i];
        if (!(f.read(&mip.width, 2) && f.read(&mip.height, 2))) return ST_ERR_IO;
        const size_t q = sizeof(TexelQuad) * ((size_t)mip.width + 1) * ((size_t)mip.height + 1);
        mip.texel_quads = reinterpret_cast<TexelQuad *>(base + at);
        if (!f.read(mip.texel_quads, q)) return ST_ERR_IO;
        at += align16(q);
    }
    *texture = t;
    return ST_OK;
}

int st_write_texture_file(const char *path, const Texture *texture) {
    if (!path || !texture || (texture->mip_count && !texture->mips)) return ST_ERR_INVALID_ARG;
    for (u8 i = 0; i < texture->mip_count; i++)
        if (!texture->mips[i].texel_quads) return ST_ERR_INVALID_ARG;
    File f(path, "wb");
    if (!f.f) return ST_ERR_IO;
    const Texture &t = *texture;
    bool ok = f.write(&t.width, 2) && f.write(&t.height, 2) && f.write(&t.mipmap, 1) && f.write(&t.wrap, 1) &&
              f.write(&t.mip_count, 1);
    for (u8 i = 0; ok && i < t.mip_count; i++) {
        const TextureMip &mip = t.mips[i];
        ok = f.write(&mip.width, 2) && f.write(&mip.height, 2) &&
             f.write(mip.texel_quads, sizeof(TexelQuad) * ((size_t)mip.width + 1) * ((size_t)mip.height + 1));
    }
    return ok ? ST_OK : ST_ERR_IO;
}

// .scene: SceneSettings, then settings.cameras Camera records, then settings.primitives Primitive
// records (each only when the scene has that array).
int st_read_scene_file(const char *path, Scene *scene, uint32_t camera_capacity, uint32_t primitive_capacity) {
    if (!path || !scene) return ST_ERR_INVALID_ARG;
    File f(path, "rb");
    if (!f.f) return ST_ERR_IO;
    SceneSettings s;
    if (!f.read(&s, sizeof(s))) return ST_ERR_IO;
    if ((scene->cameras && s.cameras > camera_capacity) || (scene->primitives && s.primitives > primitive_capacity))
        return ST_ERR_BUDGET;
    std::vector<Camera> cams(scene->cameras ? s.cameras : 0);
    std::vector<Primitive> prims(scene->primitives ? s.primitives : 0);
    if (!f.read(cams.data(), sizeof(Camera) * cams.size()) || !f.read(prims.data(), sizeof(Primitive) * prims.size()))
        return ST_ERR_IO;
    // counts from the file; the caller's strings stay (the file's pointers belong to the writer)
    s.file = scene->settings.file;
    s.mesh_files = scene->settings.mesh_files;
    s.texture_files = scene->settings.texture_files;
    scene->settings = s;
    for (size_t i = 0; i < cams.size(); i++) {
        Camera &c = scene->cameras[i];
        c = cams[i];
        c.transform.right_direction = &c.transform.rotation_matrix.X;
        c.transform.up_direction = &c.transform.rotation_matrix.Y;
        c.transform.forward_direction = &c.transform.rotation_matrix.Z;
    }
    if (!prims.empty()) memcpy(scene->primitives, prims.data(), sizeof(Primitive) * prims.size());
    return ST_OK;
}

int st_write_scene_file(const char *path, const Scene *scene) {
    if (!path || !scene) return ST_ERR_INVALID_ARG;
    File f(path, "wb");
    if (!f.f) return ST_ERR_IO;
    bool ok = f.write(&scene->settings, sizeof(SceneSettings));
    if (ok && scene->cameras) ok = f.write(scene->cameras, sizeof(Camera) * (size_t)scene->settings.cameras);
    if (ok && scene->primitives) ok = f.write(scene->primitives, sizeof(Primitive) * (size_t)scene->settings.primitives);
    return ok ? ST_OK : ST_ERR_IO;
}

}  // extern "C"
