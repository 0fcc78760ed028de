// st_api.cu — the C ABI of libslimtracin_b200 (include/slimtracin_b200.h): context, scene residency,
// BVH builds and the render entry points.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include "slimtracin_b200.h"
#include "slimtracin_layout.h"
#include "st_kernels.h"

using namespace st;

namespace {

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

// The arrays a transform update rewrites: primitive records and the TLAS.  The serving loop gives a
// scene a fresh copy of them when batches still in flight read the current one (scene versions).
struct MotionBufs {
    DevBuf prims_raw, prims, tlas_nodes, tlas_leaf_ids, tlas_pairs, tlas_aabbs, tlas_scratch;
};

struct SceneSlot {
    bool allocated = false;
    u32t n_prims = 0, n_materials = 0, n_lights = 0, n_meshes = 0, n_textures = 0;
    u32t cap_prims = 0, cap_materials = 0, cap_lights = 0, cap_tris = 0, cap_meshes = 0, cap_mips = 0;
    size_t cap_quads = 0;
    DevBuf prims_raw, prims, materials, lights;
    DevBuf tlas_nodes, tlas_leaf_ids, tlas_pairs, tlas_aabbs, tlas_scratch;
    u32t tlas_node_count = 0, tlas_height = 0;
    u32t moved_since_build = 0;            // primitives moved since the TLAS was last built in full
    bool tlas_valid = false;
    BVHNode tlas_root{};
    DevBuf meshes, mesh_pairs, tri_hot, tri_full;
    std::vector<MeshDev> mesh_host;
    DevBuf outlines, outline_ranges;       // BLAS nodes drawBVH outlines (depth <= 5), per mesh ranges
    std::vector<uint2> outline_host;       // per mesh: (first outline, count)
    bool meshes_valid = false;
    DevBuf textures, mips, quads;
    DevBuf emissive, occluders;
    u32t n_emissive = 0, n_occluders = 0;
    vec3 ambient{};
    bool lights_present = false;
    std::vector<Primitive> prims_host;    // host copy for the emissive/occluder lists
    std::vector<Material> materials_host;
    std::vector<MotionBufs> spare;        // released scene versions, reused by the next update
};

DevBuf *motion_field(SceneSlot &S, MotionBufs &m, int k, DevBuf **mine) {
    DevBuf *a[7] = {&S.prims_raw, &S.prims, &S.tlas_nodes, &S.tlas_leaf_ids, &S.tlas_pairs, &S.tlas_aabbs, &S.tlas_scratch};
    DevBuf *b[7] = {&m.prims_raw, &m.prims, &m.tlas_nodes, &m.tlas_leaf_ids, &m.tlas_pairs, &m.tlas_aabbs, &m.tlas_scratch};
    *mine = a[k];
    return b[k];
}

}  // namespace

// A scene class's tuned batch launch: kernel variant (or kPerViewVariant), queue chunk and the
// warp-vote compaction threshold (0: no parking).
struct Tuned {
    int variant = 0, chunk = 1, threshold = 0;
};

struct BatchState {
    DevBuf table, ssb, seg, out_float, out_u8, counter;
    DevBuf park;                        // the parked-ray queue (ParkedRay records), when compaction is on
    BatchView *staging = nullptr;       // pinned host copy of the device view table
    size_t staging_cap = 0;
    BatchTable host_table;              // the view table of the launch group being issued (a kernel parameter)
    // launch mode 1 (one kernel per view): the streams the views are spread over and the events that
    // fork them from and join them back to the launching stream (created on first use)
    cudaStream_t aux[kAuxStreams] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kAuxStreams] = {};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::map<std::string, Tuned> tuned;                 // scene-class key -> tuned launch
};

struct ServeReq {
    uint64_t id = 0;
    int slot = 0;
    ViewDev view{};
    bool has_scene_values = false;
    vec3 ambient{};
    bool lights_present = false;
    FloatPixel *out_float = nullptr;
    Pixel *out_u8 = nullptr;
    std::vector<Primitive> moved;
    std::vector<uint32_t> moved_ids;
    double arrival = 0, launch = 0, done = 0;
    int status = ST_ERR_NOT_READY;
    uint64_t rays = 0;
    int batch_size = 0;
    size_t dev_float = 0, dev_ssb = 0, dev_seg = 0, dev_u8 = 0;   // byte offsets in the batch's device arena
    size_t host_float = 0, host_u8 = 0;                           // byte offsets in the flight's pinned staging
    uint32_t *mapped_u8 = nullptr;     // the device view of a page-locked out_u8 (written by the resolve kernel)
    bool pinned_float = false;         // out_float is page-locked (one direct device-to-host copy)
};

cudaError_t ensure_aux(BatchState &B) {
    if (B.fork_ev) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < kAuxStreams && e == cudaSuccess; i++) {
        e = cudaStreamCreateWithFlags(&B.aux[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B.join_ev[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B.fork_ev, cudaEventDisableTiming);
    return e;
}
void release_aux(BatchState &B) {
    for (int i = 0; i < kAuxStreams; i++) {
        if (B.aux[i]) cudaStreamDestroy(B.aux[i]);
        if (B.join_ev[i]) cudaEventDestroy(B.join_ev[i]);
        B.aux[i] = nullptr;
        B.join_ev[i] = nullptr;
    }
    if (B.fork_ev) cudaEventDestroy(B.fork_ev);
    B.fork_ev = nullptr;
}

struct InFlight {
    bool busy = false;
    cudaStream_t stream = nullptr;
    cudaEvent_t done_ev = nullptr;
    BatchState B;
    DevBuf status;
    char *pinned = nullptr;            // host staging of the batch's outputs and status word
    size_t pinned_cap = 0;
    size_t bytes = 0;                  // device bytes this batch holds against the frame budget
    std::vector<std::shared_ptr<ServeReq>> reqs;
    std::set<int> scenes;
    uint64_t launch_id = 0;
};

// A scene version replaced while batches in flight still read it; it returns to the scene's
// spare list once every one of those batches has finished.
struct RetiredVersion {
    int slot = 0;
    MotionBufs bufs;
    std::vector<std::pair<int, uint64_t>> readers;   // (flight, launch id)
};

struct Server {
    std::thread worker;
    std::mutex m;
    std::condition_variable cv_work, cv_done;
    bool running = false, stop = false;
    std::deque<std::shared_ptr<ServeReq>> pending;
    std::map<uint64_t, std::shared_ptr<ServeReq>> tickets;
    std::vector<InFlight> flights;
    st_serve_config cfg{};
    uint64_t frame_budget = 0, inflight_bytes = 0;
    uint64_t next_id = 1, next_launch = 1;
    std::vector<RetiredVersion> retired;
    cudaMemPool_t pool = nullptr;       // per-batch arenas; keeps freed memory for the next batch
};

// A render into host memory is traced in up to this many column strips, so that each strip's float
// grid is copied to the host while the other strips are traced.  All strips are in flight at once:
// holding strip k back until strip k - 2 is done spreads their ends over the frame, but costs more
// in the trace than it gains in the copies.
constexpr int kRenderStrips = 8;

struct st_ctx {
    int device = 0;
    Server server;
    int sm_count = 148;
    int blocks_per_sm[BATCH_VARIANTS] = {1, 1, 1, 1, 1, 1, 1, 1};
    BatchState batch;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0, in_use = 0;
    std::vector<SceneSlot> slots;
    DevBuf ssb, dirs, out_float, out_u8, prim_ids, status, counters;
    DevBuf upd_host_dev;                 // st_update_primitives: records and ids on the device
    DevBuf sah_scratch;                  // binned-SAH builds (kept between builds)
    DevBuf overlay_scratch, overlay_frags;   // debug overlays: boxes/edges, and the plotted pixels
    char *upd_pinned = nullptr;          // ... and their pinned staging
    char *bvh_pinned = nullptr;          // a TLAS build's counts, nodes and leaf order, read back at once
    size_t bvh_pinned_cap = 0;
    size_t upd_pinned_cap = 0;
    // page-locked landing place of a render's status words and work counters, so that reading them
    // back is an asynchronous copy rather than a staged one
    unsigned long long *readback = nullptr;
    // renders into host memory, traced in column strips: one stream per strip (so that the strips
    // run as one grid does, and each strip's copy follows its own trace), a stream for the strips'
    // resolves, and the events that order them (created on first use)
    cudaStream_t strip_trace[kRenderStrips] = {}, strip_resolve = nullptr;
    cudaEvent_t strip_ev[2 * kRenderStrips + 2] = {};
    LbvhScratch lbvh;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::string cuda_error;
};

namespace {

int fail_cuda(st_ctx *ctx, cudaError_t e) {
    ctx->cuda_error = cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? ST_ERR_OUT_OF_MEMORY : ST_ERR_CUDA;
}
int ST_CUDA_LAST_impl(st_ctx *ctx) {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ST_OK : fail_cuda(ctx, e);
}
#define ST_CUDA_LAST() ST_CUDA_LAST_impl(ctx)
int ST_CUDA_SYNC(st_ctx *ctx) {
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? ST_OK : fail_cuda(ctx, e);
}
#define ST_CUDA(call)                                     \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return fail_cuda(ctx, e_); \
    } while (0)

void release(st_ctx *ctx, DevBuf &b) {
    if (b.ptr) {
        cudaFree(b.ptr);
        ctx->in_use -= b.bytes;
    }
    b = DevBuf();
}
// Grow `b` to at least `bytes` (contents are not kept).  Refuses past the context's budget.
int reserve(st_ctx *ctx, DevBuf &b, size_t bytes) {
    if (bytes <= b.bytes && b.ptr) return ST_OK;
    if (bytes == 0) bytes = 16;
    size_t add = bytes - (b.ptr ? b.bytes : 0);
    if (ctx->in_use + add > ctx->budget) return ST_ERR_BUDGET;
    release(ctx, b);
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    b.bytes = bytes;
    ctx->in_use += bytes;
    return ST_OK;
}
#define ST_TRY(x)                    \
    do {                             \
        int s_ = (x);                \
        if (s_ != ST_OK) return s_;  \
    } while (0)

template <class T> T *P(DevBuf &b) { return static_cast<T *>(b.ptr); }

SceneSlot *slot_of(st_ctx *ctx, int slot) {
    if (!ctx || slot < 0 || slot >= (int)ctx->slots.size()) return nullptr;
    return &ctx->slots[slot];
}

u32t total_triangles(const Scene *s) {
    u32t t = 0;
    for (u32t i = 0; i < s->settings.meshes; i++) t += s->meshes[i].triangle_count;
    return t;
}

int allocate(st_ctx *ctx, SceneSlot &S, const Scene *scene) {
    const u32t np = scene->settings.primitives, nm = scene->settings.materials, nl = scene->settings.lights;
    const u32t nt = scene->meshes ? total_triangles(scene) : 0;
    const u32t nmesh = scene->meshes ? scene->settings.meshes : 0;
    u32t nmip = 0;
    size_t nquad = 0;
    for (u32t t = 0; scene->textures && t < scene->settings.textures; t++) {
        nmip += scene->textures[t].mip_count;
        for (u32t m = 0; m < scene->textures[t].mip_count; m++)
            nquad += (size_t)(scene->textures[t].mips[m].width + 1) * (scene->textures[t].mips[m].height + 1);
    }
    ST_TRY(reserve(ctx, S.prims_raw, sizeof(Primitive) * np));
    ST_TRY(reserve(ctx, S.prims, sizeof(PrimDev) * np));
    ST_TRY(reserve(ctx, S.materials, sizeof(Material) * std::max(nm, 1u)));
    ST_TRY(reserve(ctx, S.lights, sizeof(Light) * std::max(nl, 1u)));
    ST_TRY(reserve(ctx, S.tlas_nodes, sizeof(BVHNode) * 2 * std::max(np, 1u)));
    ST_TRY(reserve(ctx, S.tlas_leaf_ids, sizeof(u32t) * std::max(np, 1u)));
    ST_TRY(reserve(ctx, S.tlas_pairs, sizeof(NodePair) * std::max(np, 1u)));
    ST_TRY(reserve(ctx, S.tlas_aabbs, sizeof(float) * 6 * std::max(np, 1u)));
    ST_TRY(reserve(ctx, S.tlas_scratch, (sizeof(u32t) * 2 + sizeof(unsigned) * 6) * 2 * std::max(np, 1u)));
    ST_TRY(reserve(ctx, S.meshes, sizeof(MeshDev) * std::max(nmesh, 1u)));
    ST_TRY(reserve(ctx, S.mesh_pairs, sizeof(NodePair) * std::max(nt, 1u)));
    ST_TRY(reserve(ctx, S.tri_hot, sizeof(TriHot) * std::max(nt, 1u)));
    ST_TRY(reserve(ctx, S.tri_full, sizeof(Triangle) * std::max(nt, 1u)));
    ST_TRY(reserve(ctx, S.textures, sizeof(TexDev) * std::max(scene->settings.textures, 1u)));
    ST_TRY(reserve(ctx, S.mips, sizeof(MipDev) * std::max(nmip, 1u)));
    ST_TRY(reserve(ctx, S.quads, sizeof(TexelQuad) * std::max(nquad, (size_t)1)));
    ST_TRY(reserve(ctx, S.emissive, sizeof(u32t) * std::max(np, 1u)));
    ST_TRY(reserve(ctx, S.occluders, sizeof(u32t) * std::max(np, 1u)));
    S.cap_prims = np;
    S.cap_materials = nm;
    S.cap_lights = nl;
    S.cap_tris = nt;
    S.cap_meshes = nmesh;
    S.cap_mips = nmip;
    S.cap_quads = nquad;
    S.allocated = true;
    return ST_OK;
}

bool fits(const SceneSlot &S, const Scene *scene) {
    if (!S.allocated) return false;
    if (scene->settings.primitives > S.cap_prims || scene->settings.materials > S.cap_materials ||
        scene->settings.lights > S.cap_lights)
        return false;
    if (scene->meshes && (scene->settings.meshes > S.cap_meshes || total_triangles(scene) > S.cap_tris)) return false;
    return true;
}

int ensure(st_ctx *ctx, SceneSlot &S, const Scene *scene) {
    if (fits(S, scene)) return ST_OK;
    return allocate(ctx, S, scene);
}

// emissive quads (closest_hit/surface.h:46-49,172-178) and the sphere/quad occluders of the
// analytic area-light shadow (surface.h:84-114), both in primitive index order
int refresh_lists(st_ctx *ctx, SceneSlot &S) {
    std::vector<u32t> em, oc;
    for (u32t i = 0; i < S.prims_host.size(); i++) {
        const Primitive &p = S.prims_host[i];
        if (p.type == PrimitiveType_Quad && p.material_id < S.materials_host.size() &&
            (S.materials_host[p.material_id].is & EMISSIVE))
            em.push_back(i);
        if (p.type == PrimitiveType_Sphere || p.type == PrimitiveType_Quad) oc.push_back(i);
    }
    S.n_emissive = (u32t)em.size();
    S.n_occluders = (u32t)oc.size();
    if (!em.empty()) ST_CUDA(cudaMemcpyAsync(S.emissive.ptr, em.data(), em.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (!oc.empty()) ST_CUDA(cudaMemcpyAsync(S.occluders.ptr, oc.data(), oc.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    return ST_CUDA_SYNC(ctx);
}

}  // namespace

// ================================================================================================
extern "C" {

const char *st_strerror(int s) {
    switch (s) {
        case ST_OK: return "ok";
        case ST_ERR_INVALID_ARG: return "invalid argument";
        case ST_ERR_NO_DEVICE: return "no usable CUDA device (sm_100 required)";
        case ST_ERR_CUDA: return "CUDA runtime error";
        case ST_ERR_OUT_OF_MEMORY: return "device allocation failed";
        case ST_ERR_BUDGET: return "device-memory budget exceeded";
        case ST_ERR_STACK_OVERFLOW: return "traversal stack overflow";
        case ST_ERR_TIMEOUT: return "device-side wait timed out";
        case ST_ERR_NOT_RESIDENT: return "scene slot is not resident";
        case ST_ERR_BAD_SCENE: return "inconsistent scene data";
        case ST_ERR_QUEUE_FULL: return "request queue full";
        case ST_ERR_NOT_READY: return "request not finished";
        case ST_ERR_CANCELLED: return "request cancelled";
        case ST_ERR_IO: return "file missing or truncated";
        default: return "unknown status";
    }
}

long st_layout_query(const char *name) {
    if (!name) return -1;
#define ST_Q_S(T) if (!strcmp(name, #T)) return (long)sizeof(T);
#define ST_Q_F(T, F) if (!strcmp(name, #T "." #F)) return (long)offsetof(T, F);
    ST_LAYOUT_LIST(ST_Q_S, ST_Q_F)
#undef ST_Q_S
#undef ST_Q_F
    return -1;
}

int st_init(st_ctx **out, const st_config *cfg) {
    if (!out) return ST_ERR_INVALID_ARG;
    *out = nullptr;
    int device = cfg ? cfg->device : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return ST_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return ST_ERR_NO_DEVICE;
    st_ctx *ctx = new st_ctx();
    ctx->device = device;
    ctx->budget = (cfg && cfg->memory_budget) ? cfg->memory_budget : (uint64_t)120 << 30;
    ctx->slots.resize((cfg && cfg->max_scenes > 0) ? cfg->max_scenes : 16);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e == cudaSuccess; i++) e = cudaEventCreate(&ctx->ev[i]);

    if (e != cudaSuccess) {
        delete ctx;
        return ST_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    for (int t = 0; t < BATCH_VARIANTS; t++) ctx->blocks_per_sm[t] = batch_blocks_per_sm(t);
    if (const char *path = getenv("ST_AUTOTUNE_CACHE")) {
        // one line per scene class: key, kernel variant, chunk, compaction threshold
        std::ifstream f(path);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream in(line);
            std::string key;
            Tuned t;
            if (in >> key >> t.variant >> t.chunk) {
                if (!(in >> t.threshold)) t.threshold = 0;
                ctx->batch.tuned[key] = t;
            }
        }
    }
    int s = reserve(ctx, ctx->status, 16);
    if (s == ST_OK) s = reserve(ctx, ctx->counters, sizeof(unsigned long long) * 16);
    if (s == ST_OK && cudaMallocHost((void **)&ctx->readback, sizeof(unsigned long long) * 20) != cudaSuccess) {
        ctx->readback = nullptr;
        s = ST_ERR_OUT_OF_MEMORY;
    }
    if (s != ST_OK) {
        st_shutdown(ctx);
        return s;
    }
    *out = ctx;
    return ST_OK;
}

void st_shutdown(st_ctx *ctx) {
    if (!ctx) return;
    st_serve_stop(ctx);
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < (int)ctx->slots.size(); i++) st_free_scene(ctx, i);
    for (DevBuf *b : {&ctx->ssb, &ctx->dirs, &ctx->out_float, &ctx->out_u8, &ctx->prim_ids, &ctx->status, &ctx->counters,
                      &ctx->upd_host_dev, &ctx->sah_scratch, &ctx->overlay_scratch, &ctx->overlay_frags})
        release(ctx, *b);
    if (ctx->upd_pinned) cudaFreeHost(ctx->upd_pinned);
    if (ctx->bvh_pinned) cudaFreeHost(ctx->bvh_pinned);
    if (ctx->readback) cudaFreeHost(ctx->readback);
    for (cudaEvent_t e : ctx->strip_ev) if (e) cudaEventDestroy(e);
    for (cudaStream_t t : ctx->strip_trace) if (t) cudaStreamDestroy(t);
    if (ctx->strip_resolve) cudaStreamDestroy(ctx->strip_resolve);
    lbvh_release(ctx->lbvh);
    for (DevBuf *b : {&ctx->batch.table, &ctx->batch.ssb, &ctx->batch.seg, &ctx->batch.out_float, &ctx->batch.out_u8,
                      &ctx->batch.counter, &ctx->batch.park})
        release(ctx, *b);
    if (ctx->batch.exec) cudaGraphExecDestroy(ctx->batch.exec);
    if (ctx->batch.graph) cudaGraphDestroy(ctx->batch.graph);
    if (ctx->batch.staging) cudaFreeHost(ctx->batch.staging);
    for (auto &e : ctx->ev) if (e) cudaEventDestroy(e);
    release_aux(ctx->batch);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *st_last_cuda_error(st_ctx *ctx) { return ctx ? ctx->cuda_error.c_str() : ""; }
void *st_get_stream(st_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
uint64_t st_device_bytes_in_use(st_ctx *ctx) { return ctx ? ctx->in_use : 0; }

int st_free_scene(st_ctx *ctx, int slot) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S) return ST_ERR_INVALID_ARG;
    for (DevBuf *b : {&S->prims_raw, &S->prims, &S->materials, &S->lights, &S->tlas_nodes, &S->tlas_leaf_ids,
                      &S->tlas_pairs, &S->tlas_aabbs, &S->tlas_scratch, &S->meshes, &S->mesh_pairs, &S->tri_hot,
                      &S->tri_full, &S->textures, &S->mips, &S->quads, &S->emissive, &S->occluders, &S->outlines,
                      &S->outline_ranges})
        release(ctx, *b);
    for (MotionBufs &m : S->spare)
        for (int k = 0; k < 7; k++) {
            DevBuf *mine;
            release(ctx, *motion_field(*S, m, k, &mine));
        }
    *S = SceneSlot();
    return ST_OK;
}

int st_allocate_device_scene(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    return allocate(ctx, *S, scene);
}

int st_upload_primitives(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene || (scene->settings.primitives && !scene->primitives)) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    ST_TRY(ensure(ctx, *S, scene));
    const u32t n = scene->settings.primitives;
    for (u32t i = 0; i < n; i++) {
        const Primitive &p = scene->primitives[i];
        if (p.type == PrimitiveType_Mesh && (!scene->meshes || p.id >= scene->settings.meshes)) return ST_ERR_BAD_SCENE;
        if (p.material_id >= scene->settings.materials) return ST_ERR_BAD_SCENE;
    }
    S->n_prims = n;
    S->prims_host.assign(scene->primitives, scene->primitives + n);
    if (n) {
        ST_CUDA(cudaMemcpyAsync(S->prims_raw.ptr, scene->primitives, sizeof(Primitive) * n, cudaMemcpyHostToDevice, ctx->stream));
        launch_make_primdev(P<Primitive>(S->prims_raw), n, P<PrimDev>(S->prims), ctx->stream);
    }
    return refresh_lists(ctx, *S);
}

int st_upload_materials(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene || (scene->settings.materials && !scene->materials)) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    ST_TRY(ensure(ctx, *S, scene));
    const u32t n = scene->settings.materials;
    for (u32t i = 0; i < n; i++) {
        const Material &m = scene->materials[i];
        if (m.texture_count && m.use) {
            for (u32t k = 0; k < m.texture_count && k < 2; k++)
                if (m.texture_ids[k] >= scene->settings.textures || !scene->textures) return ST_ERR_BAD_SCENE;
        }
    }
    S->n_materials = n;
    S->materials_host.assign(scene->materials, scene->materials + n);
    if (n) ST_CUDA(cudaMemcpyAsync(S->materials.ptr, scene->materials, sizeof(Material) * n, cudaMemcpyHostToDevice, ctx->stream));
    return refresh_lists(ctx, *S);
}

int st_upload_lights(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene || (scene->settings.lights && !scene->lights)) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    ST_TRY(ensure(ctx, *S, scene));
    S->n_lights = scene->settings.lights;
    S->lights_present = scene->lights != nullptr;
    if (S->n_lights)
        ST_CUDA(cudaMemcpyAsync(S->lights.ptr, scene->lights, sizeof(Light) * S->n_lights, cudaMemcpyHostToDevice, ctx->stream));
    return ST_CUDA_SYNC(ctx);
}

static int upload_textures(st_ctx *ctx, SceneSlot &S, const Scene *scene) {
    std::vector<TexDev> tex;
    std::vector<MipDev> mips;
    size_t quad_off = 0;
    S.n_textures = scene->textures ? scene->settings.textures : 0;
    for (u32t t = 0; t < S.n_textures; t++) {
        const Texture &T = scene->textures[t];
        if (!T.mip_count || !T.mips) return ST_ERR_BAD_SCENE;
        TexDev d;
        d.width = T.width;
        d.height = T.height;
        d.mip_count = T.mip_count;
        d.wrap = T.wrap;
        d.mipmap = T.mipmap;
        d.pad = 0;
        d.mip_offset = (u32t)mips.size();
        tex.push_back(d);
        for (u32t m = 0; m < T.mip_count; m++) {
            const TextureMip &M = T.mips[m];
            size_t nq = (size_t)(M.width + 1) * (M.height + 1);
            if (quad_off + nq > S.cap_quads) return ST_ERR_BAD_SCENE;
            MipDev md;
            md.width = M.width;
            md.height = M.height;
            md.quad_offset = (u32t)quad_off;
            mips.push_back(md);
            ST_CUDA(cudaMemcpyAsync(P<TexelQuad>(S.quads) + quad_off, M.texel_quads, sizeof(TexelQuad) * nq,
                                    cudaMemcpyHostToDevice, ctx->stream));
            quad_off += nq;
        }
    }
    if (!tex.empty()) ST_CUDA(cudaMemcpyAsync(S.textures.ptr, tex.data(), sizeof(TexDev) * tex.size(), cudaMemcpyHostToDevice, ctx->stream));
    if (!mips.empty()) ST_CUDA(cudaMemcpyAsync(S.mips.ptr, mips.data(), sizeof(MipDev) * mips.size(), cudaMemcpyHostToDevice, ctx->stream));
    return ST_CUDA_SYNC(ctx);
}

int st_upload_scene(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (!fits(*S, scene)) ST_TRY(allocate(ctx, *S, scene));
    S->ambient = scene->ambient_light.color;
    ST_TRY(st_upload_lights(ctx, slot, scene));
    ST_TRY(st_upload_materials(ctx, slot, scene));
    ST_TRY(st_upload_primitives(ctx, slot, scene));
    return upload_textures(ctx, *S, scene);
}

// A reference-layout BVH is safe to walk when, starting from the root, every internal node's
// children pair lies inside the array and is reached exactly once (no cycles, no sharing), every
// leaf range lies inside the item array, and both the stated height and the depth the walk
// actually reaches leave stack room.  The walked depth is checked because the reference's
// top-down SAH builder (builder_top_down.h:243-266) records as a node's depth, and as the height,
// the index of its explicit build stack, where a left child keeps its parent's index and only a
// right child takes the next: that counts the right turns on a node's path, not its depth (11
// against 15 for a 4096-primitive TLAS).  A near-first walk keeps at most one pending sibling per
// level, so a tree whose deepest node is at depth d needs d stack entries; d + 2 <= kStack keeps
// the reference's two entries of slack.
static bool check_bvh(const BVHNode *nodes, u32t count, u32t items, u32t height) {
    if (!nodes || !count || height + 2 > (u32t)kStack) return false;
    if (nodes[0].child_count) return (uint64_t)nodes[0].first_child_id + nodes[0].child_count <= items;
    std::vector<uint8_t> seen(count, 0);
    std::vector<std::pair<u32t, u32t>> stack;    // (node, its depth)
    stack.push_back({0u, 0u});
    seen[0] = 1;
    while (!stack.empty()) {
        const u32t at = stack.back().first, depth = stack.back().second;
        stack.pop_back();
        const BVHNode &n = nodes[at];
        if (n.child_count) {
            if ((uint64_t)n.first_child_id + n.child_count > items) return false;
            continue;
        }
        if (depth + 1 + 2 > (u32t)kStack) return false;
        const u32t f = n.first_child_id;
        if (!(f & 1u) || (uint64_t)f + 1 >= count || seen[f] || seen[f + 1]) return false;
        seen[f] = seen[f + 1] = 1;
        stack.push_back({f, depth + 1});
        stack.push_back({f + 1, depth + 1});
    }
    return true;
}

int st_validate_bvh(const BVHNode *nodes, uint32_t node_count, uint32_t items, uint32_t height) {
    if (!nodes) return ST_ERR_INVALID_ARG;
    return check_bvh(nodes, node_count, items, height) ? ST_OK : ST_ERR_BAD_SCENE;
}

static int finish_tlas(st_ctx *ctx, SceneSlot &S) {
    if (S.tlas_node_count > 1)
        launch_make_pairs(P<BVHNode>(S.tlas_nodes), S.tlas_node_count, P<NodePair>(S.tlas_pairs), ctx->stream);
    ST_CUDA(cudaMemcpyAsync(&S.tlas_root, S.tlas_nodes.ptr, sizeof(BVHNode), cudaMemcpyDeviceToHost, ctx->stream));
    ST_TRY(ST_CUDA_SYNC(ctx));
    S.tlas_valid = true;
    return ST_OK;
}

int st_upload_scene_bvh(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene || !scene->bvh.nodes || !scene->bvh.leaf_ids) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    ST_TRY(ensure(ctx, *S, scene));
    const u32t n = scene->settings.primitives;
    if (!check_bvh(scene->bvh.nodes, scene->bvh.node_count, n, scene->bvh.height)) return ST_ERR_BAD_SCENE;
    for (u32t i = 0; i < n; i++) if (scene->bvh.leaf_ids[i] >= n) return ST_ERR_BAD_SCENE;
    S->tlas_node_count = scene->bvh.node_count;
    S->tlas_height = scene->bvh.height;
    cudaError_t e = cudaMemcpyAsync(S->tlas_nodes.ptr, scene->bvh.nodes, sizeof(BVHNode) * S->tlas_node_count,
                                    cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S->tlas_leaf_ids.ptr, scene->bvh.leaf_ids, sizeof(u32t) * n, cudaMemcpyHostToDevice, ctx->stream);
    S->moved_since_build = 0;
    const int status = e == cudaSuccess ? finish_tlas(ctx, *S) : fail_cuda(ctx, e);
    if (status != ST_OK) S->tlas_valid = false;     // the arrays may hold part of the new tree
    return status;
}

int st_upload_mesh_bvhs(st_ctx *ctx, int slot, const Scene *scene) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !scene || (scene->settings.meshes && !scene->meshes)) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    ST_TRY(ensure(ctx, *S, scene));
    S->mesh_host.clear();
    S->outline_host.clear();
    std::vector<OutlineBox> outlines;
    u32t tri_off = 0, pair_off = 0;
    for (u32t m = 0; m < scene->settings.meshes; m++) {
        const Mesh &M = scene->meshes[m];
        if (!M.triangles || !M.bvh.nodes || !check_bvh(M.bvh.nodes, M.bvh.node_count, M.triangle_count, M.bvh.height))
            return ST_ERR_BAD_SCENE;
        MeshDev d;
        memset(&d, 0, sizeof(d));
        d.pair_offset = pair_off;
        d.tri_offset = tri_off;
        d.triangle_count = M.triangle_count;
        d.root_count = M.bvh.nodes[0].child_count;
        d.root_first = M.bvh.nodes[0].first_child_id;
        d.normals_count = M.normals_count;
        d.uvs_count = M.uvs_count;
        d.height = M.bvh.height;
        memcpy(d.aabb, &M.bvh.nodes[0].aabb, sizeof(d.aabb));
        memcpy(d.mesh_aabb, &M.aabb, sizeof(d.mesh_aabb));
        S->mesh_host.push_back(d);
        ST_CUDA(cudaMemcpyAsync(P<Triangle>(S->tri_full) + tri_off, M.triangles, sizeof(Triangle) * M.triangle_count,
                                cudaMemcpyHostToDevice, ctx->stream));
        launch_make_trihot(P<Triangle>(S->tri_full) + tri_off, M.triangle_count, P<TriHot>(S->tri_hot) + tri_off, ctx->stream);
        if (M.bvh.node_count > 1) {
            // stage the nodes through the TLAS AABB scratch-free path: a temporary device copy
            BVHNode *tmp = nullptr;
            ST_CUDA(cudaMallocAsync((void **)&tmp, sizeof(BVHNode) * M.bvh.node_count, ctx->stream));
            ST_CUDA(cudaMemcpyAsync(tmp, M.bvh.nodes, sizeof(BVHNode) * M.bvh.node_count, cudaMemcpyHostToDevice, ctx->stream));
            launch_make_pairs(tmp, M.bvh.node_count, P<NodePair>(S->mesh_pairs) + pair_off, ctx->stream);
            ST_CUDA(cudaFreeAsync(tmp, ctx->stream));
        }
        // the nodes drawMeshAccelerationStructure (raytracer.h:33) outlines: depth <= 5, coloured
        // Magenta (leaf), Green (inner) or Blue (root)
        const u32t first_outline = (u32t)outlines.size();
        for (u32t k = 0; k < M.bvh.node_count; k++) {
            const BVHNode &nd = M.bvh.nodes[k];
            if (nd.depth > 5) continue;
            OutlineBox o;
            memcpy(o.aabb, &nd.aabb, sizeof(o.aabb));
            o.color = nd.child_count ? 7u : (k ? 4u : 5u);
            o.pad = 0;
            outlines.push_back(o);
        }
        S->outline_host.push_back(make_uint2(first_outline, (u32t)outlines.size() - first_outline));
        tri_off += M.triangle_count;
        pair_off += M.bvh.node_count > 1 ? (M.bvh.node_count - 1) / 2 : 0;
    }
    ST_TRY(reserve(ctx, S->outlines, sizeof(OutlineBox) * std::max<size_t>(outlines.size(), 1)));
    ST_TRY(reserve(ctx, S->outline_ranges, sizeof(uint2) * std::max<size_t>(S->outline_host.size(), 1)));
    if (!outlines.empty())
        ST_CUDA(cudaMemcpyAsync(S->outlines.ptr, outlines.data(), sizeof(OutlineBox) * outlines.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
    if (!S->outline_host.empty())
        ST_CUDA(cudaMemcpyAsync(S->outline_ranges.ptr, S->outline_host.data(), sizeof(uint2) * S->outline_host.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
    S->n_meshes = (u32t)S->mesh_host.size();
    if (S->n_meshes)
        ST_CUDA(cudaMemcpyAsync(S->meshes.ptr, S->mesh_host.data(), sizeof(MeshDev) * S->n_meshes, cudaMemcpyHostToDevice, ctx->stream));
    S->meshes_valid = true;
    return ST_CUDA_SYNC(ctx);
}

int st_update_primitives(st_ctx *ctx, int slot, const Primitive *primitives, const uint32_t *ids, uint32_t count) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !S->allocated || (count && (!primitives || !ids))) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (!count) return ST_OK;
    // ids must be in range and distinct (the last write to an id would otherwise be undefined)
    std::vector<uint8_t> seen(S->n_prims, 0);
    for (uint32_t k = 0; k < count; k++) {
        if (ids[k] >= S->n_prims || seen[ids[k]]) return ST_ERR_INVALID_ARG;
        seen[ids[k]] = 1;
    }
    // one copy of the records and ids, then a scatter kernel (not one copy per primitive)
    const size_t rec_bytes = sizeof(Primitive) * count, id_off = (rec_bytes + 255) & ~(size_t)255;
    ST_TRY(reserve(ctx, ctx->upd_host_dev, id_off + sizeof(u32t) * count));
    if (ctx->upd_pinned_cap < id_off + sizeof(u32t) * count) {
        if (ctx->upd_pinned) cudaFreeHost(ctx->upd_pinned);
        ctx->upd_pinned = nullptr;
        ctx->upd_pinned_cap = 0;
        const size_t cap = std::max(id_off + sizeof(u32t) * count, (size_t)1 << 20);
        ST_CUDA(cudaMallocHost((void **)&ctx->upd_pinned, cap));
        ctx->upd_pinned_cap = cap;
    }
    memcpy(ctx->upd_pinned, primitives, rec_bytes);
    memcpy(ctx->upd_pinned + id_off, ids, sizeof(u32t) * count);
    ST_CUDA(cudaMemcpyAsync(ctx->upd_host_dev.ptr, ctx->upd_pinned, id_off + sizeof(u32t) * count, cudaMemcpyHostToDevice,
                            ctx->stream));
    char *d = static_cast<char *>(ctx->upd_host_dev.ptr);
    launch_scatter_prims(reinterpret_cast<const Primitive *>(d), reinterpret_cast<const u32t *>(d + id_off), count,
                         P<Primitive>(S->prims_raw), P<PrimDev>(S->prims), ctx->stream);
    for (uint32_t k = 0; k < count; k++) S->prims_host[ids[k]] = primitives[k];
    return ST_CUDA_SYNC(ctx);
}

static int update_scene_bvh(st_ctx *ctx, SceneSlot *S, Scene *scene, int mode);

int st_update_scene_bvh(st_ctx *ctx, int slot, Scene *scene, int mode) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !S->allocated) return ST_ERR_NOT_RESIDENT;
    if (mode != ST_BVH_LBVH30 && mode != ST_BVH_BINNED_SAH && mode != ST_BVH_REFIT && mode != ST_BVH_REF_SAH)
        return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    const u32t n = S->n_prims;
    if (!n) return ST_ERR_BAD_SCENE;
    for (u32t i = 0; i < n; i++)
        if (S->prims_host[i].type == PrimitiveType_Mesh && (!S->meshes_valid || S->prims_host[i].id >= S->n_meshes))
            return ST_ERR_NOT_RESIDENT;
    // An update writes the node and leaf arrays (or the boxes) before it can check them: one that
    // fails part way leaves no TLAS that a render or a refit may use, until a later build succeeds.
    const int status = update_scene_bvh(ctx, S, scene, mode);
    if (status != ST_OK) S->tlas_valid = false;
    return status;
}

// An LBVH30 TLAS update waits once: the build's counts, its nodes (at most 2n - 1) and its leaf order
// come back together into page-locked staging, are checked there and, when the host scene has BVH
// arrays, copied into them from there (the other modes wait for the build, the check and the copy
// one after another).
static int update_scene_lbvh(st_ctx *ctx, SceneSlot *S, Scene *scene) {
    const u32t n = S->n_prims;
    cudaStream_t st = ctx->stream;
    if (lbvh_reserve(ctx->lbvh, n) != cudaSuccess) return ST_ERR_OUT_OF_MEMORY;
    const size_t node_bytes = sizeof(BVHNode) * 2 * (size_t)n, need = 64 + node_bytes + sizeof(u32t) * (size_t)n;
    if (need > ctx->bvh_pinned_cap) {
        if (ctx->bvh_pinned) cudaFreeHost(ctx->bvh_pinned);
        ctx->bvh_pinned = nullptr;
        ctx->bvh_pinned_cap = 0;
        ST_CUDA(cudaHostAlloc((void **)&ctx->bvh_pinned, need, cudaHostAllocDefault));
        ctx->bvh_pinned_cap = need;
    }
    u32t *counts = reinterpret_cast<u32t *>(ctx->bvh_pinned);
    BVHNode *nodes = reinterpret_cast<BVHNode *>(ctx->bvh_pinned + 64);
    u32t *ids = reinterpret_cast<u32t *>(ctx->bvh_pinned + 64 + node_bytes);
    launch_prim_aabbs(P<Primitive>(S->prims_raw), P<MeshDev>(S->meshes), n, ctx->lbvh.aabbs, st);
    lbvh_enqueue(ctx->lbvh, n, MAX_OBJS_PER_SCENE_BVH_NODE, P<BVHNode>(S->tlas_nodes), P<u32t>(S->tlas_leaf_ids),
                 counts, st);
    ST_CUDA(cudaGetLastError());
    ST_CUDA(cudaMemcpyAsync(nodes, S->tlas_nodes.ptr, node_bytes - sizeof(BVHNode), cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaMemcpyAsync(ids, S->tlas_leaf_ids.ptr, sizeof(u32t) * n, cudaMemcpyDeviceToHost, st));
    ST_TRY(ST_CUDA_SYNC(ctx));
    const u32t count = 1 + 2 * counts[2], height = counts[1];
    // the walk trusts every index it reads: check the new arrays before first use
    if (count > 2 * n - 1 || height + 2 > (u32t)kStack) return ST_ERR_BAD_SCENE;
    if (!check_bvh(nodes, count, n, height)) return ST_ERR_BAD_SCENE;
    for (u32t i = 0; i < n; i++) if (ids[i] >= n) return ST_ERR_BAD_SCENE;
    S->tlas_node_count = count;
    S->tlas_height = height;
    if (count > 1) {
        launch_make_pairs(P<BVHNode>(S->tlas_nodes), count, P<NodePair>(S->tlas_pairs), st);
        ST_CUDA(cudaGetLastError());
    }
    S->tlas_root = nodes[0];
    S->tlas_valid = true;
    S->moved_since_build = 0;
    if (scene && scene->bvh.nodes && scene->bvh.leaf_ids) {
        memcpy(scene->bvh.nodes, nodes, sizeof(BVHNode) * count);
        memcpy(scene->bvh.leaf_ids, ids, sizeof(u32t) * n);
        scene->bvh.node_count = count;
        scene->bvh.height = height;
    }
    return ST_OK;
}

static int update_scene_bvh(st_ctx *ctx, SceneSlot *S, Scene *scene, int mode) {
    const u32t n = S->n_prims;
    if (mode == ST_BVH_LBVH30) {
        return update_scene_lbvh(ctx, S, scene);
    } else if (mode == ST_BVH_BINNED_SAH) {
        if (lbvh_reserve(ctx->lbvh, n) != cudaSuccess) return ST_ERR_OUT_OF_MEMORY;
        launch_prim_aabbs(P<Primitive>(S->prims_raw), P<MeshDev>(S->meshes), n, ctx->lbvh.aabbs, ctx->stream);
        u32t info[2];
        ST_TRY(reserve(ctx, ctx->sah_scratch, sah_scratch_bytes(n)));
        cudaError_t e = sah_build(ctx->lbvh.aabbs, n, MAX_OBJS_PER_SCENE_BVH_NODE, P<BVHNode>(S->tlas_nodes),
                                  P<u32t>(S->tlas_leaf_ids), info, ctx->stream, ctx->sah_scratch.ptr, ctx->sah_scratch.bytes);
        if (e != cudaSuccess) return fail_cuda(ctx, e);
        S->tlas_node_count = info[0];
        S->tlas_height = info[1];
        if (S->tlas_height + 2 > (u32t)kStack) return ST_ERR_BAD_SCENE;
    } else if (mode == ST_BVH_REF_SAH) {
        if (lbvh_reserve(ctx->lbvh, n) != cudaSuccess) return ST_ERR_OUT_OF_MEMORY;
        launch_prim_aabbs(P<Primitive>(S->prims_raw), P<MeshDev>(S->meshes), n, ctx->lbvh.aabbs, ctx->stream);
        u32t info[2];
        cudaError_t e = refsah_build(ctx->lbvh.aabbs, n, MAX_OBJS_PER_SCENE_BVH_NODE, P<BVHNode>(S->tlas_nodes),
                                     P<u32t>(S->tlas_leaf_ids), info, ctx->stream);
        if (e != cudaSuccess) return fail_cuda(ctx, e);
        S->tlas_node_count = info[0];
        S->tlas_height = info[1];
    } else if (mode == ST_BVH_REFIT) {
        if (!S->tlas_valid) return ST_ERR_NOT_RESIDENT;
        launch_prim_aabbs(P<Primitive>(S->prims_raw), P<MeshDev>(S->meshes), n, P<float>(S->tlas_aabbs), ctx->stream);
        u32t *par = P<u32t>(S->tlas_scratch);
        u32t *arr = par + 2 * n;
        unsigned *box = reinterpret_cast<unsigned *>(arr + 2 * n);
        cudaError_t e = refit_bvh(P<BVHNode>(S->tlas_nodes), S->tlas_node_count, P<u32t>(S->tlas_leaf_ids),
                                  P<float>(S->tlas_aabbs), par, arr, box, ctx->stream);
        if (e != cudaSuccess) return fail_cuda(ctx, e);
    } else {
        return ST_ERR_INVALID_ARG;
    }
    // the walk trusts every index it reads: check a newly built array before first use (a refit
    // rewrites boxes only, so the topology checked when it was built still holds)
    if (mode != ST_BVH_REFIT) {
        std::vector<BVHNode> host(S->tlas_node_count);
        std::vector<u32t> ids(n);
        ST_CUDA(cudaMemcpyAsync(host.data(), S->tlas_nodes.ptr, sizeof(BVHNode) * host.size(), cudaMemcpyDeviceToHost, ctx->stream));
        ST_CUDA(cudaMemcpyAsync(ids.data(), S->tlas_leaf_ids.ptr, sizeof(u32t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        ST_TRY(ST_CUDA_SYNC(ctx));
        if (!check_bvh(host.data(), S->tlas_node_count, n, S->tlas_height)) return ST_ERR_BAD_SCENE;
        for (u32t i = 0; i < n; i++) if (ids[i] >= n) return ST_ERR_BAD_SCENE;
    }
    ST_TRY(finish_tlas(ctx, *S));
    if (mode != ST_BVH_REFIT) S->moved_since_build = 0;
    if (scene && scene->bvh.nodes && scene->bvh.leaf_ids) {
        ST_CUDA(cudaMemcpyAsync(scene->bvh.nodes, S->tlas_nodes.ptr, sizeof(BVHNode) * S->tlas_node_count, cudaMemcpyDeviceToHost, ctx->stream));
        ST_CUDA(cudaMemcpyAsync(scene->bvh.leaf_ids, S->tlas_leaf_ids.ptr, sizeof(u32t) * n, cudaMemcpyDeviceToHost, ctx->stream));
        ST_TRY(ST_CUDA_SYNC(ctx));
        scene->bvh.node_count = S->tlas_node_count;
        scene->bvh.height = S->tlas_height;
    }
    return ST_OK;
}

int st_update_mesh_bvh(st_ctx *ctx, Mesh *mesh, int mode) {
    if (!ctx || !mesh || !mesh->vertex_positions || !mesh->vertex_position_indices || !mesh->vertex_normals ||
        !mesh->vertex_normal_indices || !mesh->triangles || !mesh->bvh.nodes || !mesh->bvh.leaf_ids)
        return ST_ERR_INVALID_ARG;
    if (mode != ST_BVH_LBVH30 && mode != ST_BVH_BINNED_SAH) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    const u32t n = mesh->triangle_count;
    if (!n) return ST_ERR_BAD_SCENE;
    for (u32t i = 0; i < 3 * n; i++) {
        if (((const uint32_t *)mesh->vertex_position_indices)[i] >= mesh->vertex_count) return ST_ERR_BAD_SCENE;
        if (((const uint32_t *)mesh->vertex_normal_indices)[i] >= mesh->normals_count) return ST_ERR_BAD_SCENE;
        if (mesh->uvs_count && ((const uint32_t *)mesh->vertex_uvs_indices)[i] >= mesh->uvs_count) return ST_ERR_BAD_SCENE;
    }
    if (lbvh_reserve(ctx->lbvh, n) != cudaSuccess) return ST_ERR_OUT_OF_MEMORY;
    cudaStream_t st = ctx->stream;
    size_t bytes = sizeof(vec3) * (mesh->vertex_count + mesh->normals_count) + sizeof(vec2) * (mesh->uvs_count + 1) +
                   sizeof(uint32_t) * 9 * (size_t)n + sizeof(BVHNode) * 2 * (size_t)n + sizeof(u32t) * 2 * (size_t)n +
                   sizeof(Triangle) * (size_t)n + 256 * 8;
    if (ctx->in_use + bytes > ctx->budget) return ST_ERR_BUDGET;
    char *base = nullptr;
    ST_CUDA(cudaMallocAsync((void **)&base, bytes, st));
    char *cur = base;
    auto take = [&](size_t b) { char *p = cur; cur += (b + 255) & ~(size_t)255; return p; };
    vec3 *pos = (vec3 *)take(sizeof(vec3) * mesh->vertex_count);
    vec3 *nrm = (vec3 *)take(sizeof(vec3) * mesh->normals_count);
    vec2 *uv = (vec2 *)take(sizeof(vec2) * (mesh->uvs_count + 1));
    uint32_t *pidx = (uint32_t *)take(sizeof(uint32_t) * 3 * n);
    uint32_t *nidx = (uint32_t *)take(sizeof(uint32_t) * 3 * n);
    uint32_t *uidx = (uint32_t *)take(sizeof(uint32_t) * 3 * n);
    BVHNode *nodes = (BVHNode *)take(sizeof(BVHNode) * 2 * n);
    u32t *order = (u32t *)take(sizeof(u32t) * n);
    u32t *inverse = (u32t *)take(sizeof(u32t) * n);
    Triangle *tris = (Triangle *)take(sizeof(Triangle) * n);
    cudaMemcpyAsync(pos, mesh->vertex_positions, sizeof(vec3) * mesh->vertex_count, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(nrm, mesh->vertex_normals, sizeof(vec3) * mesh->normals_count, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(pidx, mesh->vertex_position_indices, sizeof(uint32_t) * 3 * n, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(nidx, mesh->vertex_normal_indices, sizeof(uint32_t) * 3 * n, cudaMemcpyHostToDevice, st);
    if (mesh->uvs_count) {
        cudaMemcpyAsync(uv, mesh->vertex_uvs, sizeof(vec2) * mesh->uvs_count, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(uidx, mesh->vertex_uvs_indices, sizeof(uint32_t) * 3 * n, cudaMemcpyHostToDevice, st);
    }
    launch_tri_aabbs(pos, pidx, n, ctx->lbvh.aabbs, st);
    u32t info[2];
    cudaError_t e = mode == ST_BVH_LBVH30
        ? lbvh_build(ctx->lbvh, n, MAX_TRIANGLES_PER_MESH_BVH_NODE, nodes, order, info, st)
        : sah_build(ctx->lbvh.aabbs, n, MAX_TRIANGLES_PER_MESH_BVH_NODE, nodes, order, info, st,
                    ctx->sah_scratch.ptr, ctx->sah_scratch.bytes);
    if (e == cudaSuccess) {
        launch_tri_records(pos, nrm, uv, pidx, nidx, uidx, mesh->uvs_count ? 1 : 0, order, n, tris, inverse, st);
        cudaMemcpyAsync(mesh->bvh.nodes, nodes, sizeof(BVHNode) * info[0], cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(mesh->bvh.leaf_ids, inverse, sizeof(u32t) * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(mesh->triangles, tris, sizeof(Triangle) * n, cudaMemcpyDeviceToHost, st);
        cudaFreeAsync(base, st);
        e = cudaStreamSynchronize(st);
    } else {
        cudaFreeAsync(base, st);
        cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    mesh->bvh.node_count = info[0];
    mesh->bvh.height = info[1];
    return ST_OK;
}

int st_build_bvh(st_ctx *ctx, int mode, const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *codes,
                 uint32_t *order, BVHNode *nodes, uint32_t info[2]) {
    if (!ctx || !aabbs || !nodes || !order || !info || n == 0 || max_leaf == 0 || max_leaf > 0xFFFF ||
        (mode != ST_BVH_LBVH30 && mode != ST_BVH_BINNED_SAH && mode != ST_BVH_REF_SAH))
        return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (lbvh_reserve(ctx->lbvh, n) != cudaSuccess) return ST_ERR_OUT_OF_MEMORY;
    cudaStream_t st = ctx->stream;
    char *base = nullptr;
    const size_t bytes = sizeof(BVHNode) * 2 * (size_t)n + sizeof(u32t) * 2 * (size_t)n + 512;
    if (ctx->in_use + bytes > ctx->budget) return ST_ERR_BUDGET;
    ST_CUDA(cudaMallocAsync((void **)&base, bytes, st));
    BVHNode *d_nodes = (BVHNode *)base;
    u32t *d_order = (u32t *)(base + ((sizeof(BVHNode) * 2 * (size_t)n + 255) & ~(size_t)255));
    u32t *d_codes = d_order + n;
    cudaMemcpyAsync(ctx->lbvh.aabbs, aabbs, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice, st);
    u32t inf[2];
    cudaError_t e = mode == ST_BVH_LBVH30     ? lbvh_build(ctx->lbvh, n, max_leaf, d_nodes, d_order, inf, st)
                    : mode == ST_BVH_REF_SAH ? refsah_build(ctx->lbvh.aabbs, n, max_leaf, d_nodes, d_order, inf, st)
                                             : sah_build(ctx->lbvh.aabbs, n, max_leaf, d_nodes, d_order, inf, st,
                                                         ctx->sah_scratch.ptr, ctx->sah_scratch.bytes);
    if (e == cudaSuccess) {
        if (mode == ST_BVH_LBVH30) launch_codes_by_item(ctx->lbvh, n, d_codes, st);
        else codes = nullptr;
        cudaMemcpyAsync(nodes, d_nodes, sizeof(BVHNode) * inf[0], cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(order, d_order, sizeof(u32t) * n, cudaMemcpyDeviceToHost, st);
        if (codes) cudaMemcpyAsync(codes, d_codes, sizeof(u32t) * n, cudaMemcpyDeviceToHost, st);
        e = cudaStreamSynchronize(st);
    }
    cudaFreeAsync(base, st);
    cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    info[0] = inf[0];
    info[1] = inf[1];
    return ST_OK;
}

// ---- render ------------------------------------------------------------------------------------
static int make_view(const Viewport *vp, ViewDev &v) {
    if (!vp || !vp->camera || !vp->frame_buffer) return ST_ERR_INVALID_ARG;
    const Camera &cam = *vp->camera;
    const Dimensions &d = vp->frame_buffer->dimensions;
    if (d.width < 2 || d.height < 2) return ST_ERR_INVALID_ARG;
    v.cam_pos = {cam.transform.position.x, cam.transform.position.y, cam.transform.position.z};
    v.cam_rot_inv.axis = {cam.transform.rotation_inverted.axis.x, cam.transform.rotation_inverted.axis.y,
                          cam.transform.rotation_inverted.axis.z};
    v.cam_rot_inv.w = cam.transform.rotation_inverted.amount;
    memcpy(v.cam_rot_matrix_inv, &cam.transform.rotation_matrix_inverted, sizeof(v.cam_rot_matrix_inv));
    v.focal_length = cam.focal_length;
    const ProjectionPlane &pp = vp->projection_plane;
    v.pp_start = {pp.start.x, pp.start.y, pp.start.z};
    v.pp_right = {pp.right.x, pp.right.y, pp.right.z};
    v.pp_down = {pp.down.x, pp.down.y, pp.down.z};
    v.cone_angle = pp.cone_angle;
    v.grid_w = d.width;
    v.grid_h = d.height;
    v.f_width = d.f_width;
    v.f_height = d.f_height;
    v.h_width = d.h_width;
    v.h_height = d.h_height;
    v.width_over_height = d.width_over_height;
    v.height_over_width = d.height_over_width;
    v.mode = vp->settings.render_mode;
    v.depth = vp->trace.depth;
    v.primary_tlas = 0;
    return ST_OK;
}

// The device address of a page-locked (pinned or registered) host buffer, or null for pageable
// memory, which the device cannot write.
static void *device_view_of_host(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

static SceneDev scene_view(SceneSlot &S, const Scene *scene) {
    SceneDev d;
    d.prims = P<PrimDev>(S.prims);
    d.prims_raw = P<Primitive>(S.prims_raw);
    d.n_prims = S.n_prims;
    d.materials = P<Material>(S.materials);
    const bool lights = scene ? (scene->lights != nullptr && scene->settings.lights) : S.lights_present;
    d.lights = lights ? P<Light>(S.lights) : nullptr;
    d.n_lights = lights ? S.n_lights : 0;
    d.ambient = scene ? scene->ambient_light.color : S.ambient;
    d.tlas_pairs = P<NodePair>(S.tlas_pairs);
    d.tlas_leaf_ids = P<u32t>(S.tlas_leaf_ids);
    d.tlas_root_count = S.tlas_root.child_count;
    d.tlas_root_first = S.tlas_root.first_child_id;
    memcpy(d.tlas_root_aabb, &S.tlas_root.aabb, sizeof(d.tlas_root_aabb));
    d.meshes = P<MeshDev>(S.meshes);
    d.mesh_pairs = P<NodePair>(S.mesh_pairs);
    d.tri_hot = P<TriHot>(S.tri_hot);
    d.tri_full = P<Triangle>(S.tri_full);
    d.textures = P<TexDev>(S.textures);
    d.mips = P<MipDev>(S.mips);
    d.quads = P<TexelQuad>(S.quads);
    d.emissive_quads = P<u32t>(S.emissive);
    d.n_emissive = S.n_emissive;
    d.occluders = P<u32t>(S.occluders);
    d.n_occluders = S.n_occluders;
    return d;
}

// drawBVH (raytracer.h:46) and drawSSB (SSB.h:175) over the traced grid: the scene's device TLAS,
// primitives and outlined BLAS nodes, the SSB of this render (ctx->ssb), the viewport's projection
// matrix and clipping planes.
static int draw_overlays(st_ctx *ctx, SceneSlot &S, const Viewport *vp, const ViewDev &v, int what, FloatPixel *grid,
                         FloatPixel *grid_host, cudaStream_t st) {
    OverlayParams op;
    memset(&op, 0, sizeof(op));
    const bool bvh = (what & ST_OVERLAY_BVH) != 0;
    op.nodes = P<BVHNode>(S.tlas_nodes);
    op.node_count = bvh ? S.tlas_node_count : 0;
    op.leaf_ids = P<u32t>(S.tlas_leaf_ids);
    op.prims = P<Primitive>(S.prims_raw);
    op.n_prims = (what & ST_OVERLAY_SSB) ? S.n_prims : 0;
    op.outlines = P<OutlineBox>(S.outlines);
    op.outline_range = P<uint2>(S.outline_ranges);
    op.n_meshes = (u32t)S.outline_host.size();
    op.cam_pos = v.cam_pos;
    op.cam_rot_inv = v.cam_rot_inv;
    memcpy(op.proj, &vp->projection_matrix, sizeof(op.proj));
    op.near_plane = vp->settings.near_clipping_plane_distance;
    op.far_plane = vp->settings.far_clipping_plane_distance;
    op.focal_length = v.focal_length;
    const Dimensions &d = vp->frame_buffer->dimensions;
    op.width_over_height = d.width_over_height;
    op.h_width = d.h_width;
    op.h_height = d.h_height;
    op.f_height = d.f_height;
    op.width = d.width;
    op.height = d.height;
    op.stride = d.width;
    op.pos_x = vp->position.x;
    op.pos_y = vp->position.y;
    op.grid_pixels = v.grid_w * v.grid_h;
    // boxes drawBVH draws: one per node, one per implicit primitive, the outlines of each mesh
    // instance (every primitive sits in exactly one leaf of a valid TLAS)
    u32t n_boxes = 0;
    if (bvh) {
        n_boxes = S.tlas_node_count;
        for (const Primitive &p : S.prims_host) {
            if (p.type == PrimitiveType_Mesh) n_boxes += p.id < S.outline_host.size() ? S.outline_host[p.id].y : 0;
            else if (p.type == PrimitiveType_Box || p.type == PrimitiveType_Quad || p.type == PrimitiveType_Sphere ||
                     p.type == PrimitiveType_Tetrahedron)
                n_boxes += 1;
        }
    }
    ST_TRY(reserve(ctx, ctx->overlay_scratch, overlay_scratch_bytes(op, n_boxes)));
    u32t n_frags = 0;
    ST_CUDA(overlay_count(op, P<int4>(ctx->ssb), n_boxes, ctx->overlay_scratch.ptr, &n_frags, st));
    if (!n_frags) return ST_OK;
    ST_TRY(reserve(ctx, ctx->overlay_frags, overlay_fragment_bytes(n_frags)));
    ST_CUDA(overlay_draw(op, P<int4>(ctx->ssb), n_boxes, ctx->overlay_scratch.ptr, n_frags, ctx->overlay_frags.ptr, grid,
                         grid_host, st));
    return ST_OK;
}

// The strips' streams get priorities falling with the strip's position, so that the block
// scheduler starts a strip's blocks before the next strip's and the strips finish left to right,
// each early enough for its copy to overlap the strips still being traced.
static cudaError_t ensure_strips(st_ctx *ctx) {
    cudaError_t e = cudaSuccess;
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (int k = 0; k < kRenderStrips && e == cudaSuccess; k++) {
        const int prio = greatest + (int)((long)(least - greatest) * k / (kRenderStrips - 1));
        if (!ctx->strip_trace[k]) e = cudaStreamCreateWithPriority(&ctx->strip_trace[k], cudaStreamNonBlocking, prio);
    }
    // the resolves go ahead of the trace blocks still waiting to start
    if (e == cudaSuccess && !ctx->strip_resolve)
        e = cudaStreamCreateWithPriority(&ctx->strip_resolve, cudaStreamNonBlocking, greatest);
    for (cudaEvent_t &ev : ctx->strip_ev)
        if (e == cudaSuccess && !ev) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    return e;
}

int st_render_ex(st_ctx *ctx, int slot, const Scene *scene, const Viewport *viewport, st_render_options *o) {
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !viewport) return ST_ERR_INVALID_ARG;
    if (!S->allocated || !S->tlas_valid || !S->n_prims) return ST_ERR_NOT_RESIDENT;
    for (const Primitive &p : S->prims_host)
        if (p.type == PrimitiveType_Mesh && !S->meshes_valid) return ST_ERR_NOT_RESIDENT;
    cudaSetDevice(ctx->device);
    ViewDev v;
    ST_TRY(make_view(viewport, v));
    v.primary_tlas = S->n_prims > 64 ? 1 : 0;
    st_render_options defaults;
    memset(&defaults, 0, sizeof(defaults));
    if (!o) o = &defaults;
    cudaStream_t st = o->stream ? (cudaStream_t)o->stream : ctx->stream;
    const size_t grid = (size_t)v.grid_w * v.grid_h;
    const u32t W = v.grid_w - 1, H = v.grid_h - 1;
    ST_TRY(reserve(ctx, ctx->ssb, sizeof(int4) * std::max(S->n_prims, 1u)));
    ST_TRY(reserve(ctx, ctx->dirs, sizeof(float) * ray_rows_floats(v)));
    FloatPixel *host_float = o->out_float ? o->out_float : viewport->frame_buffer->float_pixels;
    Pixel *host_u8 = o->out_u8 ? o->out_u8 : viewport->frame_buffer->pixels;
    FloatPixel *dev_float;
    uint32_t *dev_u8 = nullptr;
    u32t *dev_ids = nullptr;
    if (o->device_outputs) {
        dev_float = o->out_float;
        dev_u8 = reinterpret_cast<uint32_t *>(o->out_u8);
        dev_ids = o->out_prim_id;
        if (!dev_float) {
            ST_TRY(reserve(ctx, ctx->out_float, sizeof(FloatPixel) * grid));
            dev_float = P<FloatPixel>(ctx->out_float);
        }
    } else {
        ST_TRY(reserve(ctx, ctx->out_float, sizeof(FloatPixel) * grid));
        dev_float = P<FloatPixel>(ctx->out_float);
        if (host_u8) {
            ST_TRY(reserve(ctx, ctx->out_u8, sizeof(uint32_t) * (size_t)W * H));
            dev_u8 = P<uint32_t>(ctx->out_u8);
        }
        if (o->out_prim_id) {
            ST_TRY(reserve(ctx, ctx->prim_ids, sizeof(u32t) * grid));
            dev_ids = P<u32t>(ctx->prim_ids);
        }
    }
    SceneDev sd = scene_view(*S, scene);
    ST_CUDA(cudaMemsetAsync(ctx->status.ptr, 0, 16, st));
    if (o->count_work) ST_CUDA(cudaMemsetAsync(ctx->counters.ptr, 0, sizeof(unsigned long long) * 16, st));
    ST_CUDA(cudaEventRecord(ctx->ev[0], st));
    launch_ssb(sd, v, P<int4>(ctx->ssb), st);
    launch_ray_rows(v, P<float>(ctx->dirs), st);
    // Host outputs.  A page-locked frame (pinned or registered) is written by the resolve kernel
    // itself; a page-locked float grid is traced in column strips, one stream per strip, and each
    // strip's columns are copied to the host by a 2-D DMA copy on its own stream, and its pixels
    // resolved on the resolve stream, as soon as it is traced, so that only the last strip's copy
    // and resolve follow the trace.  Pageable buffers receive one copy at the end.
    const bool host_out = !o->device_outputs;
    const bool want_float = host_out && host_float && !o->skip_float_copy;
    uint32_t *mapped_u8 = host_out && host_u8 && dev_u8 ? static_cast<uint32_t *>(device_view_of_host(host_u8)) : nullptr;
    const bool float_pinned = want_float && device_view_of_host(host_float) != nullptr;
    const bool overlays = (o->overlays & (ST_OVERLAY_BVH | ST_OVERLAY_SSB)) != 0;
    const u32t bw = (v.grid_w + 7) / 8;
    const int strips = (host_out && !overlays && (!want_float || float_pinned))
                           ? (int)std::max(1u, std::min((u32t)kRenderStrips, bw / 24)) : 1;
    uint32_t *u8_target = mapped_u8 ? mapped_u8 : dev_u8;
    ST_CUDA(cudaEventRecord(ctx->ev[1], st));
    if (strips > 1) {
        ST_CUDA(ensure_strips(ctx));
        cudaEvent_t *done = ctx->strip_ev, *joined = ctx->strip_ev + kRenderStrips;   // per strip
        cudaEvent_t fork = ctx->strip_ev[2 * kRenderStrips], resolved_ev = ctx->strip_ev[2 * kRenderStrips + 1];
        ST_CUDA(cudaEventRecord(fork, st));
        const size_t pitch = sizeof(FloatPixel) * v.grid_w;
        auto strip_cols = [&](int k, u32t &gx0, u32t &gx1) {
            gx0 = (u32t)((uint64_t)bw * k / strips) * 8;
            gx1 = std::min((u32t)((uint64_t)bw * (k + 1) / strips) * 8, v.grid_w);
        };
        // every trace is launched before any copy, so that a stream which shares a hardware queue
        // with another never holds that stream's trace behind its own copy
        for (int k = 0; k < strips; k++) {
            u32t gx0, gx1;
            strip_cols(k, gx0, gx1);
            cudaStream_t ts = ctx->strip_trace[k];
            ST_CUDA(cudaStreamWaitEvent(ts, fork, 0));
            launch_trace(sd, v, P<int4>(ctx->ssb), P<float>(ctx->dirs), dev_float, dev_ids, P<unsigned>(ctx->status),
                         P<unsigned long long>(ctx->counters), o->count_work != 0, ts, gx0 / 8, (gx1 - gx0 + 7) / 8,
                         want_float);
            ST_CUDA(cudaGetLastError());
            ST_CUDA(cudaEventRecord(done[k], ts));
        }
        // each strip's columns are copied behind its own trace, whatever order the strips end in;
        // the resolve stream takes the strips in order: pixel x reads grid columns x and x + 1, so a
        // strip's pixels [gx0 - 1, gx1 - 1) are resolved once it and the strips left of it are
        // traced, on their own stream so that the last strip's resolve overlaps its copy
        for (int k = 0; k < strips; k++) {
            u32t gx0, gx1;
            strip_cols(k, gx0, gx1);
            cudaStream_t ts = ctx->strip_trace[k];
            if (want_float)
                ST_CUDA(cudaMemcpy2DAsync(host_float + gx0, pitch, dev_float + gx0, pitch, sizeof(FloatPixel) * (gx1 - gx0),
                                          v.grid_h, cudaMemcpyDeviceToHost, ts));
            ST_CUDA(cudaEventRecord(joined[k], ts));
            if (u8_target) {
                ST_CUDA(cudaStreamWaitEvent(ctx->strip_resolve, done[k], 0));
                launch_resolve(dev_float, v.grid_w, W, H, u8_target, ctx->strip_resolve, k > 0 ? gx0 - 1 : 0,
                               k + 1 == strips ? W : gx1 - 1);
            }
        }
        for (int k = 0; k < strips; k++) ST_CUDA(cudaStreamWaitEvent(st, done[k], 0));
        ST_CUDA(cudaEventRecord(ctx->ev[2], st));
        for (int k = 0; k < strips; k++) ST_CUDA(cudaStreamWaitEvent(st, joined[k], 0));
        if (u8_target) {
            ST_CUDA(cudaEventRecord(resolved_ev, ctx->strip_resolve));
            ST_CUDA(cudaStreamWaitEvent(st, resolved_ev, 0));
        }
    } else {
        launch_trace(sd, v, P<int4>(ctx->ssb), P<float>(ctx->dirs), dev_float, dev_ids, P<unsigned>(ctx->status),
                     P<unsigned long long>(ctx->counters), o->count_work != 0, st);
        ST_CUDA(cudaGetLastError());
        ST_CUDA(cudaEventRecord(ctx->ev[2], st));
        if (overlays) ST_TRY(draw_overlays(ctx, *S, viewport, v, o->overlays, dev_float, nullptr, st));
        if (u8_target) launch_resolve(dev_float, v.grid_w, W, H, u8_target, st);
        if (want_float)
            ST_CUDA(cudaMemcpyAsync(host_float, dev_float, sizeof(FloatPixel) * grid, cudaMemcpyDeviceToHost, st));
    }
    ST_CUDA(cudaEventRecord(ctx->ev[3], st));
    if (host_out) {
        if (host_u8 && dev_u8 && !mapped_u8)
            ST_CUDA(cudaMemcpyAsync(host_u8, dev_u8, sizeof(uint32_t) * (size_t)W * H, cudaMemcpyDeviceToHost, st));
        if (o->out_prim_id)
            ST_CUDA(cudaMemcpyAsync(o->out_prim_id, dev_ids, sizeof(u32t) * grid, cudaMemcpyDeviceToHost, st));
    }
    unsigned *status = reinterpret_cast<unsigned *>(ctx->readback + 16);
    unsigned long long *c = ctx->readback;
    ST_CUDA(cudaMemcpyAsync(status, ctx->status.ptr, 16, cudaMemcpyDeviceToHost, st));
    if (o->count_work) ST_CUDA(cudaMemcpyAsync(c, ctx->counters.ptr, sizeof(unsigned long long) * 16, cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaStreamSynchronize(st));
    if (o->count_work)
        for (int k = 0; k < 16; k++) o->counters[k] = k < C_COUNT ? c[k] : 0;
    cudaEventElapsedTime(&o->trace_ms, ctx->ev[1], ctx->ev[2]);
    cudaEventElapsedTime(&o->total_ms, ctx->ev[0], ctx->ev[3]);
    if (status[0] & S_STACK_OVERFLOW) return ST_ERR_STACK_OVERFLOW;
    return ST_OK;
}

// ---- batched views ---------------------------------------------------------------------------
namespace {

struct BatchPlan {
    std::vector<BatchView> table;
    std::vector<size_t> ssb_off, seg_off, float_off, u8_off;   // element offsets into the batch arena
    std::vector<bool> want_u8;
    size_t ssb_total = 0, seg_total = 0, float_total = 0, u8_total = 0;
    u32t total_tiles = 0;
    uint64_t rays = 0;
    std::string shape_key, class_key;
};

// A view's tiles are numbered in groups of four warp tiles (group_tiles_w across), groups down
// the view's columns, so that the four warps of a block, which take one group, trace one compact
// region as the per-frame kernel's blocks do.  Sets b.groups_y and returns the number of tile
// slots (4 per group; slots of a group that fall outside the view have no grid points).
u32t view_tiles(BatchView &b, u32t tw, u32t th) {
    const u32t gw = group_tiles_w((int)tw), gh = 4 / gw;
    const u32t tx = (b.view.grid_w + tw - 1) / tw, ty = (b.view.grid_h + th - 1) / th;
    b.groups_y = (ty + gh - 1) / gh;
    return 4 * ((tx + gw - 1) / gw) * b.groups_y;
}

int plan_batch(st_ctx *ctx, const st_view *views, int n, int tile, const st_batch_options &o, BatchPlan &p) {
    u32t tw, th;
    tile_dims(tile, tw, th);
    p = BatchPlan();
    std::ostringstream shape, cls;
    shape << "t" << tile << "n" << n;
    for (int i = 0; i < n; i++) {
        const st_view &V = views[i];
        SceneSlot *S = slot_of(ctx, V.slot);
        if (!S || !V.viewport) return ST_ERR_INVALID_ARG;
        if (!S->allocated || !S->tlas_valid || !S->n_prims) return ST_ERR_NOT_RESIDENT;
        BatchView b;
        memset(&b, 0, sizeof(b));
        ST_TRY(make_view(V.viewport, b.view));
        b.view.primary_tlas = S->n_prims > 64 ? 1 : 0;
        b.scene = scene_view(*S, V.scene);
        b.tile_begin = p.total_tiles;
        p.total_tiles += view_tiles(b, tw, th);
        const size_t grid = (size_t)b.view.grid_w * b.view.grid_h;
        p.ssb_off.push_back(p.ssb_total);
        p.ssb_total += std::max(S->n_prims, 1u);
        p.seg_off.push_back(p.seg_total);
        p.seg_total += ray_rows_floats(b.view);
        p.float_off.push_back(p.float_total);
        if (!(o.device_outputs && V.out_float)) p.float_total += grid;
        const bool u8 = V.out_u8 != nullptr;
        p.want_u8.push_back(u8);
        p.u8_off.push_back(p.u8_total);
        if (u8 && !o.device_outputs) p.u8_total += (size_t)(b.view.grid_w - 1) * (b.view.grid_h - 1);
        p.rays += grid;
        p.table.push_back(b);
        shape << "_" << V.slot << ":" << b.view.grid_w << "x" << b.view.grid_h << "m" << b.view.mode << "d"
              << b.view.depth << "u" << (V.out_u8 != nullptr);
        // device outputs are baked into the captured launches; host outputs are copied after them
        if (o.device_outputs) shape << "o" << (const void *)V.out_float << "/" << (const void *)V.out_u8;
        // the scene class: primitive and triangle counts (log2 buckets) and the bounce count
        u32t tris = 0;
        for (const MeshDev &m : S->mesh_host) tris += m.triangle_count;
        int pb = 0, tb = 0;
        for (u32t x = S->n_prims; x > 1; x >>= 1) pb++;
        for (u32t x = tris; x > 1; x >>= 1) tb++;
        cls << "p" << pb << "t" << tb << "d" << b.view.depth << ";";
    }
    p.shape_key = shape.str();
    p.class_key = cls.str();
    return ST_OK;
}

// A batch's launches, kTableViews views at a time: the views' SSBs and ray-row starts, the trace
// (the persistent kernel over the group's tiles, or with kPerViewVariant one trace kernel per view
// spread over the batch's aux streams), and the resolves of the views that want a frame.  The
// set-up and resolve launches carry the group's view table as their kernel parameter.
int launch_groups(st_ctx *ctx, BatchState &B, const BatchPlan &p, int tile, u32t chunk, u32t threshold,
                  unsigned *status, cudaStream_t st) {
    const int n = (int)p.table.size();
    if (tile == kPerViewVariant) {
        // one per-frame trace kernel per view, the views spread over the auxiliary streams (the
        // kernels run side by side wherever one leaves SMs idle), between the set-up and the resolves
        for (int g0 = 0; g0 < n; g0 += kTableViews) {
            const int gn = std::min(kTableViews, n - g0);
            u32t max_prims = 0, max_rows = 0, max_w = 0, max_h = 0;
            for (int i = 0; i < gn; i++) {
                const BatchView &b = p.table[g0 + i];
                B.host_table.v[i] = b;
                max_prims = std::max(max_prims, b.scene.n_prims);
                max_rows = std::max(max_rows, b.view.grid_h);
                if (b.out_u8) {
                    max_w = std::max(max_w, b.view.grid_w - 1);
                    max_h = std::max(max_h, b.view.grid_h - 1);
                }
            }
            launch_batch_setup(B.host_table, (u32t)gn, max_prims, max_rows, st);
            ST_CUDA(ensure_aux(B));
            ST_CUDA(cudaEventRecord(B.fork_ev, st));
            const int streams = std::min(gn, kAuxStreams);
            for (int k = 0; k < streams; k++) ST_CUDA(cudaStreamWaitEvent(B.aux[k], B.fork_ev, 0));
            for (int i = 0; i < gn; i++) {
                const BatchView &b = B.host_table.v[i];
                launch_trace(b.scene, b.view, b.ssb, b.dirs, b.out, nullptr, status, P<unsigned long long>(ctx->counters),
                             false, B.aux[i % streams]);
            }
            for (int k = 0; k < streams; k++) {
                ST_CUDA(cudaEventRecord(B.join_ev[k], B.aux[k]));
                ST_CUDA(cudaStreamWaitEvent(st, B.join_ev[k], 0));
            }
            if (max_w) launch_batch_resolve(B.host_table, (u32t)gn, max_w, max_h, st);
        }
        return ST_CUDA_LAST();
    }
    const u32t blocks = (u32t)(ctx->sm_count * ctx->blocks_per_sm[tile]);
    // the device copy of the table, tile numbers rebased per group, for the trace kernel
    for (int i = 0; i < n; i++) {
        B.staging[i] = p.table[i];
        B.staging[i].tile_begin -= p.table[i - i % kTableViews].tile_begin;
    }
    ST_CUDA(cudaMemcpyAsync(B.table.ptr, B.staging, sizeof(BatchView) * n, cudaMemcpyHostToDevice, st));
    for (int g0 = 0; g0 < n; g0 += kTableViews) {
        const int gn = std::min(kTableViews, n - g0);
        const u32t first = p.table[g0].tile_begin;
        const u32t end = g0 + gn < n ? p.table[g0 + gn].tile_begin : p.total_tiles;
        u32t max_prims = 0, max_rows = 0, max_w = 0, max_h = 0;
        for (int i = 0; i < gn; i++) {
            const BatchView &b = B.staging[g0 + i];
            B.host_table.v[i] = b;
            max_prims = std::max(max_prims, b.scene.n_prims);
            max_rows = std::max(max_rows, b.view.grid_h);
            if (b.out_u8) {
                max_w = std::max(max_w, b.view.grid_w - 1);
                max_h = std::max(max_h, b.view.grid_h - 1);
            }
        }
        // the tile counter, and the parked-ray queue's reserved and drained counts
        ST_CUDA(cudaMemsetAsync(B.counter.ptr, 0, 16, st));
        ParkQueue park;
        if (threshold) {
            park.rays = P<ParkedRay>(B.park);
            park.reserved = P<u32t>(B.counter) + 1;
            park.taken = P<u32t>(B.counter) + 2;
            park.drained = P<u32t>(B.counter) + 4;
            park.capacity = (u32t)(B.park.bytes / sizeof(ParkedRay));
            park.threshold = threshold;
        }
        launch_batch_setup(B.host_table, (u32t)gn, max_prims, max_rows, st);
        if (launch_batch(P<BatchView>(B.table) + g0, (u32t)gn, end - first, tile, chunk, blocks, P<u32t>(B.counter),
                         status, P<unsigned long long>(ctx->counters), false, st, park) != 0)
            return ST_ERR_INVALID_ARG;
        if (threshold &&
            launch_drain(P<BatchView>(B.table) + g0, park, tile, blocks, status, P<unsigned long long>(ctx->counters),
                         false, st) != 0)
            return ST_ERR_INVALID_ARG;
        if (max_w) launch_batch_resolve(B.host_table, (u32t)gn, max_w, max_h, st);
    }
    return ST_CUDA_LAST();
}

int enqueue_batch(st_ctx *ctx, BatchState &B, unsigned *status, const st_view *views, int n, BatchPlan &p, int tile,
                  u32t chunk, u32t threshold, cudaStream_t st, const st_batch_options &o) {
    // per-view pointers into the arena (or the caller's device outputs)
    for (int i = 0; i < n; i++) {
        BatchView &b = p.table[i];
        b.ssb = P<int4>(B.ssb) + p.ssb_off[i];
        b.dirs = P<float>(B.seg) + p.seg_off[i];
        b.out = (o.device_outputs && views[i].out_float) ? views[i].out_float : P<FloatPixel>(B.out_float) + p.float_off[i];
        b.prim_ids = nullptr;
        b.out_u8 = !p.want_u8[i] ? nullptr
                   : o.device_outputs ? reinterpret_cast<uint32_t *>(views[i].out_u8) : P<uint32_t>(B.out_u8) + p.u8_off[i];
    }
    ST_CUDA(cudaMemsetAsync(status, 0, 16, st));
    ST_CUDA(cudaMemsetAsync(P<u32t>(B.counter) + 4, 0, 4, st));   // the batch's parked-path total
    return launch_groups(ctx, B, p, tile, chunk, threshold, status, st);
}

// Device and pinned room for n views' table (grown geometrically: cudaFreeHost waits for the device).
int table_reserve(st_ctx *ctx, BatchState &B, int n) {
    ST_TRY(reserve(ctx, B.table, sizeof(BatchView) * n));
    if (B.staging_cap < (size_t)n) {
        const size_t cap = std::max((size_t)n, 2 * B.staging_cap);
        if (B.staging) cudaFreeHost(B.staging);
        B.staging = nullptr;
        B.staging_cap = 0;
        ST_CUDA(cudaMallocHost((void **)&B.staging, sizeof(BatchView) * cap));
        B.staging_cap = cap;
    }
    return ST_OK;
}

int batch_reserve(st_ctx *ctx, BatchState &B, const BatchPlan &p, int n, u32t threshold) {
    ST_TRY(table_reserve(ctx, B, n));
    // the parked-ray queue: room for every ray of the batch, at most kParkCapacity (a launch group's
    // parks beyond it are traced in place)
    if (threshold) ST_TRY(reserve(ctx, B.park, sizeof(ParkedRay) * (size_t)std::min<uint64_t>(p.rays, kParkCapacity)));
    ST_TRY(reserve(ctx, B.ssb, sizeof(int4) * p.ssb_total));
    ST_TRY(reserve(ctx, B.seg, sizeof(float) * p.seg_total));
    ST_TRY(reserve(ctx, B.out_float, sizeof(FloatPixel) * std::max(p.float_total, (size_t)1)));
    ST_TRY(reserve(ctx, B.out_u8, sizeof(uint32_t) * std::max(p.u8_total, (size_t)1)));
    ST_TRY(reserve(ctx, B.counter, 32));     // per group: tile counter, queue counts; then the parked total
    return ST_OK;
}

}  // namespace

// One autotuning trial: the batch run twice with one kernel variant, chunk and compaction threshold,
// the faster device time kept (the first run also absorbs one-time costs such as the per-view
// streams' creation).
static int time_batch(st_ctx *ctx, BatchState &B, const st_view *views, int n, int variant, u32t chunk, u32t threshold,
                      cudaStream_t st, const st_batch_options &o, float &best_ms) {
    BatchPlan q;
    ST_TRY(plan_batch(ctx, views, n, variant, o, q));
    ST_TRY(batch_reserve(ctx, B, q, n, threshold));
    if (variant == kPerViewVariant) ST_CUDA(ensure_aux(B));
    best_ms = INFINITY;
    for (int rep = 0; rep < 2; rep++) {
        ST_CUDA(cudaEventRecord(ctx->ev[0], st));
        ST_TRY(enqueue_batch(ctx, B, P<unsigned>(ctx->status), views, n, q, variant, chunk, threshold, st, o));
        ST_CUDA(cudaEventRecord(ctx->ev[1], st));
        ST_CUDA(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        best_ms = std::min(best_ms, ms);
    }
    return ST_OK;
}

int st_render_batch(st_ctx *ctx, const st_view *views, int n, st_batch_options *opt) {
    if (!ctx || !views || n <= 0) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    st_batch_options dflt;
    memset(&dflt, 0, sizeof(dflt));
    dflt.tile_shape = -1;
    dflt.stack_placement = -1;
    dflt.launch_mode = ST_LAUNCH_AUTOTUNED;
    dflt.compaction_threshold = -1;
    st_batch_options &o = opt ? *opt : dflt;
    cudaStream_t st = o.stream ? (cudaStream_t)o.stream : ctx->stream;
    BatchState &B = ctx->batch;
    // the kernel variant (tile shape, stack placement) and queue chunk: given, cached for this scene
    // class, or tuned now
    if (o.tile_shape >= TILE_SHAPES || o.stack_placement >= STACK_PLACEMENTS || o.launch_mode < ST_LAUNCH_AUTOTUNED ||
        o.launch_mode > ST_LAUNCH_PERSISTENT || o.compaction_threshold < -1 || o.compaction_threshold > 32)
        return ST_ERR_INVALID_ARG;
    BatchPlan p;
    // one kernel per view has no tile shape, stack placement or chunk to choose; the persistent kernel
    // with every knob given needs no tuning; otherwise the choice is cached per scene class or tuned
    const bool fixed_tile = o.tile_shape >= 0 || o.stack_placement >= 0;
    int tile = o.launch_mode == ST_LAUNCH_PER_VIEW ? kPerViewVariant
               : (o.tile_shape >= 0 && o.stack_placement >= 0) ? o.tile_shape + TILE_SHAPES * o.stack_placement : -1;
    u32t chunk = o.launch_mode == ST_LAUNCH_PER_VIEW ? 1u : o.chunk > 0 ? (u32t)o.chunk : 0;
    // the warp-vote compaction threshold applies to the persistent kernel only
    int threshold = o.launch_mode == ST_LAUNCH_PER_VIEW ? 0 : o.compaction_threshold;
    ST_TRY(plan_batch(ctx, views, n, o.tile_shape >= 0 ? o.tile_shape : 0, o, p));
    if (tile < 0 || chunk == 0 || threshold < 0) {
        auto it = B.tuned.find(p.class_key);
        const bool per_view = it != B.tuned.end() && it->second.variant == kPerViewVariant;
        const bool fits = it != B.tuned.end() &&
                          (per_view ? (o.launch_mode != ST_LAUNCH_PERSISTENT && !fixed_tile && !o.chunk &&
                                       o.compaction_threshold < 0)
                                    : (o.launch_mode != ST_LAUNCH_PER_VIEW &&
                                       (o.tile_shape < 0 || variant_tile(it->second.variant) == o.tile_shape) &&
                                       (o.stack_placement < 0 || variant_stack(it->second.variant) == o.stack_placement)));
        if (fits) {
            if (tile < 0) tile = it->second.variant;
            if (!chunk) chunk = (u32t)it->second.chunk;
            if (threshold < 0) threshold = tile == kPerViewVariant ? 0 : it->second.threshold;
        } else {
            // the persistent kernel's variants and chunks without compaction, then compaction
            // thresholds on the fastest of them, then one kernel per view
            const int shapes[4] = {TILE_8x4, TILE_16x2, TILE_4x8, TILE_32x1};
            const u32t chunks[2] = {1, 4};
            const u32t thresholds[3] = {8, 16, 24};
            const bool persistent = o.launch_mode != ST_LAUNCH_PER_VIEW;
            float best = INFINITY;
            int best_variant = TILE_8x4;
            u32t best_chunk = 1, best_threshold = threshold > 0 ? (u32t)threshold : 0;
            for (int stack = 0; persistent && stack < STACK_PLACEMENTS; stack++) {
                if (o.stack_placement >= 0 && stack != o.stack_placement) continue;
                for (int si = 0; si < 4; si++) {
                    if (o.tile_shape >= 0 && shapes[si] != o.tile_shape) continue;
                    const int variant = shapes[si] + TILE_SHAPES * stack;
                    if (tile >= 0 && variant != tile) continue;
                    for (u32t c : chunks) {
                        if (chunk && c != chunk) continue;
                        float ms = 0;
                        ST_TRY(time_batch(ctx, B, views, n, variant, c, best_threshold, st, o, ms));
                        if (ms < best) { best = ms; best_variant = variant; best_chunk = c; }
                    }
                }
            }
            if (persistent && threshold < 0) {
                for (u32t th : thresholds) {
                    float ms = 0;
                    ST_TRY(time_batch(ctx, B, views, n, best_variant, best_chunk, th, st, o, ms));
                    if (ms < best) { best = ms; best_threshold = th; }
                }
            }
            if (o.launch_mode < 0 && !fixed_tile && !o.chunk && o.compaction_threshold < 0) {   // one kernel per view
                float ms = 0;
                ST_TRY(time_batch(ctx, B, views, n, kPerViewVariant, 1, 0, st, o, ms));
                if (ms < best) { best = ms; best_variant = kPerViewVariant; best_chunk = 1; best_threshold = 0; }
            }
            if (o.tile_shape < 0 && o.stack_placement < 0 && !o.chunk && o.launch_mode < 0 && o.compaction_threshold < 0) {
                B.tuned[p.class_key] = Tuned{best_variant, (int)best_chunk, (int)best_threshold};
                if (const char *path = getenv("ST_AUTOTUNE_CACHE")) {
                    std::ofstream f(path, std::ios::app);
                    f << p.class_key << " " << best_variant << " " << best_chunk << " " << best_threshold << "\n";
                }
            }
            if (tile < 0) tile = best_variant;
            if (!chunk) chunk = best_chunk;
            if (threshold < 0) threshold = (int)best_threshold;
        }
        ST_TRY(plan_batch(ctx, views, n, tile, o, p));
    }
    if (tile == kPerViewVariant) threshold = 0;
    ST_TRY(batch_reserve(ctx, B, p, n, (u32t)threshold));
    o.graph_replayed = 0;
    ST_CUDA(cudaEventRecord(ctx->ev[0], st));
    if (o.use_graph) {
        // The batch's launches are captured; an instantiated graph of the same topology (the same
        // view groups and views wanting frames) is updated in place from the capture, so every kernel
        // parameter - view tables, cameras, arena and output pointers - is this call's.
        ST_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int s = enqueue_batch(ctx, B, P<unsigned>(ctx->status), views, n, p, tile, chunk, (u32t)threshold, st, o);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (s != ST_OK) { if (g) cudaGraphDestroy(g); return s; }
        if (e != cudaSuccess) return fail_cuda(ctx, e);
        bool updated = false;
        if (B.exec) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(B.exec, g, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();
                cudaGraphExecDestroy(B.exec);
                B.exec = nullptr;
            }
        }
        if (B.graph) cudaGraphDestroy(B.graph);
        B.graph = g;
        if (!B.exec) ST_CUDA(cudaGraphInstantiate(&B.exec, g, 0));
        ST_CUDA(cudaGraphLaunch(B.exec, st));
        o.graph_replayed = updated ? 1 : 0;
    } else {
        ST_TRY(enqueue_batch(ctx, B, P<unsigned>(ctx->status), views, n, p, tile, chunk, (u32t)threshold, st, o));
    }
    ST_CUDA(cudaEventRecord(ctx->ev[1], st));
    if (!o.device_outputs) {
        for (int i = 0; i < n; i++) {
            const BatchView &b = p.table[i];
            const size_t grid = (size_t)b.view.grid_w * b.view.grid_h;
            if (views[i].out_float)
                ST_CUDA(cudaMemcpyAsync(views[i].out_float, P<FloatPixel>(B.out_float) + p.float_off[i],
                                        sizeof(FloatPixel) * grid, cudaMemcpyDeviceToHost, st));
            if (views[i].out_u8)
                ST_CUDA(cudaMemcpyAsync(views[i].out_u8, P<uint32_t>(B.out_u8) + p.u8_off[i],
                                        sizeof(uint32_t) * (size_t)(b.view.grid_w - 1) * (b.view.grid_h - 1),
                                        cudaMemcpyDeviceToHost, st));
        }
    }
    unsigned status[4] = {0, 0, 0, 0};
    u32t parked = 0;
    ST_CUDA(cudaMemcpyAsync(status, ctx->status.ptr, 16, cudaMemcpyDeviceToHost, st));
    if (threshold) ST_CUDA(cudaMemcpyAsync(&parked, P<u32t>(B.counter) + 4, 4, cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&o.batch_ms, ctx->ev[0], ctx->ev[1]);
    o.parked_rays = parked;
    o.rays = p.rays;
    o.launch_mode_used = tile == kPerViewVariant ? ST_LAUNCH_PER_VIEW : ST_LAUNCH_PERSISTENT;
    o.tile_shape_used = tile == kPerViewVariant ? -1 : variant_tile(tile);
    o.stack_placement_used = tile == kPerViewVariant ? -1 : variant_stack(tile);
    o.chunk_used = (int)chunk;
    o.compaction_threshold_used = threshold;
    if (status[0] & S_STACK_OVERFLOW) return ST_ERR_STACK_OVERFLOW;
    return ST_OK;
}

int st_pick(st_ctx *ctx, int slot, const Scene *scene, const Viewport *viewport, int x, int y, st_pick_result *result) {
    static_assert(sizeof(PickDev) == sizeof(st_pick_result), "st_pick_result mirrors PickDev");
    SceneSlot *S = slot_of(ctx, slot);
    if (!S || !viewport || !result || x < 0 || y < 0) return ST_ERR_INVALID_ARG;
    if (!S->allocated || !S->tlas_valid || !S->n_prims) return ST_ERR_NOT_RESIDENT;
    for (const Primitive &p : S->prims_host)
        if (p.type == PrimitiveType_Mesh && !S->meshes_valid) return ST_ERR_NOT_RESIDENT;
    cudaSetDevice(ctx->device);
    ViewDev v;
    ST_TRY(make_view(viewport, v));
    ST_TRY(reserve(ctx, ctx->ssb, sizeof(int4) * std::max(S->n_prims, 1u)));
    ST_TRY(reserve(ctx, ctx->counters, sizeof(unsigned long long) * 16));
    SceneDev sd = scene_view(*S, scene);
    cudaStream_t st = ctx->stream;
    launch_ssb(sd, v, P<int4>(ctx->ssb), st);
    PickDev *d = reinterpret_cast<PickDev *>(ctx->counters.ptr);     // 128 bytes of scratch
    launch_pick(sd, v, P<int4>(ctx->ssb), x, y, d, st);
    ST_CUDA(cudaGetLastError());
    PickDev h;
    ST_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaStreamSynchronize(st));
    memcpy(result, &h, sizeof(h));
    return ST_OK;
}

int st_render_scene(st_ctx *ctx, int slot, const Scene *scene, Viewport *viewport) {
    if (!viewport || !viewport->frame_buffer) return ST_ERR_INVALID_ARG;
    st_render_options o;
    memset(&o, 0, sizeof(o));
    o.overlays = (viewport->settings.show_BVH ? ST_OVERLAY_BVH : 0) | (viewport->settings.show_SSB ? ST_OVERLAY_SSB : 0);
    return st_render_ex(ctx, slot, scene, viewport, &o);
}

// ---- texture baking ----------------------------------------------------------------------------
uint64_t st_texture_bytes(uint16_t width, uint16_t height, int mipmap) {
    const int mips = texture_mip_count(width, height, mipmap != 0);
    return ((sizeof(TextureMip) * mips + 15) & ~(size_t)15) + sizeof(TexelQuad) * texture_quad_count(width, height, mipmap != 0);
}

int st_bake_texture(st_ctx *ctx, const uint8_t *components, uint16_t width, uint16_t height, int bit_count, int wrap,
                    int mipmap, Texture *texture, void *memory, uint64_t memory_bytes) {
    if (!ctx || !components || !texture || !memory || width < 2 || height < 2 || (bit_count != 24 && bit_count != 32))
        return ST_ERR_INVALID_ARG;
    if (memory_bytes < st_texture_bytes(width, height, mipmap)) return ST_ERR_BUDGET;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const int mips = texture_mip_count(width, height, mipmap != 0);
    const size_t quads = texture_quad_count(width, height, mipmap != 0);
    const size_t image = (size_t)width * height * (bit_count / 8);
    const size_t table = (sizeof(TextureMip) * mips + 15) & ~(size_t)15;
    const size_t bytes = ((image + 255) & ~(size_t)255) + texture_scratch_bytes(width, height) + sizeof(TexelQuad) * quads + 512;
    if (ctx->in_use + bytes > ctx->budget) return ST_ERR_BUDGET;
    char *base = nullptr;
    ST_CUDA(cudaMallocAsync((void **)&base, bytes, st));
    uint8_t *dev_image = reinterpret_cast<uint8_t *>(base);
    char *scratch = base + ((image + 255) & ~(size_t)255);
    TexelQuad *dev_quads = reinterpret_cast<TexelQuad *>(scratch + ((texture_scratch_bytes(width, height) + 255) & ~(size_t)255));
    cudaError_t e = cudaMemcpyAsync(dev_image, components, image, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = bake_texture(dev_image, width, height, bit_count, wrap != 0, mipmap != 0, scratch, dev_quads, st);
    char *host = static_cast<char *>(memory);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host + table, dev_quads, sizeof(TexelQuad) * quads, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(base, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    TextureMip *mip = reinterpret_cast<TextureMip *>(host);
    TexelQuad *q = reinterpret_cast<TexelQuad *>(host + table);
    u32t w = width, h = height;
    for (int m = 0; m < mips; m++, w /= 2, h /= 2) {
        mip[m].width = (u16)w;
        mip[m].height = (u16)h;
        mip[m].texel_quads = q;
        q += (size_t)(w + 1) * (h + 1);
    }
    texture->width = width;
    texture->height = height;
    texture->wrap = wrap != 0;
    texture->mipmap = mipmap != 0;
    texture->mip_count = (u8)mips;
    texture->mips = mip;
    return ST_OK;
}

// ---- OBJ ingestion: obj2mesh.c:25 ---------------------------------------------------------------
namespace {
struct ObjCarve {
    size_t nodes, leaf_ids, positions, position_ids, edges, triangles, uvs, uv_ids, normals, normal_ids, total;
};
ObjCarve obj_carve(const ObjCounts &c) {
    ObjCarve k;
    size_t at = 0;
    auto take = [&](size_t b) { size_t o = at; at += (b + 15) & ~(size_t)15; return o; };
    const size_t t = c.triangles;
    k.nodes = take(sizeof(BVHNode) * 2 * t);
    k.leaf_ids = take(sizeof(u32t) * t);
    k.positions = take(sizeof(vec3) * (size_t)c.vertices);
    k.position_ids = take(sizeof(TriangleVertexIndices) * t);
    k.edges = take(sizeof(EdgeVertexIndices) * 3 * t);
    k.triangles = take(sizeof(Triangle) * t);
    k.uvs = take(sizeof(vec2) * (size_t)c.uvs);
    k.uv_ids = take(sizeof(TriangleVertexIndices) * t);
    k.normals = take(sizeof(vec3) * (size_t)c.normals);
    k.normal_ids = take(sizeof(TriangleVertexIndices) * t);
    k.total = at;
    return k;
}
}  // namespace

int64_t st_obj_mesh_bytes(const char *obj_path) {
    ObjCounts c;
    if (!obj_path || obj_count(obj_path, c) != 0) return -1;
    return (int64_t)obj_carve(c).total;
}

int st_obj_to_mesh(st_ctx *ctx, const char *obj_path, int invert_winding_order, int mode, Mesh *mesh, void *memory,
                   uint64_t memory_bytes) {
    if (!ctx || !obj_path || !mesh || !memory || (mode != ST_BVH_LBVH30 && mode != ST_BVH_BINNED_SAH))
        return ST_ERR_INVALID_ARG;
    ObjCounts c;
    if (obj_count(obj_path, c) != 0) return ST_ERR_IO;
    // updateMeshBVH reads vertex normals and obj2mesh reads uvs for every face, so only the
    // positions/uvs/normals face layout converts
    if (c.layout != 3 || !c.triangles || !c.vertices || !c.uvs || !c.normals) return ST_ERR_BAD_SCENE;
    const ObjCarve k = obj_carve(c);
    if (k.total > memory_bytes) return ST_ERR_BUDGET;
    char *base = static_cast<char *>(memory);
    Mesh m;
    memset(&m, 0, sizeof(m));
    m.vertex_count = c.vertices;
    m.triangle_count = c.triangles;
    m.uvs_count = c.uvs;
    m.normals_count = c.normals;
    m.bvh.nodes = reinterpret_cast<BVHNode *>(base + k.nodes);
    m.bvh.leaf_ids = reinterpret_cast<u32t *>(base + k.leaf_ids);
    m.vertex_positions = reinterpret_cast<vec3 *>(base + k.positions);
    m.vertex_position_indices = reinterpret_cast<TriangleVertexIndices *>(base + k.position_ids);
    m.edge_vertex_indices = reinterpret_cast<EdgeVertexIndices *>(base + k.edges);
    m.triangles = reinterpret_cast<Triangle *>(base + k.triangles);
    m.vertex_uvs = reinterpret_cast<vec2 *>(base + k.uvs);
    m.vertex_uvs_indices = reinterpret_cast<TriangleVertexIndices *>(base + k.uv_ids);
    m.vertex_normals = reinterpret_cast<vec3 *>(base + k.normals);
    m.vertex_normal_indices = reinterpret_cast<TriangleVertexIndices *>(base + k.normal_ids);
    const int parsed = obj_parse(obj_path, invert_winding_order != 0, c, m.vertex_positions, m.vertex_normals, m.vertex_uvs,
                                 reinterpret_cast<uint32_t *>(m.vertex_position_indices),
                                 reinterpret_cast<uint32_t *>(m.vertex_uvs_indices),
                                 reinterpret_cast<uint32_t *>(m.vertex_normal_indices));
    if (parsed == -1) return ST_ERR_IO;
    if (parsed != 0) return ST_ERR_BAD_SCENE;
    // the AABB over the vertices and the origin (obj2mesh.c:185-193), then centred on its middle
    // when that is not the origin (:195-202)
    AABB box;
    memset(&box, 0, sizeof(box));
    for (u32t i = 0; i < m.vertex_count; i++) {
        const vec3 &v = m.vertex_positions[i];
        box.min.x = box.min.x < v.x ? box.min.x : v.x;
        box.min.y = box.min.y < v.y ? box.min.y : v.y;
        box.min.z = box.min.z < v.z ? box.min.z : v.z;
        box.max.x = box.max.x > v.x ? box.max.x : v.x;
        box.max.y = box.max.y > v.y ? box.max.y : v.y;
        box.max.z = box.max.z > v.z ? box.max.z : v.z;
    }
    vec3 centre;
    centre.x = (box.min.x + box.max.x) * 0.5f;
    centre.y = (box.min.y + box.max.y) * 0.5f;
    centre.z = (box.min.z + box.max.z) * 0.5f;
    if (centre.x != 0 || centre.y != 0 || centre.z != 0) {
        box.min.x -= centre.x; box.min.y -= centre.y; box.min.z -= centre.z;
        box.max.x -= centre.x; box.max.y -= centre.y; box.max.z -= centre.z;
        for (u32t i = 0; i < m.vertex_count; i++) {
            vec3 &v = m.vertex_positions[i];
            v.x -= centre.x;
            v.y -= centre.y;
            v.z -= centre.z;
        }
    }
    m.aabb = box;
    // unique edges on the device
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t ids_bytes = sizeof(uint32_t) * 3 * (size_t)m.triangle_count;
    const size_t edges_bytes = sizeof(EdgeVertexIndices) * 3 * (size_t)m.triangle_count;
    const size_t bytes = ((ids_bytes + 255) & ~(size_t)255) + ((edges_bytes + 255) & ~(size_t)255) +
                         unique_edges_scratch_bytes(m.triangle_count);
    if (ctx->in_use + bytes > ctx->budget) return ST_ERR_BUDGET;
    char *dev = nullptr;
    ST_CUDA(cudaMallocAsync((void **)&dev, bytes, st));
    uint32_t *dev_ids = reinterpret_cast<uint32_t *>(dev);
    EdgeVertexIndices *dev_edges = reinterpret_cast<EdgeVertexIndices *>(dev + ((ids_bytes + 255) & ~(size_t)255));
    void *scratch = dev + ((ids_bytes + 255) & ~(size_t)255) + ((edges_bytes + 255) & ~(size_t)255);
    u32t n_edges = 0;
    cudaError_t e = cudaMemcpyAsync(dev_ids, m.vertex_position_indices, ids_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = unique_edges(dev_ids, m.triangle_count, m.vertex_count, scratch, dev_edges, &n_edges, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m.edge_vertex_indices, dev_edges, sizeof(EdgeVertexIndices) * n_edges, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(dev, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    m.edge_count = n_edges;
    // updateMeshBVH on the device: BLAS and the leaf-ordered Triangle records
    ST_TRY(st_update_mesh_bvh(ctx, &m, mode));
    *mesh = m;
    return ST_OK;
}

// ---- serving ---------------------------------------------------------------------------------
double st_clock(void) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // extern "C"

namespace {

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t request_bytes(const ServeReq &r, u32t n_prims) {
    const size_t grid = (size_t)r.view.grid_w * r.view.grid_h;
    size_t b = align256(sizeof(FloatPixel) * grid) + align256(sizeof(int4) * std::max(n_prims, 1u)) +
               align256(sizeof(float) * ray_rows_floats(r.view));
    if (r.out_u8) b += align256(sizeof(uint32_t) * (size_t)(r.view.grid_w - 1) * (r.view.grid_h - 1));
    return b;
}

// Copy a finished batch's outputs to the requests' buffers and complete them.
void finish_flight(st_ctx *ctx, InFlight &F) {
    Server &V = ctx->server;
    const unsigned status = *reinterpret_cast<unsigned *>(F.pinned);
    const double now = st_clock();
    for (auto &r : F.reqs) {
        const size_t grid = (size_t)r->view.grid_w * r->view.grid_h;
        if (r->out_float && !r->pinned_float) memcpy(r->out_float, F.pinned + r->host_float, sizeof(FloatPixel) * grid);
        if (r->out_u8 && !r->mapped_u8)
            memcpy(r->out_u8, F.pinned + r->host_u8, sizeof(uint32_t) * (size_t)(r->view.grid_w - 1) * (r->view.grid_h - 1));
    }
    std::lock_guard<std::mutex> lk(V.m);
    for (auto &r : F.reqs) {
        r->done = now;
        r->status = (status & S_STACK_OVERFLOW) ? ST_ERR_STACK_OVERFLOW : ST_OK;
    }
    V.inflight_bytes -= F.bytes;
    F.reqs.clear();
    F.scenes.clear();
    F.busy = false;
    V.cv_done.notify_all();
    // scene versions this batch was the last reader of go back to their scenes' spare lists
    const int me = (int)(&F - V.flights.data());
    for (size_t i = 0; i < V.retired.size();) {
        auto &rd = V.retired[i].readers;
        rd.erase(std::remove(rd.begin(), rd.end(), std::make_pair(me, F.launch_id)), rd.end());
        if (rd.empty()) {
            slot_of(ctx, V.retired[i].slot)->spare.push_back(V.retired[i].bufs);
            V.retired.erase(V.retired.begin() + i);
        } else {
            i++;
        }
    }
}

// Give scene `slot` a private copy of its primitive and TLAS arrays when batches in flight still
// read the current ones, so that a transform update can proceed at once: those batches keep the
// version they were launched with.  The copy is device to device on the context's stream, which
// the update that follows also uses.
int new_scene_version(st_ctx *ctx, int slot) {
    Server &V = ctx->server;
    SceneSlot *S = slot_of(ctx, slot);
    RetiredVersion old;
    old.slot = slot;
    for (size_t i = 0; i < V.flights.size(); i++)
        if (V.flights[i].busy && V.flights[i].scenes.count(slot)) old.readers.push_back({(int)i, V.flights[i].launch_id});
    if (old.readers.empty()) return ST_OK;
    MotionBufs m;
    if (!S->spare.empty()) {
        m = S->spare.back();
        S->spare.pop_back();
    }
    for (int k = 0; k < 7; k++) {
        DevBuf *mine;
        DevBuf *copy = motion_field(*S, m, k, &mine);
        if (!mine->ptr) continue;
        const int e = reserve(ctx, *copy, mine->bytes);
        if (e != ST_OK) {
            S->spare.push_back(m);
            return e;
        }
        ST_CUDA(cudaMemcpyAsync(copy->ptr, mine->ptr, mine->bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    for (int k = 0; k < 7; k++) {
        DevBuf *mine;
        DevBuf *copy = motion_field(*S, m, k, &mine);
        std::swap(*mine, *copy);
    }
    old.bufs = m;                       // after the swap: the buffers the readers hold
    V.retired.push_back(old);
    return ST_OK;
}

// Enqueue one admitted batch on its flight's stream: per-view SSB and ray rows, the trace (per view
// or persistent, as launch_groups does it), resolves, and the copies of every output into pinned
// staging.
int enqueue_flight(st_ctx *ctx, InFlight &F, BatchPlan &p, std::vector<std::shared_ptr<ServeReq>> &reqs, int tile,
                   u32t chunk, char *arena) {
    const int n = (int)reqs.size();
    cudaStream_t st = F.stream;
    for (int i = 0; i < n; i++) {
        BatchView &b = p.table[i];
        const ServeReq &r = *reqs[i];
        b.out = reinterpret_cast<FloatPixel *>(arena + r.dev_float);
        b.ssb = reinterpret_cast<int4 *>(arena + r.dev_ssb);
        b.dirs = reinterpret_cast<float *>(arena + r.dev_seg);
        b.prim_ids = nullptr;
        // page-locked frames are written by the resolve kernel itself; others go through the arena
        b.out_u8 = !r.out_u8 ? nullptr : r.mapped_u8 ? r.mapped_u8 : reinterpret_cast<uint32_t *>(arena + r.dev_u8);
    }
    ST_CUDA(cudaMemsetAsync(F.status.ptr, 0, 16, st));
    ST_TRY(launch_groups(ctx, F.B, p, tile, chunk, 0, P<unsigned>(F.status), st));
    for (int i = 0; i < n; i++) {
        const ServeReq &r = *reqs[i];
        const BatchView &b = p.table[i];
        const size_t grid = (size_t)b.view.grid_w * b.view.grid_h;
        if (r.out_u8 && !r.mapped_u8)
            ST_CUDA(cudaMemcpyAsync(F.pinned + r.host_u8, b.out_u8, (size_t)(b.view.grid_w - 1) * (b.view.grid_h - 1) * 4,
                                    cudaMemcpyDeviceToHost, st));
        if (r.out_float)
            ST_CUDA(cudaMemcpyAsync(r.pinned_float ? reinterpret_cast<char *>(r.out_float) : F.pinned + r.host_float, b.out,
                                    sizeof(FloatPixel) * grid, cudaMemcpyDeviceToHost, st));
    }
    ST_CUDA(cudaMemcpyAsync(F.pinned, F.status.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaEventRecord(F.done_ev, st));
    return ST_CUDA_LAST();
}

// Apply the batch's transform updates and TLAS maintenance, then launch it on flight slot f.
int launch_flight(st_ctx *ctx, int f, std::vector<std::shared_ptr<ServeReq>> &reqs) {
    Server &V = ctx->server;
    InFlight &F = V.flights[f];
    // transform updates, in submission order; a scene read by a batch in flight gets a new version
    std::map<int, uint32_t> moved_count;
    for (auto &r : reqs) {
        if (r->moved.empty()) continue;
        ST_TRY(new_scene_version(ctx, r->slot));
        ST_TRY(st_update_primitives(ctx, r->slot, r->moved.data(), r->moved_ids.data(), (uint32_t)r->moved.size()));
        moved_count[r->slot] += (uint32_t)r->moved.size();
    }
    for (auto &kv : moved_count) {
        SceneSlot *S = slot_of(ctx, kv.first);
        // refit while the primitives moved since the last full build stay below the fraction: a
        // refit keeps the topology, whose quality decays as motion accumulates
        S->moved_since_build += kv.second;
        const int mode = (double)S->moved_since_build < V.cfg.refit_fraction * S->n_prims ? ST_BVH_REFIT : ST_BVH_LBVH30;
        ST_TRY(st_update_scene_bvh(ctx, kv.first, nullptr, mode));
    }
    // view table and arena layout
    const int n = (int)reqs.size();
    BatchPlan p;
    int tile = V.cfg.launch_mode == ST_LAUNCH_PER_VIEW ? kPerViewVariant : V.cfg.tile_shape >= 0 ? V.cfg.tile_shape : TILE_8x4;
    u32t chunk = V.cfg.chunk > 0 ? (u32t)V.cfg.chunk : 1;
    std::ostringstream cls;
    size_t dev = 0, host = 64;
    u32t tw, th;
    for (auto &r : reqs) {
        SceneSlot *S = slot_of(ctx, r->slot);
        u32t tris = 0;
        for (const MeshDev &m : S->mesh_host) tris += m.triangle_count;
        int pb = 0, tb = 0;
        for (u32t x = S->n_prims; x > 1; x >>= 1) pb++;
        for (u32t x = tris; x > 1; x >>= 1) tb++;
        cls << "p" << pb << "t" << tb << "d" << r->view.depth << ";";
    }
    if (V.cfg.launch_mode == ST_LAUNCH_PERSISTENT && (V.cfg.tile_shape < 0 || V.cfg.chunk <= 0)) {
        auto it = ctx->batch.tuned.find(cls.str());
        if (it != ctx->batch.tuned.end() && it->second.variant != kPerViewVariant) {
            if (V.cfg.tile_shape < 0) tile = it->second.variant;
            if (V.cfg.chunk <= 0) chunk = (u32t)it->second.chunk;
        }
    }
    tile_dims(tile, tw, th);
    for (auto &r : reqs) {
        SceneSlot *S = slot_of(ctx, r->slot);
        BatchView b;
        memset(&b, 0, sizeof(b));
        b.view = r->view;
        b.view.primary_tlas = S->n_prims > 64 ? 1 : 0;
        b.scene = scene_view(*S, nullptr);
        if (r->has_scene_values) {
            b.scene.ambient = r->ambient;
            b.scene.lights = r->lights_present ? P<Light>(S->lights) : nullptr;
            b.scene.n_lights = r->lights_present ? S->n_lights : 0;
        }
        b.tile_begin = p.total_tiles;
        p.total_tiles += view_tiles(b, tw, th);
        const size_t grid = (size_t)b.view.grid_w * b.view.grid_h;
        r->dev_float = dev; dev += align256(sizeof(FloatPixel) * grid);
        r->dev_ssb = dev; dev += align256(sizeof(int4) * std::max(S->n_prims, 1u));
        r->dev_seg = dev; dev += align256(sizeof(float) * ray_rows_floats(b.view));
        const size_t u8b = (size_t)(b.view.grid_w - 1) * (b.view.grid_h - 1) * sizeof(uint32_t);
        if (r->out_u8) { r->dev_u8 = dev; dev += align256(u8b); }
        r->rays = grid;
        r->batch_size = n;
        p.table.push_back(b);
        F.scenes.insert(r->slot);
    }
    // host staging: the status word, then each request's float grid and u8 frame
    for (auto &r : reqs) {
        const size_t grid = (size_t)r->view.grid_w * r->view.grid_h;
        if (r->out_float && !r->pinned_float) { r->host_float = host; host += align256(sizeof(FloatPixel) * grid); }
        if (r->out_u8 && !r->mapped_u8) {
            r->host_u8 = host;
            host += align256((size_t)(r->view.grid_w - 1) * (r->view.grid_h - 1) * 4);
        }
    }
    if (F.pinned_cap < host) {                  // grows geometrically: cudaFreeHost waits for the device
        const size_t cap = std::max(host, 2 * F.pinned_cap);
        if (F.pinned) cudaFreeHost(F.pinned);
        F.pinned = nullptr;
        F.pinned_cap = 0;
        ST_CUDA(cudaMallocHost((void **)&F.pinned, cap));
        F.pinned_cap = cap;
    }
    ST_TRY(reserve(ctx, F.B.counter, 16));
    ST_TRY(table_reserve(ctx, F.B, std::max(n, V.cfg.max_views_per_batch)));
    cudaStream_t st = F.stream;
    char *arena = nullptr;
    ST_CUDA(cudaMallocFromPoolAsync((void **)&arena, std::max(dev, (size_t)256), V.pool, st));
    const int s = enqueue_flight(ctx, F, p, reqs, tile, chunk, arena);
    cudaFreeAsync(arena, st);   // stream-ordered: released once the batch's work has run
    ST_TRY(s);
    const double t = st_clock();
    for (auto &r : reqs) r->launch = t;
    F.launch_id = V.next_launch++;
    F.bytes = dev;
    F.reqs = reqs;
    F.busy = true;
    return ST_OK;
}

void serve_loop(st_ctx *ctx) {
    Server &V = ctx->server;
    cudaSetDevice(ctx->device);
    for (;;) {
        for (InFlight &F : V.flights)
            if (F.busy && cudaEventQuery(F.done_ev) == cudaSuccess) finish_flight(ctx, F);
        std::vector<std::shared_ptr<ServeReq>> batch;
        int free_slot = -1;
        {
            std::unique_lock<std::mutex> lk(V.m);
            bool any_busy = false;
            for (size_t i = 0; i < V.flights.size(); i++) {
                if (V.flights[i].busy) any_busy = true;
                else if (free_slot < 0) free_slot = (int)i;
            }
            if (V.stop && V.pending.empty() && !any_busy) break;
            if (free_slot >= 0 && !V.pending.empty()) {
                // admit in order while the budget and the batch rules allow
                uint64_t bytes = 0;
                std::set<int> scenes;
                while (!V.pending.empty() && (int)batch.size() < V.cfg.max_views_per_batch) {
                    auto &r = V.pending.front();
                    SceneSlot *S = slot_of(ctx, r->slot);
                    const size_t need = request_bytes(*r, S->n_prims);
                    if (!r->moved.empty() && scenes.count(r->slot)) break;   // it changes a scene this batch renders
                    if (V.inflight_bytes + bytes + need > V.frame_budget) {
                        if (batch.empty() && !any_busy) {                   // can never fit
                            r->status = ST_ERR_BUDGET;
                            r->done = st_clock();
                            V.pending.pop_front();
                            V.cv_done.notify_all();
                            continue;
                        }
                        break;
                    }
                    bytes += need;
                    scenes.insert(r->slot);
                    batch.push_back(r);
                    V.pending.pop_front();
                }
                V.inflight_bytes += bytes;
                if (batch.empty()) free_slot = -1;
            } else {
                V.cv_work.wait_for(lk, std::chrono::microseconds(any_busy ? 50 : 2000));
                continue;
            }
        }
        if (free_slot >= 0 && !batch.empty()) {
            uint64_t held = 0;
            for (auto &r : batch) held += request_bytes(*r, slot_of(ctx, r->slot)->n_prims);
            int s = launch_flight(ctx, free_slot, batch);
            std::lock_guard<std::mutex> lk(V.m);
            V.inflight_bytes -= held;                    // the flight now accounts its own bytes
            if (s == ST_OK) V.inflight_bytes += V.flights[free_slot].bytes;
            else {
                V.flights[free_slot].scenes.clear();
                for (auto &r : batch) { r->status = s; r->done = st_clock(); }
                V.cv_done.notify_all();
            }
        }
    }
}

}  // namespace

extern "C" {

int st_serve_start(st_ctx *ctx, const st_serve_config *cfg) {
    if (!ctx) return ST_ERR_INVALID_ARG;
    Server &V = ctx->server;
    if (V.running) return ST_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    V.cfg = cfg ? *cfg : st_serve_config{};
    if (V.cfg.max_in_flight <= 0) V.cfg.max_in_flight = 3;
    if (V.cfg.max_views_per_batch <= 0) V.cfg.max_views_per_batch = 64;
    if (V.cfg.refit_fraction <= 0) V.cfg.refit_fraction = 0.25;
    if (!cfg) { V.cfg.tile_shape = -1; V.cfg.chunk = 0; }
    if (V.cfg.launch_mode != ST_LAUNCH_PER_VIEW && V.cfg.launch_mode != ST_LAUNCH_PERSISTENT) return ST_ERR_INVALID_ARG;
    V.frame_budget = V.cfg.frame_budget ? V.cfg.frame_budget
                                        : (ctx->budget > ctx->in_use ? ctx->budget - ctx->in_use : 0);
    V.flights.resize(V.cfg.max_in_flight);
    for (InFlight &F : V.flights) {
        ST_CUDA(cudaStreamCreateWithFlags(&F.stream, cudaStreamNonBlocking));
        ST_CUDA(cudaEventCreateWithFlags(&F.done_ev, cudaEventDisableTiming));
        ST_TRY(reserve(ctx, F.status, 16));
        F.pinned_cap = 64u << 20;              // output staging; grows if a batch needs more
        ST_CUDA(cudaMallocHost((void **)&F.pinned, F.pinned_cap));
    }
    // batch arenas come from a pool that keeps what batches free (the default pool would hand
    // memory back at every synchronisation and map it again for the next batch)
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    ST_CUDA(cudaMemPoolCreate(&V.pool, &props));
    uint64_t keep = UINT64_MAX;
    ST_CUDA(cudaMemPoolSetAttribute(V.pool, cudaMemPoolAttrReleaseThreshold, &keep));
    {   // grow the pool now (up to 2 GB of the frame budget) rather than under the first heavy load
        const size_t warm = (size_t)std::min<uint64_t>(V.frame_budget, 2ull << 30);
        void *p = nullptr;
        if (warm && cudaMallocFromPoolAsync(&p, warm, V.pool, ctx->stream) == cudaSuccess) cudaFreeAsync(p, ctx->stream);
        cudaGetLastError();
        ST_TRY(ST_CUDA_SYNC(ctx));
    }
    // spare scene versions for the resident scenes, so that the first updates under load do not
    // allocate (one per batch that can be in flight)
    for (int slot = 0; slot < (int)ctx->slots.size(); slot++) {
        SceneSlot &S = ctx->slots[slot];
        if (!S.allocated || !S.tlas_valid) continue;
        while ((int)S.spare.size() < V.cfg.max_in_flight) {
            MotionBufs m;
            for (int k = 0; k < 7; k++) {
                DevBuf *mine;
                DevBuf *copy = motion_field(S, m, k, &mine);
                if (mine->ptr) ST_TRY(reserve(ctx, *copy, mine->bytes));
            }
            S.spare.push_back(m);
        }
    }
    V.stop = false;
    V.running = true;
    V.inflight_bytes = 0;
    V.worker = std::thread(serve_loop, ctx);
    return ST_OK;
}

int st_submit(st_ctx *ctx, const st_request *req, st_ticket *ticket) {
    if (!ctx || !req || !ticket || !req->view.viewport) return ST_ERR_INVALID_ARG;
    Server &V = ctx->server;
    if (!V.running) return ST_ERR_INVALID_ARG;
    SceneSlot *S = slot_of(ctx, req->view.slot);
    if (!S || !S->allocated || !S->tlas_valid) return ST_ERR_NOT_RESIDENT;
    auto r = std::make_shared<ServeReq>();
    r->slot = req->view.slot;
    ST_TRY(make_view(req->view.viewport, r->view));
    if (req->view.scene) {
        r->has_scene_values = true;
        r->ambient = req->view.scene->ambient_light.color;
        r->lights_present = req->view.scene->lights != nullptr && req->view.scene->settings.lights;
    }
    r->out_float = req->view.out_float;
    r->out_u8 = req->view.out_u8;
    // page-locked outputs need no staging and no copy on the worker thread
    if (r->out_u8) r->mapped_u8 = static_cast<uint32_t *>(device_view_of_host(r->out_u8));
    if (r->out_float) r->pinned_float = device_view_of_host(r->out_float) != nullptr;
    if (req->moved_count) {
        if (!req->moved || !req->moved_ids) return ST_ERR_INVALID_ARG;
        for (uint32_t k = 0; k < req->moved_count; k++)
            if (req->moved_ids[k] >= S->n_prims) return ST_ERR_INVALID_ARG;
        r->moved.assign(req->moved, req->moved + req->moved_count);
        r->moved_ids.assign(req->moved_ids, req->moved_ids + req->moved_count);
    }
    r->arrival = req->arrival_time;
    std::lock_guard<std::mutex> lk(V.m);
    r->id = V.next_id++;
    V.tickets[r->id] = r;
    V.pending.push_back(r);
    *ticket = r->id;
    V.cv_work.notify_one();
    return ST_OK;
}

static void fill_result(const ServeReq &r, st_result *out) {
    out->status = r.status;
    out->arrival_time = r.arrival;
    out->launch_time = r.launch;
    out->completion_time = r.done;
    out->rays = r.rays;
    out->batch_size = r.batch_size;
}

int st_poll(st_ctx *ctx, st_ticket ticket, st_result *result) {
    if (!ctx) return ST_ERR_INVALID_ARG;
    Server &V = ctx->server;
    std::lock_guard<std::mutex> lk(V.m);
    auto it = V.tickets.find(ticket);
    if (it == V.tickets.end()) return ST_ERR_INVALID_ARG;
    if (it->second->status == ST_ERR_NOT_READY) return ST_ERR_NOT_READY;
    if (result) fill_result(*it->second, result);
    V.tickets.erase(it);
    return ST_OK;
}

int st_wait(st_ctx *ctx, st_ticket ticket, st_result *result, double timeout_s) {
    if (!ctx) return ST_ERR_INVALID_ARG;
    Server &V = ctx->server;
    std::unique_lock<std::mutex> lk(V.m);
    auto it = V.tickets.find(ticket);
    if (it == V.tickets.end()) return ST_ERR_INVALID_ARG;
    auto r = it->second;
    if (!V.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->status != ST_ERR_NOT_READY; }))
        return ST_ERR_TIMEOUT;
    if (result) fill_result(*r, result);
    V.tickets.erase(ticket);
    return ST_OK;
}

int st_serve_stop(st_ctx *ctx) {
    if (!ctx) return ST_ERR_INVALID_ARG;
    Server &V = ctx->server;
    if (!V.running) return ST_OK;
    {
        std::lock_guard<std::mutex> lk(V.m);
        V.stop = true;
        V.cv_work.notify_all();
    }
    V.worker.join();
    for (InFlight &F : V.flights) {
        if (F.pinned) cudaFreeHost(F.pinned);
        if (F.B.staging) cudaFreeHost(F.B.staging);
        release_aux(F.B);
        for (DevBuf *b : {&F.B.table, &F.B.counter, &F.status}) release(ctx, *b);
        if (F.done_ev) cudaEventDestroy(F.done_ev);
        if (F.stream) cudaStreamDestroy(F.stream);
    }
    V.flights.clear();
    for (RetiredVersion &rv : V.retired) slot_of(ctx, rv.slot)->spare.push_back(rv.bufs);
    V.retired.clear();
    if (V.pool) {
        cudaDeviceSynchronize();
        cudaMemPoolDestroy(V.pool);
        V.pool = nullptr;
    }
    V.running = false;
    return ST_OK;
}

}  // extern "C"


// ---- LBVH30 build that allocates nothing ---------------------------------------------------------
// st_build_bvh and updateSceneBVH take their scratch from a per-context pool that grows with
// cudaMalloc, and cudaMalloc/cudaFree can wait for work queued on every stream of the device.  A
// host that rebuilds a TLAS between batches still running on other streams (a serving worker), or
// one whose memory budget is fully reserved up front, cannot afford that wait or that growth.  This
// variant keeps its scratch in one static device array sized for ST_NOALLOC_LBVH_MAX_ITEMS items.
namespace {

constexpr size_t kNoAllocScratchBytes = lbvh_scratch_bytes(ST_NOALLOC_LBVH_MAX_ITEMS);
// Nothing here has to start at zero: every word a build reads was written earlier in the same
// build (bounds_init_kernel, the radix histograms, cudaMemsetAsync of the arrival counters and of
// the height word).  Calls that overlap on one device share this array and race.
static __device__ __align__(256) unsigned char g_lbvh_noalloc_scratch[kNoAllocScratchBytes];

// The array's device address on the current device.  It is looked up on every call rather than
// cached: a cudaDeviceReset or a primary-context teardown reloads the module at another address,
// and after the first call (which may load the module) the lookup is cheap.  The symbol itself is
// never handed to a kernel.
int noalloc_scratch(st_ctx *ctx, void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_lbvh_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    if (!p || (reinterpret_cast<uintptr_t>(p) & 255)) return fail_cuda(ctx, cudaErrorInvalidSymbol);
    *out = p;
    return ST_OK;
}

}  // namespace

extern "C" {

int st_build_lbvh_noalloc(st_ctx *ctx, const float *aabbs, uint32_t n, uint32_t max_leaf, uint32_t *codes,
                          uint32_t *order, BVHNode *nodes, uint32_t info[2], void *stream) {
    if (!ctx || !aabbs || !order || !nodes || !info || n == 0 || max_leaf == 0 || max_leaf > 0xFFFF)
        return ST_ERR_INVALID_ARG;
    if (n > ST_NOALLOC_LBVH_MAX_ITEMS) return ST_ERR_INVALID_ARG;   // beyond the static scratch
    ST_CUDA(cudaSetDevice(ctx->device));
    void *scratch = nullptr;
    ST_TRY(noalloc_scratch(ctx, &scratch));
    LbvhScratch s;
    lbvh_carve(s, scratch, ST_NOALLOC_LBVH_MAX_ITEMS);
    s.aabbs = const_cast<float *>(aabbs);   // only read by the build
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    u32t inf[2];
    cudaError_t e = lbvh_build(s, n, max_leaf, nodes, order, inf, st);
    if (e == cudaSuccess && codes) {
        launch_codes_by_item(s, n, codes, st);
        e = cudaStreamSynchronize(st);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(ctx, e);
    info[0] = inf[0];
    info[1] = inf[1];
    return ST_OK;
}

}  // extern "C"
