"""Mixed-request workloads over several resident scenes, seeded.

resident_scenes()   eight scenes: four 16-primitive implicit scenes, three mesh scenes whose
                    displaced icospheres have 81,920 / 327,680 / 1,310,720 triangles (8 instances,
                    Cook-Torrance, glass, mirror, textures, 2 emissive quads), and one 4096-primitive
                    implicit scene
random_view()       a request's view: scene, resolution from {256x256, 640x480, 1280x720, 1920x1080},
                    bounce count 1..6 and a camera pose orbiting the scene
random_update()     a transform update of 0..64 primitives of a scene (rigid move of each)
poisson_arrivals()  arrival times of a Poisson stream

PerFrame / Batch    the same views through st_render_ex one view per call, or through one
                    st_render_batch call, with every ctypes argument built once beforehand so that
                    the measured time is the library's, not Python's.
"""
import ctypes as C
import math

import numpy as np

from . import api, scenes, structs as S

RESOLUTIONS = [(256, 256), (640, 480), (1280, 720), (1920, 1080)]


class Resident:
    """One resident scene: its data, the point the cameras orbit, the orbit radius and height."""

    def __init__(self, name, sd, target, radius, height, tlas):
        self.name, self.sd, self.target, self.radius, self.height, self.tlas = name, sd, target, radius, height, tlas
        self.sc, self.keep = sd.to_ctypes()


def resident_scenes(mesh_subdivisions=(6, 7, 8), texture_size=1024, big=None):
    """The eight scenes (a prebuilt 1.31M-triangle scene may be passed as `big`)."""
    out = []
    for k in range(4):
        sd, _ = scenes.implicit16_scene(seed_offset=100 + k)
        out.append(Resident(f"implicit16-{k}", sd, (0.0, 0.0, 0.0), 15.0, 2.0, "sah"))
    for sub in mesh_subdivisions:
        if big is not None and sub == 8:
            sd = big
        else:
            sd, _ = scenes.mesh_scene(seed_offset=200 + sub, subdivisions=sub, texture_size=texture_size)
        out.append(Resident(f"mesh{sd.meshes[0].triangle_count}", sd, (0.0, 1.5, 0.0), 15.0, 8.0, "sah"))
    sd, _ = scenes.moving_scene(seed_offset=300)
    out.append(Resident("implicit4096", sd, (0.0, 0.0, 0.0), 20.0, 3.0, "sah"))
    return out


def upload(renderer, residents, first_slot=0):
    """Upload every scene into consecutive slots; mesh BLASes and TLASes are built on the device
    with the binned SAH (the serving loop rebuilds moved scenes' TLASes with LBVH30)."""
    slots = []
    for k, res in enumerate(residents):
        slot = first_slot + k
        for md in res.sd.meshes:
            if md.triangle_count and not getattr(md, "device_built", False):
                renderer.build_blas(md, api.ST_BVH_BINNED_SAH)
                md.device_built = True
        renderer.upload(slot, res.sd, tlas=None)
        renderer.build_tlas(slot, res.sd, api.ST_BVH_BINNED_SAH if res.tlas == "sah" else api.ST_BVH_LBVH30)
        res.sc, res.keep = res.sd.to_ctypes()
        slots.append(slot)
    return slots


def random_camera(rng, res):
    yaw = rng.uniform(-math.pi, math.pi)
    r = res.radius * rng.uniform(0.8, 1.2)
    pos = (res.target[0] + r * math.sin(yaw), res.target[1] + res.height * rng.uniform(0.5, 1.0),
           res.target[2] - r * math.cos(yaw))
    return scenes.look_at(pos, res.target)


def random_view(rng, n_scenes):
    """(scene index, width, height, bounces)"""
    si = int(rng.integers(0, n_scenes))
    w, h = RESOLUTIONS[int(rng.integers(0, len(RESOLUTIONS)))]
    return si, w, h, int(rng.integers(1, 7))


def random_update(rng, res, max_count=64, step=0.05):
    """A rigid move (translation and a small rotation) of 0..max_count primitives of `res`; the
    scene's host copy is updated too.  Returns (records, ids) or (None, None)."""
    n = len(res.sd.primitives)
    count = int(rng.integers(0, min(max_count, n) + 1))
    if count == 0:
        return None, None
    ids = np.sort(rng.choice(n, count, replace=False)).astype(np.uint32)
    p = res.sd.primitives
    p["position"][ids] = (p["position"][ids] + rng.uniform(-step, step, (count, 3))).astype(np.float32)
    half = rng.uniform(0, step, count) * 0.5
    axis = rng.normal(size=(count, 3))
    axis /= np.maximum(np.linalg.norm(axis, axis=1, keepdims=True), 1e-12)
    dq = np.concatenate([axis * np.sin(half)[:, None], np.cos(half)[:, None]], 1)
    q = p["rotation"][ids].astype(np.float64)
    x1, y1, z1, w1 = dq.T
    x2, y2, z2, w2 = q.T
    out = np.stack([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2, w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                    w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2, w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2], 1)
    out /= np.linalg.norm(out, axis=1, keepdims=True)
    p["rotation"][ids] = out.astype(np.float32)
    return p[ids].copy(), ids


def poisson_arrivals(rng, rate, count):
    return np.cumsum(rng.exponential(1.0 / rate, count))


class PerFrame:
    """Views rendered one st_render_ex call each, outputs to device buffers."""

    def __init__(self, renderer, items, out_float_ptr, out_u8_ptr):
        """items: [(slot, Resident, Frame)]; the output buffers must hold the largest view."""
        self.r, self.items = renderer, items
        self.opts = []
        for _ in items:
            o = api.st_render_options()
            o.device_outputs = 1
            o.out_float = out_float_ptr
            o.out_u8 = out_u8_ptr
            self.opts.append(o)

    def run(self):
        L, ctx = self.r.L, self.r.ctx
        for (slot, res, fr), o in zip(self.items, self.opts):
            s = L.st_render_ex(ctx, slot, C.byref(res.sc), C.byref(fr.viewport), C.byref(o))
            if s:
                self.r._check(s, "st_render_ex")

    def device_ms(self):
        """Of the last run: the summed CUDA-event times of the views' whole renders and of their
        trace kernels alone."""
        return sum(o.total_ms for o in self.opts), sum(o.trace_ms for o in self.opts)


class Batch:
    """The same views in one st_render_batch call (device outputs, autotuned, CUDA graph)."""

    def __init__(self, renderer, items, out_float_ptrs, out_u8_ptrs, use_graph=True, tile_shape=-1, chunk=0,
                 stack_placement=-1, launch_mode=api.LAUNCH_AUTOTUNED, compaction_threshold=-1):
        self.r = renderer
        self.views = (api.st_view * len(items))()
        self.keep = items
        for k, (slot, res, fr) in enumerate(items):
            v = self.views[k]
            v.slot, v.scene, v.viewport = slot, C.addressof(res.sc), C.addressof(fr.viewport)
            v.out_float, v.out_u8 = out_float_ptrs[k], out_u8_ptrs[k]
        self.opt = api.st_batch_options()
        self.opt.device_outputs, self.opt.use_graph = 1, int(use_graph)
        self.opt.tile_shape, self.opt.chunk = tile_shape, chunk
        self.opt.stack_placement = stack_placement
        self.opt.launch_mode = launch_mode
        self.opt.compaction_threshold = compaction_threshold

    def run(self):
        s = self.r.L.st_render_batch(self.r.ctx, self.views, len(self.views), C.byref(self.opt))
        if s:
            self.r._check(s, "st_render_batch")
        return self.opt


class Stream:
    """A seeded Poisson request stream over resident scenes: each request is a view (scene,
    resolution, bounces, camera) plus a transform update of 0..64 primitives, delivered as a
    resolved u8 frame into host memory."""

    def __init__(self, residents, slots, rate, count, seed, refit_fraction=0.25, launch_mode=api.LAUNCH_PER_VIEW):
        rng = np.random.default_rng(seed)
        self.residents, self.slots, self.rate = residents, slots, rate
        self.refit_fraction = refit_fraction
        self.launch_mode = launch_mode
        self.arrivals = poisson_arrivals(rng, rate, count)
        # one page-locked frame per resolution, shared by the requests (the kernels write it directly)
        import torch
        self.pinned = {r: torch.zeros(r[0] * r[1] * 4, dtype=torch.uint8, pin_memory=True) for r in RESOLUTIONS}
        self.out = {r: t.data_ptr() for r, t in self.pinned.items()}
        self.requests = []
        for k in range(count):
            si, w, h, d = random_view(rng, len(residents))
            fr = scenes.Frame(w, h, random_camera(rng, residents[si]), depth=d, with_pixels=False, with_float=False)
            upd, ids = random_update(rng, residents[si])
            req = api.st_request()
            req.view.slot = slots[si]
            req.view.scene = C.addressof(residents[si].sc)
            req.view.viewport = C.addressof(fr.viewport)
            req.view.out_u8 = self.out[(w, h)]
            if upd is not None:
                req.moved, req.moved_ids, req.moved_count = upd.ctypes.data, ids.ctypes.data, len(ids)
            self.requests.append((si, w, h, fr, upd, ids, req))

    @staticmethod
    def _until(L, t):
        while L.st_clock() < t:
            pass

    def serve(self, renderer, max_in_flight=3, max_views_per_batch=64):
        """Submit at the arrival times to the library's server; returns per-request
        (arrival, completion, rays, status, width, height, batch size)."""
        L, ctx = renderer.L, renderer.ctx
        srv = api.Server(renderer, max_in_flight=max_in_flight, max_views_per_batch=max_views_per_batch,
                         refit_fraction=self.refit_fraction, launch_mode=self.launch_mode)
        tickets = []
        try:
            t0 = L.st_clock() + 0.02
            t = C.c_uint64()
            for (si, w, h, fr, upd, ids, req), a in zip(self.requests, self.arrivals):
                req.arrival_time = t0 + a
                self._until(L, req.arrival_time)
                renderer._check(L.st_submit(ctx, C.byref(req), C.byref(t)), "st_submit")
                tickets.append(t.value)
            res = []
            for tk, (si, w, h, *_r) in zip(tickets, self.requests):
                out = api.st_result()
                renderer._check(L.st_wait(ctx, tk, C.byref(out), 300.0), "st_wait")
                res.append((out.arrival_time, out.completion_time, out.rays, out.status, w, h, out.batch_size))
        finally:
            srv.stop()
        return res

    def per_frame(self, renderer):
        """The same requests, one at a time in arrival order through st_update_primitives,
        st_update_scene_bvh and st_render_ex (u8 to host)."""
        L, ctx = renderer.L, renderer.ctx
        opt = api.st_render_options()
        opt.skip_float_copy = 1
        res = []
        moved_since = {}
        t0 = L.st_clock() + 0.02
        for (si, w, h, fr, upd, ids, req), a in zip(self.requests, self.arrivals):
            arrival = t0 + a
            self._until(L, arrival)
            slot = self.slots[si]
            if upd is not None:
                renderer._check(L.st_update_primitives(ctx, slot, upd.ctypes.data, ids.ctypes.data, len(ids)),
                                "st_update_primitives")
                n = len(self.residents[si].sd.primitives)
                moved_since[si] = moved_since.get(si, 0) + len(ids)
                mode = api.ST_BVH_REFIT if moved_since[si] < self.refit_fraction * n else api.ST_BVH_LBVH30
                if mode != api.ST_BVH_REFIT:
                    moved_since[si] = 0
                renderer._check(L.st_update_scene_bvh(ctx, slot, None, mode), "st_update_scene_bvh")
            opt.out_u8 = self.out[(w, h)]
            renderer._check(L.st_render_ex(ctx, slot, C.byref(self.residents[si].sc), C.byref(fr.viewport),
                                           C.byref(opt)), "st_render_ex")
            res.append((arrival, L.st_clock(), fr.rays, 0, w, h, 1))
        return res


def latency_summary(res):
    """p50/p99 latency (ms), the same for 1080p requests, Mrays/s over the stream, batch sizes."""
    arr = np.array([r[0] for r in res])
    done = np.array([r[1] for r in res])
    rays = np.array([r[2] for r in res], dtype=np.float64)
    ok = np.array([r[3] == 0 for r in res])
    big = np.array([(r[4], r[5]) == (1920, 1080) for r in res])
    lat = (done - arr) * 1e3
    span = done.max() - arr.min()
    out = {"requests": len(res), "accepted": float(ok.mean()),
           "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
           "mrays_s": float(rays[ok].sum() / span / 1e6)}
    if big.any():
        out["p99_1080p_ms"] = float(np.percentile(lat[big], 99))
    out["mean_batch"] = float(np.mean([r[6] for r in res]))
    return out
