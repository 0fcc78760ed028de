"""ctypes binding of libslimtracin_b200 (include/slimtracin_b200.h) and a thin Python host over it.

The binding is the same one a SlimTracin host written in C links against; `Renderer` mirrors the
reference's per-frame sequence (core/init.h:36-126 uploads, builder_top_down.h:366 updateSceneBVH,
raytracer.h:302 renderScene) on reference structs built by `scenes`.  There is no CPU path: every
call goes to the CUDA library, and importing fails loudly when it is not built.
"""
import ctypes as C
import os

import numpy as np

from . import structs as S

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libslimtracin_b200.so")

ST_OK = 0
ST_ERR_INVALID_ARG, ST_ERR_BUDGET, ST_ERR_BAD_SCENE, ST_ERR_IO = 1, 5, 9, 13
ST_BVH_LBVH30, ST_BVH_BINNED_SAH, ST_BVH_REFIT, ST_BVH_REF_SAH = 1, 2, 3, 4
COUNTER_NAMES = ["primary_rays", "shadow_rays", "bounce_rays", "aabb_tests", "triangle_tests",
                 "primitive_tests", "leaf_id_reads", "shaded_hits", "texel_fetches", "mesh_entries",
                 "texel_mip_fetches"]


class st_config(C.Structure):
    _fields_ = [("device", C.c_int), ("memory_budget", C.c_uint64), ("max_scenes", C.c_int),
                ("flags", C.c_uint32)]


class st_render_options(C.Structure):
    _fields_ = [("stream", C.c_void_p), ("device_outputs", C.c_int), ("out_float", C.c_void_p),
                ("out_u8", C.c_void_p), ("out_prim_id", C.c_void_p), ("skip_float_copy", C.c_int),
                ("count_work", C.c_int), ("counters", C.c_uint64 * 16), ("trace_ms", C.c_float),
                ("total_ms", C.c_float), ("overlays", C.c_int)]


OVERLAY_BVH, OVERLAY_SSB = 1, 2     # enum st_overlay
LAUNCH_AUTOTUNED, LAUNCH_PER_VIEW, LAUNCH_PERSISTENT = -1, 0, 1   # enum st_launch_mode


class st_view(C.Structure):
    _fields_ = [("slot", C.c_int), ("scene", C.c_void_p), ("viewport", C.c_void_p), ("out_float", C.c_void_p),
                ("out_u8", C.c_void_p)]


class st_batch_options(C.Structure):
    _fields_ = [("stream", C.c_void_p), ("device_outputs", C.c_int), ("tile_shape", C.c_int), ("chunk", C.c_int),
                ("use_graph", C.c_int), ("batch_ms", C.c_float), ("rays", C.c_uint64),
                ("tile_shape_used", C.c_int), ("chunk_used", C.c_int), ("graph_replayed", C.c_int),
                ("stack_placement", C.c_int), ("stack_placement_used", C.c_int),
                ("launch_mode", C.c_int), ("launch_mode_used", C.c_int),
                ("compaction_threshold", C.c_int), ("compaction_threshold_used", C.c_int),
                ("parked_rays", C.c_uint64)]


class st_serve_config(C.Structure):
    _fields_ = [("max_in_flight", C.c_int), ("max_views_per_batch", C.c_int), ("frame_budget", C.c_uint64),
                ("tile_shape", C.c_int), ("chunk", C.c_int), ("refit_fraction", C.c_double), ("launch_mode", C.c_int)]


class st_request(C.Structure):
    _fields_ = [("view", st_view), ("moved", C.c_void_p), ("moved_ids", C.c_void_p), ("moved_count", C.c_uint32),
                ("arrival_time", C.c_double)]


class st_result(C.Structure):
    _fields_ = [("status", C.c_int), ("arrival_time", C.c_double), ("launch_time", C.c_double),
                ("completion_time", C.c_double), ("rays", C.c_uint64), ("batch_size", C.c_int)]


ST_ERR_NOT_READY, ST_ERR_TIMEOUT = 11, 7


class st_pick_result(C.Structure):
    _fields_ = [("found", C.c_int), ("object_type", C.c_int), ("object_id", C.c_uint32),
                ("position", C.c_float * 3), ("distance", C.c_float), ("object_distance", C.c_float)]


class STError(RuntimeError):
    def __init__(self, status, what, detail=""):
        self.status = status
        super().__init__(f"{what}: status {status} ({lib().st_strerror(status).decode()}) {detail}".strip())


_lib = None


def lib():
    """Load the CUDA library; raise if it is missing (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built; run `python -m slimtracin_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i, u32, u64 = C.c_void_p, C.c_int, C.c_uint32, C.c_uint64
        sig = {
            "st_init": (i, [C.POINTER(vp), C.POINTER(st_config)]),
            "st_shutdown": (None, [vp]),
            "st_strerror": (C.c_char_p, [i]),
            "st_last_cuda_error": (C.c_char_p, [vp]),
            "st_get_stream": (vp, [vp]),
            "st_device_bytes_in_use": (u64, [vp]),
            "st_layout_query": (C.c_long, [C.c_char_p]),
            "st_allocate_device_scene": (i, [vp, i, vp]),
            "st_upload_scene": (i, [vp, i, vp]),
            "st_upload_primitives": (i, [vp, i, vp]),
            "st_upload_materials": (i, [vp, i, vp]),
            "st_upload_lights": (i, [vp, i, vp]),
            "st_upload_scene_bvh": (i, [vp, i, vp]),
            "st_upload_mesh_bvhs": (i, [vp, i, vp]),
            "st_update_primitives": (i, [vp, i, vp, vp, u32]),
            "st_free_scene": (i, [vp, i]),
            "st_update_scene_bvh": (i, [vp, i, vp, i]),
            "st_update_mesh_bvh": (i, [vp, vp, i]),
            "st_render_scene": (i, [vp, i, vp, vp]),
            "st_build_bvh": (i, [vp, i, vp, u32, u32, vp, vp, vp, vp]),
            "st_validate_bvh": (i, [vp, u32, u32, u32]),
            "st_build_lbvh_noalloc": (i, [vp, vp, u32, u32, vp, vp, vp, vp, vp]),
            "st_render_ex": (i, [vp, i, vp, vp, C.POINTER(st_render_options)]),
            "st_render_batch": (i, [vp, vp, i, C.POINTER(st_batch_options)]),
            "st_pick": (i, [vp, i, vp, vp, i, i, C.POINTER(st_pick_result)]),
            "st_serve_start": (i, [vp, C.POINTER(st_serve_config)]),
            "st_submit": (i, [vp, C.POINTER(st_request), C.POINTER(u64)]),
            "st_poll": (i, [vp, u64, C.POINTER(st_result)]),
            "st_wait": (i, [vp, u64, C.POINTER(st_result), C.c_double]),
            "st_serve_stop": (i, [vp]),
            "st_clock": (C.c_double, []),
            "st_texture_bytes": (u64, [C.c_uint16, C.c_uint16, i]),
            "st_bake_texture": (i, [vp, vp, C.c_uint16, C.c_uint16, i, i, i, vp, vp, u64]),
            "st_mesh_file_bytes": (C.c_int64, [C.c_char_p]),
            "st_read_mesh_file": (i, [C.c_char_p, vp, vp, u64]),
            "st_write_mesh_file": (i, [C.c_char_p, vp]),
            "st_texture_file_bytes": (C.c_int64, [C.c_char_p]),
            "st_read_texture_file": (i, [C.c_char_p, vp, vp, u64]),
            "st_write_texture_file": (i, [C.c_char_p, vp]),
            "st_read_scene_file": (i, [C.c_char_p, vp, u32, u32]),
            "st_write_scene_file": (i, [C.c_char_p, vp]),
            "st_obj_mesh_bytes": (C.c_int64, [C.c_char_p]),
            "st_obj_to_mesh": (i, [vp, C.c_char_p, i, i, vp, vp, u64]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_functions(header=os.path.join(os.path.dirname(HERE), "include", "slimtracin_b200.h")):
    """Names of the functions the public header declares."""
    import re
    text = open(header).read()
    return sorted(set(re.findall(r"ST_API[^;(]*?\b(st_[a-z_0-9]+)\s*\(", text)))


class Renderer:
    """One library context on one GPU."""

    def __init__(self, device=0, memory_budget=0, max_scenes=16):
        self.L = lib()
        self.ctx = C.c_void_p()
        cfg = st_config(device, memory_budget, max_scenes, 0)
        self._check(self.L.st_init(C.byref(self.ctx), C.byref(cfg)), "st_init")
        self._keep = {}

    def _check(self, status, what):
        if status != ST_OK:
            detail = ""
            if getattr(self, "ctx", None) and self.ctx:
                detail = self.L.st_last_cuda_error(self.ctx).decode()
            raise STError(status, what, detail)

    def close(self):
        if self.ctx:
            self.L.st_shutdown(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    @property
    def stream(self):
        return self.L.st_get_stream(self.ctx)

    # -- residency ---------------------------------------------------------------------------------
    def upload(self, slot, sd, tlas="host"):
        """Upload a SceneData: scene arrays, mesh BLASes (as built) and the TLAS.
        tlas: "host" (sd.tlas_* as given), "lbvh" (build on the device) or None."""
        sc, keep = sd.to_ctypes()
        self._keep[slot] = (sc, keep, sd)
        self._check(self.L.st_upload_scene(self.ctx, slot, C.byref(sc)), "st_upload_scene")
        if sd.meshes:
            self._check(self.L.st_upload_mesh_bvhs(self.ctx, slot, C.byref(sc)), "st_upload_mesh_bvhs")
        if tlas == "host":
            self._check(self.L.st_upload_scene_bvh(self.ctx, slot, C.byref(sc)), "st_upload_scene_bvh")
        elif tlas == "lbvh":
            self.build_tlas(slot, sd, ST_BVH_LBVH30)
        return sc

    def build_tlas(self, slot, sd, mode=ST_BVH_LBVH30):
        sc, keep = sd.to_ctypes()
        self._check(self.L.st_update_scene_bvh(self.ctx, slot, C.byref(sc), mode), "st_update_scene_bvh")
        sd.read_back_tlas(sc)
        return sd

    def build_blas(self, md, mode=ST_BVH_LBVH30):
        """Build a MeshData's BLAS on the device (updateMeshBVH); fills md.nodes/leaf_ids/triangles."""
        keep = []
        md.allocate_bvh()
        m = md.to_ctypes(keep)
        self._check(self.L.st_update_mesh_bvh(self.ctx, C.byref(m), mode), "st_update_mesh_bvh")
        md.read_back(m)
        return md

    def update_primitives(self, slot, prims, ids):
        prims = np.ascontiguousarray(prims, dtype=S.PRIMITIVE_DT)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        self._check(self.L.st_update_primitives(self.ctx, slot, prims.ctypes.data, ids.ctypes.data, len(ids)),
                    "st_update_primitives")

    def build_lbvh(self, boxes, max_leaf, mode=ST_BVH_LBVH30):
        """A device BVH over caller boxes (n x 6 float32): returns codes, order, nodes, node_count,
        height (codes only for LBVH30)."""
        boxes = np.ascontiguousarray(boxes, dtype=np.float32)
        n = len(boxes)
        codes, order = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        nodes, info = np.zeros(2 * n, dtype=S.BVHNODE_DT), np.zeros(2, np.uint32)
        self._check(self.L.st_build_bvh(self.ctx, mode, boxes.ctypes.data, n, max_leaf, codes.ctypes.data,
                                        order.ctypes.data, nodes.ctypes.data, info.ctypes.data), "st_build_bvh")
        return codes, order, nodes[:info[0]], int(info[0]), int(info[1])

    def pick(self, slot, sd, frame, x, y):
        """st_pick: what a click at pixel (x, y) of the frame's viewport selects."""
        sc, keep = sd.to_ctypes()
        res = st_pick_result()
        self._check(self.L.st_pick(self.ctx, slot, C.byref(sc), C.byref(frame.viewport), x, y, C.byref(res)), "st_pick")
        return res

    def free(self, slot):
        self._check(self.L.st_free_scene(self.ctx, slot), "st_free_scene")
        self._keep.pop(slot, None)

    # -- render --------------------------------------------------------------------------------------
    def render(self, slot, sd, frame, prim_ids=None, count_work=False, skip_float_copy=False, overlays=0):
        """st_render_ex into the frame's host buffers; returns the options struct (timings,
        counters).  overlays: OVERLAY_BVH | OVERLAY_SSB draws drawBVH / drawSSB over the frame."""
        sc, keep = sd.to_ctypes()
        opt = st_render_options()
        if prim_ids is not None:
            opt.out_prim_id = prim_ids.ctypes.data
        opt.count_work = int(count_work)
        opt.skip_float_copy = int(skip_float_copy)
        opt.overlays = int(overlays)
        self._check(self.L.st_render_ex(self.ctx, slot, C.byref(sc), C.byref(frame.viewport), C.byref(opt)),
                    "st_render_ex")
        return opt

    def render_device(self, slot, sd, frame, out_float_ptr, out_u8_ptr=None, stream=None):
        """st_render_ex with device-resident outputs (no host copies inside the call)."""
        sc, keep = sd.to_ctypes()
        opt = st_render_options()
        opt.device_outputs = 1
        opt.out_float = out_float_ptr
        opt.out_u8 = out_u8_ptr
        opt.stream = stream
        self._check(self.L.st_render_ex(self.ctx, slot, C.byref(sc), C.byref(frame.viewport), C.byref(opt)),
                    "st_render_ex")
        return opt


def render_batch(renderer, items, tile_shape=-1, chunk=0, use_graph=False, device_outputs=False, stack_placement=-1,
                 launch_mode=LAUNCH_AUTOTUNED, compaction_threshold=0):
    """st_render_batch over items = [(slot, SceneData, Frame)]; outputs go to each Frame's buffers
    (host) unless device_outputs, in which case Frame.grid pointers are used as device pointers."""
    keep = []
    views = (st_view * len(items))()
    for k, (slot, sd, fr) in enumerate(items):
        sc, kk = sd.to_ctypes()
        keep += [sc, kk]
        views[k].slot = slot
        views[k].scene = C.addressof(sc)
        views[k].viewport = C.addressof(fr.viewport)
        views[k].out_float = fr.grid.float_pixels
        views[k].out_u8 = fr.grid.pixels
    opt = st_batch_options()
    opt.tile_shape, opt.chunk, opt.use_graph, opt.device_outputs = tile_shape, chunk, int(use_graph), int(device_outputs)
    opt.stack_placement = stack_placement
    opt.launch_mode = launch_mode
    opt.compaction_threshold = compaction_threshold
    renderer._check(renderer.L.st_render_batch(renderer.ctx, views, len(items), C.byref(opt)), "st_render_batch")
    return opt


def counters_dict(opt):
    return {k: int(opt.counters[i]) for i, k in enumerate(COUNTER_NAMES)}


class Server:
    """The serving loop of a Renderer (st_serve_start .. st_serve_stop): requests are views of resident
    scenes, optionally carrying transform updates that apply before the view renders.  While it runs,
    the Renderer takes no other calls."""

    def __init__(self, renderer, max_in_flight=3, max_views_per_batch=64, frame_budget=0, tile_shape=-1, chunk=0,
                 refit_fraction=0.25, launch_mode=LAUNCH_PER_VIEW):
        self.r = renderer
        self.L = renderer.L
        cfg = st_serve_config(max_in_flight, max_views_per_batch, frame_budget, tile_shape, chunk, refit_fraction,
                              launch_mode)
        renderer._check(self.L.st_serve_start(renderer.ctx, C.byref(cfg)), "st_serve_start")
        self._keep = {}
        self.running = True

    def submit(self, slot, sd, frame, moved=None, moved_ids=None, arrival_time=None):
        """Queue a view; `moved` (PRIMITIVE_DT records) replaces primitives `moved_ids` before it renders.
        The frame's host buffers receive the outputs; they stay referenced until the request completes."""
        sc, kk = sd.to_ctypes()
        req = st_request()
        req.view.slot = slot
        req.view.scene = C.addressof(sc)
        req.view.viewport = C.addressof(frame.viewport)
        req.view.out_float = frame.grid.float_pixels
        req.view.out_u8 = frame.grid.pixels
        keep = [sc, kk, frame]
        if moved is not None and len(moved):
            arr = np.ascontiguousarray(moved, dtype=S.PRIMITIVE_DT)
            ids = np.ascontiguousarray(moved_ids, dtype=np.uint32)
            req.moved, req.moved_ids, req.moved_count = arr.ctypes.data, ids.ctypes.data, len(ids)
            keep += [arr, ids]
        req.arrival_time = self.L.st_clock() if arrival_time is None else arrival_time
        t = C.c_uint64()
        self.r._check(self.L.st_submit(self.r.ctx, C.byref(req), C.byref(t)), "st_submit")
        self._keep[t.value] = keep
        return t.value

    def poll(self, ticket):
        """The st_result of a finished request, or None while it is still running."""
        res = st_result()
        s = self.L.st_poll(self.r.ctx, ticket, C.byref(res))
        if s == ST_ERR_NOT_READY:
            return None
        self.r._check(s, "st_poll")
        self._keep.pop(ticket, None)
        return res

    def wait(self, ticket, timeout=60.0):
        res = st_result()
        self.r._check(self.L.st_wait(self.r.ctx, ticket, C.byref(res), float(timeout)), "st_wait")
        self._keep.pop(ticket, None)
        return res

    def stop(self):
        if self.running:
            self.r._check(self.L.st_serve_stop(self.r.ctx), "st_serve_stop")
            self.running = False
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()
        return False


def clock():
    return lib().st_clock()
