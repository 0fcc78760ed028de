"""Shared test helpers: run the oracle / the reference harness on SceneData and compare frames."""
import ctypes as C

import numpy as np

import oracle
from slimtracin_b200 import scenes, structs as S


def tlas_sah(sd, which="orc"):
    """The reference's top-down SAH TLAS (updateSceneBVH) via the oracle or the reference itself."""
    sc, keep = sd.to_ctypes()
    if which == "orc":
        oracle.restatement().orc_update_scene_bvh(C.byref(sc))
    else:
        oracle.reference().ref_update_scene_bvh(C.byref(sc))
    sd.read_back_tlas(sc)
    return sd


def blas_sah(md, which="orc"):
    """The reference's BLAS build (updateMeshBVH) into md via the oracle or the reference;
    which="binned": the oracle's updateMeshBVH with the binned-SAH topology (the library's
    ST_BVH_BINNED_SAH build)."""
    keep = []
    md.allocate_bvh()
    m = md.to_ctypes(keep)
    if which == "orc":
        oracle.restatement().orc_update_mesh_bvh(C.byref(m))
    elif which == "binned":
        assert oracle.restatement().orc_update_mesh_bvh_binned(C.byref(m)) == 0
    else:
        oracle.reference().ref_update_mesh_bvh(C.byref(m))
    md.read_back(m)
    return md


def tlas_lbvh(sd):
    """The scene's TLAS as the library's ST_BVH_LBVH30 builds it (the oracle's LBVH30 over the
    primitives' world boxes, leaves of at most 2), written into sd's BVH arrays."""
    orc = oracle.restatement()
    sc, keep = sd.to_ctypes()
    n = len(sd.primitives)
    boxes = np.zeros((n, 6), np.float32)
    orc.orc_primitive_aabbs(C.byref(sc), boxes.ctypes.data)
    codes, order = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    nodes, info = np.zeros(2 * n, dtype=S.BVHNODE_DT), np.zeros(2, np.uint32)
    leaf = np.zeros(n, np.uint32)
    orc.orc_lbvh30(boxes.ctypes.data, n, 2, codes.ctypes.data, order.ctypes.data, nodes.ctypes.data,
                   leaf.ctypes.data, info.ctypes.data)
    sd.tlas_nodes[:info[0]] = nodes[:info[0]]
    sd.tlas_leaf_ids[:n] = leaf
    sd.tlas_node_count, sd.tlas_height = int(info[0]), int(info[1])
    return sd


def tlas_binned(sd):
    """The scene's TLAS as the library's ST_BVH_BINNED_SAH builds it (the oracle's binned SAH over
    the primitives' world boxes, leaves of at most 2), written into sd's BVH arrays."""
    orc = oracle.restatement()
    sc, keep = sd.to_ctypes()
    n = len(sd.primitives)
    boxes = np.zeros((n, 6), np.float32)
    orc.orc_primitive_aabbs(C.byref(sc), boxes.ctypes.data)
    order = np.zeros(n, np.uint32)
    nodes, info = np.zeros(2 * n, dtype=S.BVHNODE_DT), np.zeros(2, np.uint32)
    orc.orc_binned_sah(boxes.ctypes.data, n, 2, order.ctypes.data, nodes.ctypes.data, info.ctypes.data)
    sd.tlas_nodes[:info[0]] = nodes[:info[0]]
    sd.tlas_leaf_ids[:n] = order
    sd.tlas_node_count, sd.tlas_height = int(info[0]), int(info[1])
    return sd


def same_tlas(a, b):
    """Two scenes hold byte-identical TLAS node arrays and leaf lists."""
    n = len(a.primitives)
    return (a.tlas_node_count == b.tlas_node_count and a.tlas_height == b.tlas_height
            and a.tlas_nodes[:a.tlas_node_count].tobytes() == b.tlas_nodes[:b.tlas_node_count].tobytes()
            and np.array_equal(a.tlas_leaf_ids[:n], b.tlas_leaf_ids[:n]))


def cone_angle_for(height, focal_length):
    """The ray-cone spread angle of one pixel row: atan(2 / (H * focal_length))."""
    import math
    return float(np.float32(math.atan(2.0 / (height * focal_length))))


def oracle_frame(sd, cam, w, h, depth=2, mode=S.RM_BEAUTY, cone_angle=0.0, threads=None, counters=False):
    """The oracle's render: SSB update on a copy of the primitives, then the frame."""
    import os
    threads = threads or min(os.cpu_count() or 1, 64)
    orc = oracle.restatement()
    d = sd.copy()
    sc, keep = d.to_ctypes()
    fr = scenes.Frame(w, h, cam, depth=depth, mode=mode, cone_angle=cone_angle)
    orc.orc_update_scene_ssb(C.byref(sc), C.byref(fr.viewport))
    ids = np.zeros(fr.rays, dtype=np.uint32)
    cnt = np.zeros(16, dtype=np.uint64)
    orc.orc_render_frame(C.byref(sc), C.byref(fr.viewport), threads, ids.ctypes.data, cnt.ctypes.data)
    fr.prim_ids = ids
    fr.counters = cnt
    return fr


def reference_frame(sd, cam, w, h, depth=2, mode=S.RM_BEAUTY, cone_angle=0.0, threads=8):
    """The reference's own render of the same scene (updateSceneSSB, beginDrawing, rayTrace per
    pixel, drawViewportToWindowContent)."""
    ref = oracle.reference()
    d = sd.copy()
    sc, keep = d.to_ctypes()
    fr = scenes.Frame(w, h, cam, depth=depth, mode=mode, cone_angle=cone_angle)
    ref.ref_update_scene_ssb(C.byref(sc), C.byref(fr.viewport))
    ref.ref_begin_drawing(C.byref(fr.viewport))
    fr.viewport.projection_plane.cone_angle = np.float32(cone_angle)
    ref.ref_render_rows(C.byref(sc), C.byref(fr.viewport), threads, 0, 1, fr.grid_h)
    ref.ref_resolve(C.byref(fr.viewport))
    return fr


def gpu_frame(renderer, slot, sd, cam, w, h, depth=2, mode=S.RM_BEAUTY, cone_angle=0.0, counters=False, overlays=0):
    fr = scenes.Frame(w, h, cam, depth=depth, mode=mode, cone_angle=cone_angle)
    ids = np.zeros(fr.rays, dtype=np.uint32)
    opt = renderer.render(slot, sd, fr, prim_ids=ids, count_work=counters, overlays=overlays)
    fr.prim_ids = ids
    fr.options = opt
    fr.counters = np.array([opt.counters[k] for k in range(16)], dtype=np.uint64)
    return fr


def compare(a, b, mode):
    """Parity figures of two frames of the same view.
    exact        fraction of grid points whose FloatPixel bytes are identical
    id_match     fraction of grid points with the same primary-hit primitive id (when both have ids)
    u8_within1   fraction of resolved pixels whose RGB differ by at most 1 in every channel
    max_rel      largest relative difference of sqrt(color) over points both sides hit"""
    fa, fb = a.float_pixels, b.float_pixels
    out = {"exact": float((fa.view(np.uint8).reshape(-1, 24) == fb.view(np.uint8).reshape(-1, 24)).all(1).mean())}
    if getattr(a, "prim_ids", None) is not None and getattr(b, "prim_ids", None) is not None:
        out["id_match"] = float((a.prim_ids == b.prim_ids).mean())
    pa = a.pixels.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
    pb = b.pixels.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
    out["u8_within1"] = float((np.abs(pa - pb).max(1) <= 1).mean())
    out["u8_max"] = int(np.abs(pa - pb).max()) if len(pa) else 0
    both = np.isfinite(fa["depth"]) & np.isfinite(fb["depth"])
    ca = np.sqrt(fa["color"][both].astype(np.float64)) / 255.0
    cb = np.sqrt(fb["color"][both].astype(np.float64)) / 255.0
    rel = np.abs(ca - cb) / np.maximum(np.abs(ca), 1e-3)
    out["max_rel"] = float(rel.max()) if rel.size else 0.0
    out["rel_ok"] = float((rel.max(1) <= 1e-4).mean()) if rel.size else 1.0
    out["hit_agree"] = float((np.isfinite(fa["depth"]) == np.isfinite(fb["depth"])).mean())
    return out


def assert_parity(m, mode, id_min=0.9999, u8_min=0.999, rel_min=0.999):
    """The stated tolerances: primary-hit ids on >= 99.99% of grid points, beauty RGB within 1/255
    on >= 99.9% of pixels, depth/normal/UV within 1e-4 relative on >= 99.9% of hit points."""
    if "id_match" in m:
        assert m["id_match"] >= id_min, m
    if mode == S.RM_BEAUTY:
        assert m["u8_within1"] >= u8_min, m
    else:
        assert m["rel_ok"] >= rel_min, m
        assert m["u8_within1"] >= u8_min, m


def small_mesh_scene(subdivisions=3, texture_size=64, blas="orc"):
    """The mesh scene at test scale: a small displaced icosphere, 64^2 textures, the same 8 instances,
    materials and emissive quads."""
    sd, cam = scenes.mesh_scene(subdivisions=subdivisions, texture_size=texture_size)
    if blas in ("orc", "ref"):
        blas_sah(sd.meshes[0], blas)
    return sd, cam


def picks(sd, cam, w, h, coords, which="orc"):
    """The selection a click at each (x, y) makes, by the oracle ("orc") or by the reference's own
    picking sequence ("ref"), after the SSB update of the view.  Returns st_pick_result records."""
    from slimtracin_b200 import api
    lib = oracle.restatement() if which == "orc" else oracle.reference()
    d = sd.copy()
    sc, keep = d.to_ctypes()
    fr = scenes.Frame(w, h, cam, with_pixels=False, with_float=False)
    (lib.orc_update_scene_ssb if which == "orc" else lib.ref_update_scene_ssb)(C.byref(sc), C.byref(fr.viewport))
    fn = lib.orc_pick if which == "orc" else lib.ref_pick
    out = []
    for x, y in coords:
        r = api.st_pick_result()
        fn(C.byref(sc), C.byref(fr.viewport), int(x), int(y), C.byref(r))
        out.append(r)
    return out


def pick_key(r):
    """Every field of a pick result as exact bits."""
    import struct
    return (r.found, r.object_type, r.object_id, struct.pack("5f", *r.position, r.distance, r.object_distance))


def light_coords(sd, cam, w, h, step=2):
    """Pixels whose picking ray hits a light's glow sphere (scanned with the oracle)."""
    coords = [(x, y) for y in range(0, h, step) for x in range(0, w, step)]
    return [c for c, r in zip(coords, picks(sd, cam, w, h, coords)) if r.found and r.object_type == 6]


def overlay_frame(sd, cam, w, h, what, which="orc", depth=1, mode=S.RM_BEAUTY):
    """The oracle's render of the view with the debug overlays (what: 1 = drawBVH, 2 = drawSSB)
    drawn over it by the oracle ("orc") or by the reference's own drawBVH/drawSSB ("ref").
    Returns the Frame; its float grid holds the overlaid pixels and `base` the render under them."""
    fr = oracle_frame(sd, cam, w, h, depth=depth, mode=mode)
    fr.base = fr.float_pixels.copy()
    lib = oracle.restatement() if which == "orc" else oracle.reference()
    d = sd.copy()
    sc, keep = d.to_ctypes()
    (lib.orc_update_scene_ssb if which == "orc" else lib.ref_update_scene_ssb)(C.byref(sc), C.byref(fr.viewport))
    if which == "orc":
        lib.orc_draw_overlays(C.byref(sc), C.byref(fr.viewport), what)
    else:
        assert lib.ref_draw_overlays(C.byref(sc), C.byref(fr.viewport), what) == 0
    return fr


def overlay_scene(which):
    """Scenes of the overlay tests: the 16-primitive scene, the area-light example, the mesh scene at test scale (reference
    BLAS), cameras inside them (edges cut by the near and side planes), and 384 primitives (a TLAS
    past the reference's 255-node drawBVH limit)."""
    if which in ("implicit16", "inside"):
        sd, cam = scenes.implicit16_scene()
    elif which == "area":
        sd, cam = scenes.example_area_lights()
    elif which == "moving":
        sd, cam = scenes.moving_scene(count=384, spread=6.0)
    else:
        sd, cam = small_mesh_scene(subdivisions=3, texture_size=64, blas="ref" if oracle.reference_available() else "orc")
    if which == "inside":
        cam = scenes.CameraSpec((0.5, 0.3, -1.0), 0.4, 0.2, 2.0)
    elif which == "inside_mesh":
        cam = scenes.look_at((1.0, 1.5, -3.0), (0.0, 1.0, 4.0))
    return sd, cam
