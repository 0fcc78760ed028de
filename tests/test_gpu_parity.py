"""Device path vs the oracle, called through the C ABI (libslimtracin_b200.so)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from slimtracin_b200 import api, scenes, structs as S
from tests import helpers as H

pytestmark = pytest.mark.gpu

MODES = [S.RM_BEAUTY, S.RM_DEPTH, S.RM_NORMALS, S.RM_UVS]


@pytest.mark.parametrize("mode", MODES)
def test_implicit16_all_modes(renderer, mode):
    sd, cam = scenes.implicit16_scene()
    H.tlas_sah(sd)
    renderer.upload(0, sd, tlas="host")
    g = H.gpu_frame(renderer, 0, sd, cam, 640, 480, depth=2, mode=mode)
    o = H.oracle_frame(sd, cam, 640, 480, depth=2, mode=mode)
    m = H.compare(g, o, mode)
    print("implicit16", mode, m)
    H.assert_parity(m, mode)
    if mode != S.RM_BEAUTY:
        # no libm call on these paths: every byte equals the oracle's
        assert m["exact"] == 1.0, m


@pytest.mark.parametrize("depth", [1, 3])
def test_point_and_area_lights(renderer, depth):
    """06_AreaLights: point lights and emissive quads together, so the shadow rays' overwrite of the
    closest hit reaches the emissive-quad test (surface.h:14-17,55)."""
    sd, cam = scenes.example_area_lights()
    H.tlas_sah(sd)
    renderer.upload(1, sd, tlas="host")
    g = H.gpu_frame(renderer, 1, sd, cam, 320, 240, depth=depth)
    o = H.oracle_frame(sd, cam, 320, 240, depth=depth)
    m = H.compare(g, o, S.RM_BEAUTY)
    print("area", depth, m)
    H.assert_parity(m, S.RM_BEAUTY)


@pytest.mark.parametrize("mode", [S.RM_BEAUTY, S.RM_NORMALS, S.RM_UVS])
def test_mesh_scene_small_reference_blas(renderer, mode):
    """Meshes, Cook-Torrance, glass and mirror bounces, textures, emissive quads, BLAS from the
    reference's SAH builder."""
    sd, cam = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(sd)
    renderer.upload(2, sd, tlas="host")
    g = H.gpu_frame(renderer, 2, sd, cam, 320, 180, depth=4, mode=mode)
    o = H.oracle_frame(sd, cam, 320, 180, depth=4, mode=mode)
    m = H.compare(g, o, mode)
    print("mesh-small", mode, m)
    H.assert_parity(m, mode)


@pytest.mark.parametrize("mode", [api.ST_BVH_LBVH30, api.ST_BVH_BINNED_SAH])
def test_point_and_area_lights_device_tlas(renderer, mode):
    """Point lights and emissive quads together under a TLAS built on the device: which occluder a
    shadow ray finds first, and so the closest-hit record the emissive-quad test reads afterwards
    (surface.h:14-17,55), depends on the tree's topology; given the same tree the oracle's frame and
    work counters are the device's."""
    sd, cam = scenes.example_area_lights()
    renderer.upload(1, sd, tlas=None)
    renderer.build_tlas(1, sd, mode)
    for depth in (1, 3):
        g = H.gpu_frame(renderer, 1, sd, cam, 320, 240, depth=depth, counters=True)
        o = H.oracle_frame(sd, cam, 320, 240, depth=depth)
        m = H.compare(g, o, S.RM_BEAUTY)
        print("area, device TLAS", mode, depth, m)
        assert np.array_equal(g.counters[:11], o.counters[:11]), (g.counters[:11], o.counters[:11])
        H.assert_parity(m, S.RM_BEAUTY)


def test_counters_match_oracle(renderer):
    """Same traversal, same work: every event counter equals the oracle's."""
    sd, cam = H.small_mesh_scene(subdivisions=2, texture_size=32, blas="orc")
    H.tlas_sah(sd)
    renderer.upload(3, sd, tlas="host")
    g = H.gpu_frame(renderer, 3, sd, cam, 160, 90, depth=4, counters=True)
    o = H.oracle_frame(sd, cam, 160, 90, depth=4)
    print("gpu", g.counters[:11], "oracle", o.counters[:11])
    assert np.array_equal(g.counters[:11], o.counters[:11])
    sd0, cam0 = scenes.example_area_lights()
    H.tlas_sah(sd0)
    renderer.upload(3, sd0, tlas="host")
    g = H.gpu_frame(renderer, 3, sd0, cam0, 160, 120, depth=2, counters=True)
    o = H.oracle_frame(sd0, cam0, 160, 120, depth=2)
    assert np.array_equal(g.counters[:11], o.counters[:11]), (g.counters[:11], o.counters[:11])


def test_moving_scene_primary_tlas(renderer):
    """Hundreds of primitives: primary rays walk the TLAS with the SSB cull instead of the
    reference's brute-force loop; results must not change."""
    sd, cam = scenes.moving_scene(count=384, spread=6.0)
    H.tlas_sah(sd)
    renderer.upload(4, sd, tlas="host")
    g = H.gpu_frame(renderer, 4, sd, cam, 320, 180, depth=2)
    o = H.oracle_frame(sd, cam, 320, 180, depth=2)
    m = H.compare(g, o, S.RM_BEAUTY)
    print("moving-384", m)
    H.assert_parity(m, S.RM_BEAUTY)


def test_lbvh_tlas_bit_exact(renderer):
    """The device LBVH30 TLAS: node array, leaf order and height equal the oracle's specification."""
    orc = oracle.restatement()
    for count in (2, 3, 16, 384, 4096):
        sd, cam = scenes.moving_scene(count=count)
        renderer.upload(5, sd, tlas=None)
        renderer.build_tlas(5, sd, api.ST_BVH_LBVH30)
        sc, keep = sd.to_ctypes()
        n = count
        boxes = np.zeros(6 * n, dtype=np.float32)
        orc.orc_primitive_aabbs(C.byref(sc), boxes.ctypes.data)
        codes = np.zeros(n, np.uint32)
        order = np.zeros(n, np.uint32)
        nodes = np.zeros(2 * n, dtype=S.BVHNODE_DT)
        leaf = np.zeros(n, np.uint32)
        info = np.zeros(2, np.uint32)
        orc.orc_lbvh30(boxes.ctypes.data, n, 2, codes.ctypes.data, order.ctypes.data, nodes.ctypes.data,
                       leaf.ctypes.data, info.ctypes.data)
        assert sd.tlas_node_count == info[0] and sd.tlas_height == info[1], (count, sd.tlas_node_count, info)
        k = int(info[0])
        assert np.array_equal(sd.tlas_leaf_ids[:n], leaf)
        assert np.array_equal(sd.tlas_nodes[:k].view(np.uint8), nodes[:k].view(np.uint8)), count


def test_render_with_lbvh_tlas(renderer):
    """Any-hit shadow rays take the first occluder found, so with a different TLAS the oracle is
    given the same (device-built) TLAS."""
    sd, cam = scenes.implicit16_scene()
    renderer.upload(6, sd, tlas=None)
    renderer.build_tlas(6, sd, api.ST_BVH_LBVH30)
    g = H.gpu_frame(renderer, 6, sd, cam, 320, 240, depth=2)
    o = H.oracle_frame(sd, cam, 320, 240, depth=2)
    m = H.compare(g, o, S.RM_BEAUTY)
    H.assert_parity(m, S.RM_BEAUTY)


def test_blas_lbvh_triangle_records(renderer):
    """Device BLAS: every Triangle record equals the reference's precompute of the same source
    triangle (builder_top_down.h:330-363), and leaf_ids is the inverse of the leaf order."""
    md = scenes.displaced_icosphere(4, seed=7)
    renderer.build_blas(md)
    ref = scenes.displaced_icosphere(4, seed=7)
    H.blas_sah(ref, "orc")
    # map each leaf-ordered slot back to its source triangle through leaf_ids (source -> slot)
    n = md.triangle_count
    slot_of_src_dev = md.leaf_ids[:n]
    slot_of_src_ref = ref.leaf_ids[:n]
    assert np.array_equal(np.sort(slot_of_src_dev), np.arange(n))
    dev_by_src = md.triangles[slot_of_src_dev]
    ref_by_src = ref.triangles[slot_of_src_ref]
    assert np.array_equal(dev_by_src.view(np.uint8), ref_by_src.view(np.uint8))
    assert md.height + 2 <= 64


def test_render_with_lbvh_blas(renderer):
    sd, cam = H.small_mesh_scene(subdivisions=3, texture_size=64, blas=None)
    renderer.build_blas(sd.meshes[0])
    H.tlas_sah(sd)
    renderer.upload(7, sd, tlas="host")
    g = H.gpu_frame(renderer, 7, sd, cam, 320, 180, depth=4)
    o = H.oracle_frame(sd, cam, 320, 180, depth=4)
    m = H.compare(g, o, S.RM_BEAUTY)
    H.assert_parity(m, S.RM_BEAUTY)


def test_refit_after_motion(renderer):
    sd, cam = scenes.moving_scene(count=256)
    renderer.upload(8, sd, tlas=None)
    renderer.build_tlas(8, sd, api.ST_BVH_LBVH30)
    scenes.advance_moving_scene(sd, 3)
    renderer.update_primitives(8, sd.primitives, np.arange(256))
    renderer.build_tlas(8, sd, api.ST_BVH_REFIT)
    # every leaf box contains its primitives' boxes and every parent contains its children
    nodes = sd.tlas_nodes[:sd.tlas_node_count]
    for i, nd in enumerate(nodes):
        if nd["child_count"] == 0:
            f = nd["first_child_id"]
            for c in (f, f + 1):
                assert np.all(nodes[c]["aabb"][:3] >= nd["aabb"][:3]) and np.all(nodes[c]["aabb"][3:] <= nd["aabb"][3:])
    g = H.gpu_frame(renderer, 8, sd, cam, 256, 144, depth=2)
    o = H.oracle_frame(sd, cam, 256, 144, depth=2)
    H.assert_parity(H.compare(g, o, S.RM_BEAUTY), S.RM_BEAUTY)


def test_layout_matches_reference_headers():
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    L = api.lib()
    ref = oracle.reference()
    import re
    names = re.findall(r"ST_LAYOUT_(?:STRUCT|FIELD)\(([A-Za-z]+)(?:, ([A-Za-z_]+))?\)",
                       open(H.__file__.replace("tests/helpers.py", "include/slimtracin_layout.h")).read())
    for s, f in names:
        q = (s + ("." + f if f else "")).encode()
        assert L.st_layout_query(q) == ref.ref_layout_query(q), q


@pytest.mark.parametrize("n,max_leaf", [(1, 2), (5, 2), (1000, 4), (70000, 4)])
def test_lbvh_codes_order_topology_bit_exact(renderer, n, max_leaf):
    """st_build_lbvh over arbitrary boxes: Morton codes, sort order and node array equal the
    oracle's LBVH30 specification bit for bit (70,000 items exercise multi-block radix passes)."""
    rng = np.random.default_rng(n + 17)
    c = rng.uniform(-50, 50, (n, 3))
    e = rng.uniform(0.01, 2, (n, 3))
    boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
    # duplicated centroids: equal codes are ordered by index
    boxes[n // 2:n // 2 + min(8, n // 2)] = boxes[0]
    codes, order, nodes, count, height = renderer.build_lbvh(boxes, max_leaf)
    orc = oracle.restatement()
    oc, oo = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    on, ol, oi = np.zeros(2 * n, dtype=S.BVHNODE_DT), np.zeros(n, np.uint32), np.zeros(2, np.uint32)
    orc.orc_lbvh30(boxes.ctypes.data, n, max_leaf, oc.ctypes.data, oo.ctypes.data, on.ctypes.data,
                   ol.ctypes.data, oi.ctypes.data)
    assert np.array_equal(codes, oc)
    assert np.array_equal(order, oo)
    assert (count, height) == (int(oi[0]), int(oi[1]))
    assert np.array_equal(nodes.view(np.uint8), on[:count].view(np.uint8))


@pytest.mark.parametrize("n,max_leaf", [(1, 2), (3, 2), (100, 2), (2049, 4), (50000, 4)])
def test_binned_sah_bit_exact(renderer, n, max_leaf):
    """st_build_bvh(ST_BVH_BINNED_SAH): order and node array equal the oracle's binned-SAH
    specification (50,000 items exercise the multi-block large-task path)."""
    rng = np.random.default_rng(n + 3)
    c = rng.uniform(-20, 20, (n, 3))
    e = rng.uniform(0.01, 1.5, (n, 3))
    boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
    boxes[n // 3:n // 3 + min(40, n // 3)] = boxes[0]          # a clump of identical items
    codes, order, nodes, count, height = renderer.build_lbvh(boxes, max_leaf, api.ST_BVH_BINNED_SAH)
    orc = oracle.restatement()
    oo, on, oi = np.zeros(n, np.uint32), np.zeros(2 * n, dtype=S.BVHNODE_DT), np.zeros(2, np.uint32)
    orc.orc_binned_sah(boxes.ctypes.data, n, max_leaf, oo.ctypes.data, on.ctypes.data, oi.ctypes.data)
    assert (count, height) == (int(oi[0]), int(oi[1]))
    assert np.array_equal(order, oo)
    assert np.array_equal(nodes.view(np.uint8), on[:count].view(np.uint8))


def test_binned_sah_tlas_and_blas_render(renderer):
    """A binned-SAH TLAS (4096 moving primitives) and BLAS render like the oracle given the same BVHs."""
    sd, cam = scenes.moving_scene(count=1024)
    renderer.upload(9, sd, tlas=None)
    renderer.build_tlas(9, sd, api.ST_BVH_BINNED_SAH)
    g = H.gpu_frame(renderer, 9, sd, cam, 256, 144, depth=2)
    o = H.oracle_frame(sd, cam, 256, 144, depth=2)
    H.assert_parity(H.compare(g, o, S.RM_BEAUTY), S.RM_BEAUTY)
    sd1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas=None)
    renderer.build_blas(sd1.meshes[0], api.ST_BVH_BINNED_SAH)
    renderer.upload(10, sd1, tlas=None)
    renderer.build_tlas(10, sd1, api.ST_BVH_BINNED_SAH)
    g = H.gpu_frame(renderer, 10, sd1, cam1, 320, 180, depth=4)
    o = H.oracle_frame(sd1, cam1, 320, 180, depth=4)
    H.assert_parity(H.compare(g, o, S.RM_BEAUTY), S.RM_BEAUTY)


def test_batch_equals_per_frame_renders(renderer):
    """st_render_batch over views of different scenes, sizes, modes and bounce counts: every view's
    float grid and u8 frame equal the per-frame render's, for every tile shape, with and without
    the CUDA graph (the second graph call replays the captured graph)."""
    c0, cam0 = scenes.implicit16_scene()
    H.tlas_sah(c0)
    renderer.upload(11, c0, tlas="host")
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    renderer.upload(12, c1, tlas="host")
    c2, cam2 = scenes.moving_scene(count=300)
    H.tlas_sah(c2)
    renderer.upload(13, c2, tlas="host")
    specs = [(11, c0, cam0, 96, 64, 2, S.RM_BEAUTY), (12, c1, cam1, 160, 90, 4, S.RM_BEAUTY),
             (13, c2, cam2, 64, 48, 1, S.RM_BEAUTY), (12, c1, cam1, 80, 60, 6, S.RM_NORMALS),
             (11, c0, cam0, 33, 17, 3, S.RM_DEPTH)]
    singles = [H.gpu_frame(renderer, slot, sd, cam, w, h, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
    for tile in (0, 1, 2, 3, -1):
        for stack in (0, 1, -1):
            for graph in (False, True, True):
                frames = [scenes.Frame(w, h, cam, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
                opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)],
                                       tile_shape=tile, use_graph=graph, stack_placement=stack)
                for a, b in zip(frames, singles):
                    assert np.array_equal(a.float_pixels.view(np.uint8), b.float_pixels.view(np.uint8)), (tile, stack, graph)
                    assert np.array_equal(a.pixels.view(np.uint8), b.pixels.view(np.uint8))
                assert opt.rays == sum(fr.rays for fr in frames)
                if tile >= 0:
                    assert opt.tile_shape_used == tile
                if stack >= 0:
                    assert opt.stack_placement_used == stack
    for graph in (False, True, True):        # one trace kernel per view, on concurrent streams
        frames = [scenes.Frame(w, h, cam, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
        opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)], use_graph=graph,
                               launch_mode=api.LAUNCH_PER_VIEW)
        assert opt.launch_mode_used == api.LAUNCH_PER_VIEW
        for a, b in zip(frames, singles):
            assert np.array_equal(a.float_pixels.view(np.uint8), b.float_pixels.view(np.uint8)), ("per view", graph)
            assert np.array_equal(a.pixels.view(np.uint8), b.pixels.view(np.uint8))


def test_pinned_host_outputs_written_by_the_kernels(renderer):
    """Page-locked host buffers are written by the trace and resolve kernels directly (no copy after
    the trace); the frame equals the one rendered into pageable buffers."""
    import torch
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    renderer.upload(14, c1, tlas="host")
    pageable = scenes.Frame(320, 180, cam1, depth=4)
    renderer.render(14, c1, pageable)
    pinned = scenes.Frame(320, 180, cam1, depth=4, with_pixels=False, with_float=False)
    pf = torch.zeros(pinned.rays * 24, dtype=torch.uint8, pin_memory=True)
    pu = torch.zeros(320 * 180 * 4, dtype=torch.uint8, pin_memory=True)
    pinned.grid.float_pixels, pinned.grid.pixels = pf.data_ptr(), pu.data_ptr()
    sc, keep = c1.to_ctypes()
    assert api.lib().st_render_scene(renderer.ctx, 14, C.byref(sc), C.byref(pinned.viewport)) == 0
    assert np.array_equal(pf.numpy(), pageable.float_pixels.view(np.uint8))
    assert np.array_equal(pu.numpy(), pageable.pixels.view(np.uint8))


@pytest.mark.parametrize("w,h", [(1920, 1080), (1283, 721), (4000, 300), (400, 200), (135, 130)])
def test_pinned_outputs_traced_in_strips(renderer, w, h):
    """Page-locked outputs at frame sizes that are traced in column strips (each strip's grid copied
    to the host while later strips trace, its pixels resolved as soon as their columns are done;
    1920 and 4000 wide make eight strips, 1283 six of unequal widths, 400 two, 135 one): float grid
    and frame byte-identical to the same view rendered into pageable buffers, also with the frame
    alone (no float grid)."""
    import torch
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    renderer.upload(14, c1, tlas="host")
    pageable = scenes.Frame(w, h, cam1, depth=4)
    renderer.render(14, c1, pageable)
    sc, keep = c1.to_ctypes()
    for with_float in (True, False):
        pinned = scenes.Frame(w, h, cam1, depth=4, with_pixels=False, with_float=False)
        pf = torch.zeros(pinned.rays * 24, dtype=torch.uint8, pin_memory=True)
        pu = torch.zeros(w * h * 4, dtype=torch.uint8, pin_memory=True)
        pinned.grid.float_pixels = pf.data_ptr() if with_float else None
        pinned.grid.pixels = pu.data_ptr()
        assert api.lib().st_render_scene(renderer.ctx, 14, C.byref(sc), C.byref(pinned.viewport)) == 0
        if with_float:
            assert np.array_equal(pf.numpy(), pageable.float_pixels.view(np.uint8))
        assert np.array_equal(pu.numpy(), pageable.pixels.view(np.uint8)), with_float


def test_strip_traced_render_counts_the_same_work(renderer):
    """A render into page-locked buffers traces the frame in column strips (eight at 1920 wide), each
    strip a launch of its own: the work counters summed over the strips equal those of the same view
    traced in one launch (pageable buffers), which the oracle pins, and the frames are identical."""
    import torch
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    renderer.upload(15, c1, tlas="host")
    w, h = 1920, 1080
    one = H.gpu_frame(renderer, 15, c1, cam1, w, h, depth=4, counters=True)
    strips = scenes.Frame(w, h, cam1, depth=4, with_pixels=False, with_float=False)
    pf = torch.zeros(strips.rays * 24, dtype=torch.uint8, pin_memory=True)
    pu = torch.zeros(w * h * 4, dtype=torch.uint8, pin_memory=True)
    strips.grid.float_pixels = pf.data_ptr()
    strips.grid.pixels = pu.data_ptr()
    opt = renderer.render(15, c1, strips, count_work=True)
    counted = np.array([opt.counters[k] for k in range(16)], dtype=np.uint64)
    assert np.array_equal(counted, one.counters)
    assert counted[0] == strips.rays                     # every grid point traced once
    assert np.array_equal(pf.numpy(), one.float_pixels.view(np.uint8))
    assert np.array_equal(pu.numpy(), one.pixels.view(np.uint8))


@pytest.mark.parametrize("which", ["implicit16", "mesh"])
def test_pick_equals_oracle(renderer, which):
    """st_pick (manipulateSelection's picking ray on the device) equals the oracle's pick bit for bit
    on scattered pixels and on pixels whose ray hits a light's glow sphere."""
    if which == "implicit16":
        sd, cam = scenes.implicit16_scene()
    else:
        sd, cam = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(sd)
    renderer.upload(15, sd, tlas="host")
    w, h = 160, 120
    rng = np.random.default_rng(5)
    coords = [tuple(c) for c in rng.integers(0, [w, h], (80, 2))]
    coords += H.light_coords(sd, cam, w, h)[:10] if len(sd.lights) else []
    fr = scenes.Frame(w, h, cam, with_pixels=False, with_float=False)
    dev = [H.pick_key(renderer.pick(15, sd, fr, int(x), int(y))) for x, y in coords]
    orc = [H.pick_key(r) for r in H.picks(sd, cam, w, h, coords)]
    assert dev == orc
    assert any(k[0] for k in dev)


@pytest.mark.parametrize("which", ["implicit16", "area", "mesh", "inside", "inside_mesh", "moving"])
@pytest.mark.parametrize("what", [1, 2, 3])
def test_overlays_equal_oracle(renderer, which, what):
    """drawBVH / drawSSB (render/raytracer.h:46, render/SSB.h:175) drawn by the device over a
    byte-exact render (normals mode): the float grid equals the oracle's overlaid grid byte for
    byte.  "moving" has 384 primitives, a TLAS past the reference's 255-node drawBVH limit."""
    sd, cam = H.overlay_scene(which)
    H.tlas_sah(sd)
    renderer.upload(4, sd, tlas="host")
    g = H.gpu_frame(renderer, 4, sd, cam, 320, 240, depth=1, mode=S.RM_NORMALS, overlays=what)
    o = H.overlay_frame(sd, cam, 320, 240, what, "orc", depth=1, mode=S.RM_NORMALS)
    touched = np.count_nonzero(o.float_pixels.view(np.uint8).reshape(o.rays, -1)
                               != o.base.view(np.uint8).reshape(o.rays, -1), axis=1)
    print(which, what, "pixels drawn", np.count_nonzero(touched))
    assert np.count_nonzero(touched) > 100
    assert g.float_pixels.tobytes() == o.float_pixels.tobytes()


def test_overlays_over_beauty_add_no_difference(renderer):
    """Over a beauty render (within tolerance of the oracle, not byte-exact), the overlays add no
    difference of their own: every pixel where the overlaid grids differ already differs without
    the overlays."""
    sd, cam = H.overlay_scene("mesh")
    H.tlas_sah(sd)
    renderer.upload(4, sd, tlas="host")
    g0 = H.gpu_frame(renderer, 4, sd, cam, 320, 180, depth=4)
    g = H.gpu_frame(renderer, 4, sd, cam, 320, 180, depth=4, overlays=3)
    o = H.overlay_frame(sd, cam, 320, 180, 3, "orc", depth=4)
    diff = lambda a, b: np.any(a.view(np.uint8).reshape(len(a), -1) != b.view(np.uint8).reshape(len(b), -1), axis=1)
    before = diff(g0.float_pixels, o.base)
    after = diff(g.float_pixels, o.float_pixels)
    assert not np.any(after & ~before)
    assert np.count_nonzero(diff(g.float_pixels, g0.float_pixels)) > 100


def test_render_scene_draws_overlays_from_viewport_settings(renderer):
    """st_render_scene draws drawBVH / drawSSB when viewport->settings.show_BVH / show_SSB are set,
    as st_render_ex does with the overlay bits."""
    sd, cam = H.overlay_scene("implicit16")
    H.tlas_sah(sd)
    renderer.upload(4, sd, tlas="host")
    a = H.gpu_frame(renderer, 4, sd, cam, 200, 150, depth=1, mode=S.RM_NORMALS, overlays=3)
    fr = scenes.Frame(200, 150, cam, depth=1, mode=S.RM_NORMALS)
    fr.viewport.settings.show_BVH = 1
    fr.viewport.settings.show_SSB = 1
    sc, keep = sd.to_ctypes()
    assert renderer.L.st_render_scene(renderer.ctx, 4, C.byref(sc), C.byref(fr.viewport)) == 0
    assert fr.float_pixels.tobytes() == a.float_pixels.tobytes()
    assert np.array_equal(fr.pixels, a.pixels)


def test_graph_replay_follows_new_views(renderer):
    """A batch replayed through its CUDA graph with the same shapes but other cameras renders the
    new views: every launch parameter (view tables, cameras, outputs) comes from the call."""
    c0, cam0 = scenes.implicit16_scene()
    H.tlas_sah(c0)
    renderer.upload(13, c0, tlas="host")
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    renderer.upload(14, c1, tlas="host")
    rng = np.random.default_rng(5)
    for step in range(3):
        specs = [(13, c0, scenes.look_at((rng.uniform(-12, 12), rng.uniform(-2, 6), -15.0), (0, 0, 0)), 96, 64, 2),
                 (14, c1, scenes.look_at((rng.uniform(-10, 10), rng.uniform(1, 6), -14.0), (0, 1.5, 0)), 120, 80, 4)]
        singles = [H.gpu_frame(renderer, slot, sd, cam, w, h, depth=d) for slot, sd, cam, w, h, d in specs]
        frames = [scenes.Frame(w, h, cam, depth=d) for slot, sd, cam, w, h, d in specs]
        opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)], tile_shape=0,
                               stack_placement=0, chunk=1, use_graph=True)
        assert opt.graph_replayed == (1 if step else opt.graph_replayed)
        for a, b in zip(frames, singles):
            assert np.array_equal(a.float_pixels.view(np.uint8), b.float_pixels.view(np.uint8)), step
            assert np.array_equal(a.pixels.view(np.uint8), b.pixels.view(np.uint8)), step


def test_batch_larger_than_one_view_table(renderer):
    """More views than one launch's view table holds (64): the batch runs as several launches and
    every view equals its single render."""
    c0, cam0 = scenes.implicit16_scene()
    H.tlas_sah(c0)
    renderer.upload(15, c0, tlas="host")
    rng = np.random.default_rng(9)
    specs = []
    for k in range(70):
        cam = scenes.look_at((rng.uniform(-12, 12), rng.uniform(-2, 6), -15.0), (0, 0, 0))
        specs.append((15, c0, cam, int(rng.integers(8, 40)), int(rng.integers(8, 30)), int(rng.integers(1, 4))))
    singles = [H.gpu_frame(renderer, slot, sd, cam, w, h, depth=d) for slot, sd, cam, w, h, d in specs]
    frames = [scenes.Frame(w, h, cam, depth=d) for slot, sd, cam, w, h, d in specs]
    opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)], use_graph=False)
    assert opt.rays == sum(fr.rays for fr in frames)
    for a, b in zip(frames, singles):
        assert np.array_equal(a.float_pixels.view(np.uint8), b.float_pixels.view(np.uint8))
        assert np.array_equal(a.pixels.view(np.uint8), b.pixels.view(np.uint8))


@pytest.mark.parametrize("w,h", [(1, 1), (2, 3), (33, 17), (127, 65)])
def test_ragged_viewports(renderer, w, h):
    """Grids that fill no whole block or tile: every edge lane traces the right point, none past it."""
    sd, cam = scenes.implicit16_scene()
    H.tlas_sah(sd)
    renderer.upload(0, sd, tlas="host")
    for mode in (S.RM_NORMALS, S.RM_BEAUTY):
        g = H.gpu_frame(renderer, 0, sd, cam, w, h, depth=2, mode=mode)
        o = H.oracle_frame(sd, cam, w, h, depth=2, mode=mode)
        m = H.compare(g, o, mode)
        H.assert_parity(m, mode)
        if mode != S.RM_BEAUTY:
            assert m["exact"] == 1.0, (w, h, m)


def test_camera_facing_away_misses_everything(renderer):
    """A view with no hit: every grid point keeps the background and infinite depth, as the oracle's."""
    sd, _ = scenes.implicit16_scene()
    H.tlas_sah(sd)
    renderer.upload(0, sd, tlas="host")
    cam = scenes.CameraSpec((0.0, 0.0, -15.0), float(np.pi), 0.0, 2.0)
    g = H.gpu_frame(renderer, 0, sd, cam, 64, 48, depth=3)
    o = H.oracle_frame(sd, cam, 64, 48, depth=3)
    assert not np.isfinite(g.float_pixels["depth"]).any()
    assert g.float_pixels.tobytes() == o.float_pixels.tobytes()
    assert g.pixels.tobytes() == o.pixels.tobytes()


@pytest.mark.parametrize("count", [2, 3, 16, 17, 64, 300, 1024, 4096])
def test_ref_sah_tlas_equals_the_reference_builder(renderer, count):
    """ST_BVH_REF_SAH: the device build of the reference's updateSceneBVH (full-sweep SAH, Lomuto
    quicksort, right-first numbering) gives the oracle's node array, leaf ids and height byte for byte,
    the oracle's own TLAS being pinned to the reference's (test_sah_tlas_matches_golden)."""
    sd, cam = scenes.moving_scene(seed_offset=count, count=count)
    if count == 300:
        sd.primitives["position"][::7] = sd.primitives["position"][0]      # many equal sort keys
    renderer.upload(6, sd, tlas=None)
    renderer.build_tlas(6, sd, api.ST_BVH_REF_SAH)
    ref = sd.copy()
    H.tlas_sah(ref, "orc")
    assert H.same_tlas(sd, ref)
    boxes = np.zeros((count, 6), np.float32)
    sc, keep = sd.to_ctypes()
    oracle.restatement().orc_primitive_aabbs(C.byref(sc), boxes.ctypes.data)
    _, order, nodes, node_count, height = renderer.build_lbvh(boxes, 2, api.ST_BVH_REF_SAH)
    assert (node_count, height) == (ref.tlas_node_count, ref.tlas_height)
    assert nodes.tobytes() == ref.tlas_nodes[:node_count].tobytes()
    assert np.array_equal(order, ref.tlas_leaf_ids[:count])


def test_point_and_area_lights_ref_sah_equal_the_reference(renderer):
    """Point lights and emissive quads under the device REF_SAH TLAS: the frame equals the
    reference's own render (with its own TLAS) within the stated tolerances, the non-libm bytes
    exactly."""
    sd, cam = scenes.example_area_lights()
    renderer.upload(1, sd, tlas=None)
    renderer.build_tlas(1, sd, api.ST_BVH_REF_SAH)
    ref = sd.copy()
    H.tlas_sah(ref, "ref" if oracle.reference_available() else "orc")
    assert H.same_tlas(sd, ref)
    for depth in (1, 3):
        g = H.gpu_frame(renderer, 1, sd, cam, 320, 240, depth=depth)
        r = (H.reference_frame if oracle.reference_available() else H.oracle_frame)(ref, cam, 320, 240, depth=depth)
        m = H.compare(g, r, S.RM_BEAUTY)
        print("area, REF_SAH TLAS vs reference", depth, m)
        H.assert_parity(m, S.RM_BEAUTY)
