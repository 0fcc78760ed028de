"""The oracle (oracle/oracle.c) pinned against the reference's own code and the golden fixtures."""
import ctypes as C
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from slimtracin_b200 import api, scenes, structs as S
from tests import helpers as H
from tests.golden import make_golden as G

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
FRAMES = np.load(os.path.join(os.path.dirname(__file__), "golden", "frames.npz"))
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


@pytest.mark.parametrize("name", sorted(GOLDEN["renders"]))
def test_oracle_reproduces_golden_renders(name):
    """Bit-exact: the oracle's float grid hashes to the reference's, and its u8 frame is equal."""
    g = GOLDEN["renders"][name]
    sd, cam = G.make_scene(g["kind"], "orc")
    assert sha(sd.tlas_nodes[:sd.tlas_node_count]) == g["tlas_sha256"]
    fr = H.oracle_frame(sd, cam, g["w"], g["h"], depth=g["depth"], mode=g["mode"])
    assert sha(fr.float_pixels) == g["float_sha256"], name
    rgb = np.stack([fr.pixels["R"], fr.pixels["G"], fr.pixels["B"]], -1).reshape(g["h"], g["w"], 3)
    assert np.array_equal(rgb, FRAMES[name])


@needs_ref
@pytest.mark.parametrize("case", ["implicit16", "area", "mesh_small", "mesh_small_depth6", "moving320"])
@pytest.mark.parametrize("mode", [S.RM_BEAUTY, S.RM_NORMALS])
def test_oracle_matches_reference_live(case, mode):
    """Larger renders than the fixtures, oracle vs the reference run here, every byte equal."""
    if case == "implicit16":
        sd, cam = scenes.implicit16_scene()
        w, h, depth = 320, 240, 2
    elif case == "area":
        sd, cam = scenes.example_area_lights()
        w, h, depth = 240, 180, 4
    elif case.startswith("mesh_small"):
        sd, cam = scenes.mesh_scene(subdivisions=3, texture_size=64)
        H.blas_sah(sd.meshes[0], "ref")
        w, h, depth = (192, 108, 4) if case == "mesh_small" else (160, 90, 6)
    else:
        sd, cam = scenes.moving_scene(count=320)
        w, h, depth = 128, 72, 2
    H.tlas_sah(sd, "ref")
    r = H.reference_frame(sd, cam, w, h, depth=depth, mode=mode)
    o = H.oracle_frame(sd, cam, w, h, depth=depth, mode=mode)
    assert np.array_equal(r.float_pixels.view(np.uint8), o.float_pixels.view(np.uint8))
    assert np.array_equal(r.pixels.view(np.uint8).reshape(-1, 4)[:, :3], o.pixels.view(np.uint8).reshape(-1, 4)[:, :3])


@needs_ref
@pytest.mark.parametrize("mode", [S.RM_BEAUTY, S.RM_NORMALS])
def test_oracle_matches_reference_with_ray_cones(mode):
    """Ray-cone mip selection (common.h:336, texture.h:32): with projection_plane.cone_angle set to
    atan(2 / (H * focal_length)) the footprint of a hit spans several texels of the 256^2 textures,
    so mips above 0 are sampled; every byte equals the reference's, and the oracle's counters show
    the fetches above mip 0."""
    sd, cam = scenes.mesh_scene(subdivisions=3, texture_size=256)
    H.blas_sah(sd.meshes[0], "ref")
    H.tlas_sah(sd, "ref")
    w, h = 192, 108
    cone = H.cone_angle_for(h, cam.focal_length)
    r = H.reference_frame(sd, cam, w, h, depth=4, mode=mode, cone_angle=cone)
    o = H.oracle_frame(sd, cam, w, h, depth=4, mode=mode, cone_angle=cone)
    assert np.array_equal(r.float_pixels.view(np.uint8), o.float_pixels.view(np.uint8))
    assert np.array_equal(r.pixels.view(np.uint8).reshape(-1, 4)[:, :3], o.pixels.view(np.uint8).reshape(-1, 4)[:, :3])
    fetches, above0 = int(o.counters[8]), int(o.counters[10])
    assert fetches > 0 and 0 < above0 <= fetches, (fetches, above0)
    # the same view without the cone samples mip 0 only, and looks different
    o0 = H.oracle_frame(sd, cam, w, h, depth=4, mode=mode)
    assert int(o0.counters[10]) == 0
    assert not np.array_equal(o0.float_pixels.view(np.uint8), o.float_pixels.view(np.uint8))


@needs_ref
@pytest.mark.parametrize("w,h,yaw", [(1, 1, 0.0), (2, 3, 0.0), (33, 17, 0.0), (127, 65, 0.0), (64, 48, float(np.pi))])
def test_oracle_matches_reference_ragged_and_empty_views(w, h, yaw):
    """Grids smaller than a block or tile, and a camera facing away from every primitive."""
    sd, cam = scenes.implicit16_scene()
    cam = scenes.CameraSpec(cam.position, yaw, cam.pitch, cam.focal_length)
    H.tlas_sah(sd, "ref")
    for mode in (S.RM_BEAUTY, S.RM_NORMALS):
        r = H.reference_frame(sd, cam, w, h, depth=3, mode=mode)
        o = H.oracle_frame(sd, cam, w, h, depth=3, mode=mode)
        assert np.array_equal(r.float_pixels.view(np.uint8), o.float_pixels.view(np.uint8)), (w, h, yaw, mode)
        assert np.array_equal(r.pixels.view(np.uint8), o.pixels.view(np.uint8)), (w, h, yaw, mode)


@pytest.mark.parametrize("kind", sorted(GOLDEN["tlas"]))
def test_sah_tlas_matches_golden(kind):
    g = GOLDEN["tlas"][kind]
    sd, _ = G.make_scene(kind, "orc")
    assert sd.tlas_node_count == g["node_count"] and sd.tlas_height == g["height"]
    assert sha(sd.tlas_nodes[:sd.tlas_node_count]) == g["nodes_sha256"]
    assert sha(sd.tlas_leaf_ids) == g["leaf_ids_sha256"]


@needs_ref
@pytest.mark.parametrize("sub", [2, 3, 4])
def test_sah_blas_matches_reference(sub):
    a = H.blas_sah(scenes.displaced_icosphere(sub, seed=11), "orc")
    b = H.blas_sah(scenes.displaced_icosphere(sub, seed=11), "ref")
    assert (a.node_count, a.height) == (b.node_count, b.height)
    assert np.array_equal(a.nodes[:a.node_count].view(np.uint8), b.nodes[:b.node_count].view(np.uint8))
    assert np.array_equal(a.leaf_ids, b.leaf_ids)
    assert np.array_equal(a.triangles.view(np.uint8), b.triangles.view(np.uint8))


@needs_ref
def test_monkey_mesh_golden():
    """The one fixture the reference ships: rebuilding monkey.mesh's BLAS from its own vertex data
    reproduces the stored nodes, leaf ids and Triangle records byte for byte."""
    if not os.path.exists(G.MONKEY) or GOLDEN["monkey"] is None:
        pytest.skip("monkey.mesh not present")
    ref = oracle.reference()
    m = S.Mesh()
    arena = ref.ref_load_mesh(G.MONKEY.encode(), C.byref(m))
    g = GOLDEN["monkey"]
    t, v = m.triangle_count, m.vertex_count
    assert (t, v, m.bvh.node_count, m.bvh.height) == (g["triangles"], g["vertices"], g["node_count"], g["height"])

    def arr(ptr, n, dt, shape):
        return np.ctypeslib.as_array((C.c_uint8 * (n * np.dtype(dt).itemsize)).from_address(ptr)).view(dt).reshape(shape).copy()

    md = scenes.MeshData(arr(m.vertex_positions, 3 * v, np.float32, (v, 3)),
                         arr(m.vertex_normals, 3 * m.normals_count, np.float32, (m.normals_count, 3)),
                         arr(m.vertex_uvs, 2 * m.uvs_count, np.float32, (m.uvs_count, 2)),
                         arr(m.vertex_position_indices, 3 * t, np.uint32, (t, 3)),
                         np.array([m.aabb.min.x, m.aabb.min.y, m.aabb.min.z, m.aabb.max.x, m.aabb.max.y, m.aabb.max.z], np.float32),
                         normal_indices=arr(m.vertex_normal_indices, 3 * t, np.uint32, (t, 3)),
                         uv_indices=arr(m.vertex_uvs_indices, 3 * t, np.uint32, (t, 3)))
    ref.ref_free(arena)
    H.blas_sah(md, "orc")
    assert (md.node_count, md.height) == (g["node_count"], g["height"])
    assert sha(md.nodes[:md.node_count]) == g["nodes_sha256"]
    assert sha(md.leaf_ids) == g["leaf_ids_sha256"]
    assert sha(md.triangles) == g["triangles_sha256"]


@pytest.mark.parametrize("key", sorted(GOLDEN["textures"]))
def test_texture_bake_matches_reference(key):
    """scenes.bake_texture (the residency format the device samples) equals bmp2texture's
    loadTexture on the same image, mip by mip."""
    g = GOLDEN["textures"][key]
    wh, w_, m_ = key.split("_")
    w, h = map(int, wh.split("x"))
    wrap, mip = int(w_[1:]), int(m_[1:])
    rng = np.random.default_rng(g["seed"])
    # regenerate the same sequence of images as make_golden (one per key, in its order)
    order = ["8x8_w1_m1", "16x8_w0_m1", "12x10_w1_m1", "33x17_w0_m0", "64x64_w1_m1"]
    for k in order:
        kw, kh = map(int, k.split("_")[0].split("x"))
        img = rng.integers(0, 256, size=(kh, kw, 3), dtype=np.uint8)
        if k == key:
            break
    td = scenes.bake_texture(img, bool(wrap), bool(mip))
    assert len(td.mips) == len(g["mips"])
    for (mw, mh, quads), (gw, gh, gd) in zip(td.mips, g["mips"]):
        assert (mw, mh) == (gw, gh)
        assert hashlib.sha256(quads.tobytes()).hexdigest() == gd


@needs_ref
def test_projection_plane_matches_reference():
    ref = oracle.reference()
    for cam in (scenes.CameraSpec(), scenes.look_at((3, 8, -20), (0, 1, 0)), scenes.look_at((-7, 2, 9), (1, 0, -2))):
        for w, h in ((640, 480), (1920, 1080), (257, 99)):
            fr = scenes.Frame(w, h, cam)
            mine = (C.c_uint8 * C.sizeof(S.ProjectionPlane)).from_buffer_copy(fr.viewport.projection_plane)
            ref.ref_begin_drawing(C.byref(fr.viewport))
            theirs = (C.c_uint8 * C.sizeof(S.ProjectionPlane)).from_buffer_copy(fr.viewport.projection_plane)
            assert bytes(mine) == bytes(theirs)


@needs_ref
def test_ssb_matches_reference():
    ref, orc = oracle.reference(), oracle.restatement()
    for sd, cam in (scenes.implicit16_scene(), scenes.moving_scene(count=512), scenes.mesh_scene(subdivisions=1, texture_size=8)):
        for w, h in ((640, 480), (320, 180)):
            a, b = sd.copy(), sd.copy()
            sa, ka = a.to_ctypes()
            sb, kb = b.to_ctypes()
            fa, fb = scenes.Frame(w, h, cam), scenes.Frame(w, h, cam)
            ref.ref_update_scene_ssb(C.byref(sa), C.byref(fa.viewport))
            orc.orc_update_scene_ssb(C.byref(sb), C.byref(fb.viewport))
            for f in S.PRIMITIVE_DT.names:   # fields only: the reference may write the 2 padding bytes
                assert np.array_equal(a.primitives[f], b.primitives[f]), f


def _lbvh(boxes, max_leaf, builder="lbvh"):
    orc = oracle.restatement()
    n = len(boxes)
    codes, order = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
    nodes, leaf, info = np.zeros(2 * n, dtype=S.BVHNODE_DT), np.zeros(n, np.uint32), np.zeros(2, np.uint32)
    boxes = np.ascontiguousarray(boxes, np.float32)
    if builder == "lbvh":
        orc.orc_lbvh30(boxes.ctypes.data, n, max_leaf, codes.ctypes.data, order.ctypes.data, nodes.ctypes.data,
                       leaf.ctypes.data, info.ctypes.data)
    else:
        orc.orc_binned_sah(boxes.ctypes.data, n, max_leaf, order.ctypes.data, nodes.ctypes.data, info.ctypes.data)
        leaf = order.copy()
    return codes, order, nodes[:info[0]], leaf, int(info[0]), int(info[1])


def _morton30_numpy(boxes):
    """The 30-bit Morton code of the LBVH specification, restated independently with numpy float32:
    centroid (min + max) * 0.5; per axis t = (c - lo) * (1024 / (hi - lo)) over the union box (scale
    0 on a flat axis); q = 0 unless t > 0, 1023 from t >= 1023, else t truncated; x takes the
    highest bit of each triple."""
    b = np.asarray(boxes, np.float32)
    lo, hi = b[:, :3].min(0), b[:, 3:].max(0)
    ext = (hi - lo).astype(np.float32)
    with np.errstate(divide="ignore"):
        scale = np.where(ext > 0, np.float32(1024.0) / ext, np.float32(0.0)).astype(np.float32)
    c = ((b[:, :3] + b[:, 3:]) * np.float32(0.5)).astype(np.float32)
    t = ((c - lo) * scale).astype(np.float32)
    q = np.where(t > 0, np.where(t >= 1023, 1023, np.trunc(np.where(t > 0, t, 0))), 0).astype(np.uint32)
    code = np.zeros(len(b), np.uint32)
    for bit in range(10):
        for axis, shift in ((0, 2), (1, 1), (2, 0)):
            code |= ((q[:, axis] >> bit) & 1) << (3 * bit + shift)
    return code


MORTON_CASES = ["random", "flat_axis", "identical", "wide_range", "clustered"]


@pytest.mark.parametrize("case", MORTON_CASES)
def test_lbvh_codes_match_an_independent_restatement(case):
    """The oracle's Morton codes (orc_lbvh30) equal the numpy restatement bit for bit, including a flat
    axis (scale 0), identical boxes, coordinates spanning many binades and tight clusters."""
    rng = np.random.default_rng(1000 + MORTON_CASES.index(case))
    n = 3000
    c = rng.uniform(-10, 10, (n, 3))
    if case == "flat_axis":
        c[:, 1] = 2.5
    elif case == "identical":
        c[:] = (1.0, -2.0, 3.0)
    elif case == "wide_range":
        c = rng.choice([-1, 1], (n, 3)) * 10.0 ** rng.uniform(-6, 6, (n, 3))
    elif case == "clustered":
        c = rng.integers(0, 4, (n, 1)) * 100.0 + rng.normal(0, 1e-3, (n, 3))
    e = rng.uniform(0.0, 0.5, (n, 3)) if case != "identical" else np.full((n, 3), 0.25)
    if case == "flat_axis":
        e[:, 1] = 0.0
    boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
    codes, order, *_ = _lbvh(boxes, 2)
    want = _morton30_numpy(boxes)
    assert np.array_equal(codes, want), int((codes != want).sum())
    keys = want.astype(np.uint64) << np.uint64(32) | np.arange(n, dtype=np.uint64)
    assert np.array_equal(order, np.argsort(keys, kind="stable").astype(np.uint32))


def _lbvh_top_down(boxes, max_leaf):
    """The LBVH30 topology and layout, restated top-down: the binary radix tree of the sorted
    (code << 32 | index) keys splits a range [f, l] after the last key that shares a longer prefix
    with key f than key l does; internal node g + (0 or 1) is the child range that does not start or
    end at a leaf (Karras's numbering).  Ranges of more than max_leaf items are kept, ranked in
    internal-node order; kept node r's children go to slots 1 + 2r and 2 + 2r; every node's box is
    the union of its items' boxes; depth counts ancestors."""
    b = np.asarray(boxes, np.float32)
    n = len(b)
    keys = [(int(c) << 32) | i for i, c in enumerate(_morton30_numpy(b))]
    keys.sort()
    order = np.array([k & 0xFFFFFFFF for k in keys], np.uint32)
    nodes = np.zeros(max(1, 2 * n), dtype=S.BVHNODE_DT)

    def box(f, l):
        items = b[order[f:l + 1]]
        return np.concatenate([items[:, :3].min(0), items[:, 3:].max(0)])

    if n <= max_leaf:
        if n:
            nodes[0]["aabb"] = box(0, n - 1)
        nodes[0]["child_count"] = n
        return order, nodes[:1], 1
    internal = {}                         # internal node index -> (first, last, left, right, depth)

    def build(idx, f, l, depth):
        prefix = 64 - (keys[f] ^ keys[l]).bit_length()
        g = f
        while g + 1 < l and 64 - (keys[f] ^ keys[g + 1]).bit_length() > prefix:
            g += 1
        left = ("leaf", g) if g == f else ("node", g)
        right = ("leaf", g + 1) if g + 1 == l else ("node", g + 1)
        internal[idx] = (f, l, left, right, depth)
        if left[0] == "node":
            build(g, f, g, depth + 1)
        if right[0] == "node":
            build(g + 1, g + 1, l, depth + 1)

    build(0, 0, n - 1, 0)
    kept = sorted(k for k, v in internal.items() if v[1] - v[0] + 1 > max_leaf)
    rank = {k: r for r, k in enumerate(kept)}
    nodes[0]["aabb"] = box(0, n - 1)
    nodes[0]["first_child_id"] = 1
    height = 0
    for k in kept:
        f, l, left, right, depth = internal[k]
        g = left[1]
        for c, (kind, idx), (cf, cl) in ((0, left, (f, g)), (1, right, (g + 1, l))):
            o = nodes[1 + 2 * rank[k] + c]
            o["depth"] = depth + 1
            height = max(height, depth + 1)
            o["aabb"] = box(cf, cl)
            if kind == "node" and idx in rank:
                o["first_child_id"] = 1 + 2 * rank[idx]
            else:
                o["first_child_id"] = cf
                o["child_count"] = cl - cf + 1
    return order, nodes[:1 + 2 * len(kept)], height


@pytest.mark.parametrize("n,max_leaf", [(1, 2), (2, 2), (3, 1), (3, 2), (17, 2), (300, 1), (1000, 2), (2000, 4)])
@pytest.mark.parametrize("case", ["random", "clustered"])
def test_lbvh_topology_matches_a_top_down_restatement(n, max_leaf, case):
    """orc_lbvh30's nodes (Karras-style per-node search) equal the top-down radix-tree restatement
    byte for byte, with distinct and with heavily repeated Morton codes."""
    rng = np.random.default_rng(7 * n + max_leaf)
    c = rng.uniform(-10, 10, (n, 3)) if case == "random" else \
        rng.integers(0, 3, (n, 1)) * 50.0 + rng.uniform(0.5, 0.6, (n, 3))
    e = rng.uniform(0.01, 0.5, (n, 3))
    boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
    _, order, nodes, _, count, height = _lbvh(boxes, max_leaf)
    want_order, want_nodes, want_height = _lbvh_top_down(boxes, max_leaf)
    assert np.array_equal(order, want_order)
    assert (count, height) == (len(want_nodes), want_height)
    assert nodes.tobytes() == want_nodes.tobytes()


def _half_area(lo, hi):
    """halfArea (AABB.h:39) in float32, the reference's order: ex*ey + ey*ez + ez*ex."""
    e = (hi - lo).astype(np.float32)
    return (e[..., 0] * e[..., 1] + e[..., 1] * e[..., 2] + e[..., 2] * e[..., 0]).astype(np.float32)


def _binned_sah_numpy(boxes, max_leaf, bins=32):
    """The binned-SAH specification restated with numpy float32: level by level, a range of more
    than max_leaf items is split on the axis and bin boundary of least halfArea(L)*nL +
    halfArea(R)*nR over 32 bins of its centroid extent (axes with zero extent skipped, empty sides
    skipped, first minimum in (axis, bin) order wins), else at its middle; the partition is stable
    and each level's split nodes get child pairs in order."""
    b = np.asarray(boxes, np.float32)
    n = len(b)
    f32 = np.float32
    cent = ((b[:, :3] + b[:, 3:]) * f32(0.5)).astype(f32)
    ids = np.arange(n)
    nodes = np.zeros(max(1, 2 * n), dtype=S.BVHNODE_DT)
    tasks, pairs, height, level = [(0, n, 0)], 0, 1, 0
    while tasks:
        nxt = []
        for begin, end, slot in tasks:
            it = ids[begin:end]
            nodes[slot]["aabb"] = np.concatenate([b[it, :3].min(0), b[it, 3:].max(0)]) if len(it) else 0
            nodes[slot]["depth"] = level
            if end - begin <= max_leaf:
                nodes[slot]["first_child_id"] = begin
                nodes[slot]["child_count"] = end - begin
                height = max(height, level)
                continue
            c = cent[it]
            lo = c.min(0)
            ext = (c.max(0) - lo).astype(f32)
            best_cost, best_axis, best_k, best_bins = np.inf, -1, -1, None
            for a in range(3):
                if not ext[a] > 0:
                    continue
                t = ((c[:, a] - lo[a]) * (f32(bins) / ext[a])).astype(f32)
                bv = np.where(t >= bins - 1, bins - 1, np.trunc(np.maximum(t, 0))).astype(np.int64)
                bv[~(t > 0)] = 0
                cnt = np.bincount(bv, minlength=bins)
                bmin = np.full((bins, 3), np.inf, f32)
                bmax = np.full((bins, 3), -np.inf, f32)
                np.minimum.at(bmin, bv, b[it, :3])
                np.maximum.at(bmax, bv, b[it, 3:])
                lmin, lmax = np.minimum.accumulate(bmin, 0), np.maximum.accumulate(bmax, 0)
                rmin, rmax = np.minimum.accumulate(bmin[::-1], 0)[::-1], np.maximum.accumulate(bmax[::-1], 0)[::-1]
                nl = np.cumsum(cnt)
                nr = np.cumsum(cnt[::-1])[::-1]
                k = np.arange(bins - 1)
                ok = (nl[k] > 0) & (nr[k + 1] > 0)
                with np.errstate(invalid="ignore", over="ignore"):
                    cost = (_half_area(lmin[k], lmax[k]) * nl[k].astype(f32) +
                            _half_area(rmin[k + 1], rmax[k + 1]) * nr[k + 1].astype(f32)).astype(f32)
                cost[~ok] = np.inf
                j = int(np.argmin(cost))
                if cost[j] < best_cost:
                    best_cost, best_axis, best_k, best_bins = cost[j], a, j, bv
            if best_axis >= 0:
                left = best_bins <= best_k
                ids[begin:end] = np.concatenate([it[left], it[~left]])
                mid = begin + int(left.sum())
            else:
                mid = begin + (end - begin) // 2
            nodes[slot]["first_child_id"] = 1 + 2 * pairs
            nxt += [(begin, mid, 1 + 2 * pairs), (mid, end, 2 + 2 * pairs)]
            pairs += 1
        tasks = nxt
        level += 1
    return ids.astype(np.uint32), nodes[:1 + 2 * pairs], height


@pytest.mark.parametrize("n,max_leaf", [(1, 2), (2, 1), (3, 2), (17, 2), (700, 2), (2000, 4)])
@pytest.mark.parametrize("case", ["random", "flat_axis", "same_centroid", "clustered"])
def test_binned_sah_matches_a_numpy_restatement(n, max_leaf, case):
    """orc_binned_sah's order and node arrays equal the numpy restatement byte for byte, including
    axes of zero centroid extent and ranges that fall back to the middle split."""
    rng = np.random.default_rng(11 * n + max_leaf)
    c = rng.uniform(-10, 10, (n, 3))
    if case == "flat_axis":
        c[:, 2] = 1.25
    elif case == "same_centroid":
        c[:] = (0.5, -1.5, 2.5)
    elif case == "clustered":
        c = rng.integers(0, 3, (n, 1)) * 40.0 + rng.uniform(0.5, 0.5001, (n, 3))
    e = rng.uniform(0.01, 0.5, (n, 3))
    boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
    _, order, nodes, _, count, height = _lbvh(boxes, max_leaf, "binned_sah")
    want_order, want_nodes, want_height = _binned_sah_numpy(boxes, max_leaf)
    assert np.array_equal(order, want_order)
    assert (count, height) == (len(want_nodes), want_height)
    assert nodes.tobytes() == want_nodes.tobytes()


@pytest.mark.parametrize("builder", ["lbvh", "binned_sah"])
@pytest.mark.parametrize("n,max_leaf", [(1, 2), (2, 2), (3, 2), (17, 2), (1000, 2), (5000, 4), (4096, 2)])
def test_bvh_oracle_structure(n, max_leaf, builder):
    """The LBVH30 specification: order sorts (code, index); every item sits in exactly one leaf of at
    most max_leaf items; every node box is the union of what it covers; children pairs are
    adjacent; height is the deepest leaf's depth."""
    rng = np.random.default_rng(n)
    c = rng.uniform(-10, 10, (n, 3))
    e = rng.uniform(0.01, 1, (n, 3))
    boxes = np.concatenate([c - e, c + e], 1)
    codes, order, nodes, leaf, count, height = _lbvh(boxes, max_leaf, builder)
    if builder == "lbvh":
        keys = codes[order].astype(np.uint64) << np.uint64(32) | order.astype(np.uint64)
        assert np.all(np.diff(keys.astype(np.float64)) > 0) or n == 1
    assert np.array_equal(np.sort(order), np.arange(n))
    assert np.array_equal(leaf, order)
    covered = np.zeros(n, int)
    depth_max = 0

    def walk(i, depth):
        nonlocal depth_max
        nd = nodes[i]
        if nd["child_count"]:
            f, k = nd["first_child_id"], nd["child_count"]
            assert k <= max(max_leaf, 1) or (i == 0 and n <= max_leaf)
            covered[f:f + k] += 1
            items = boxes[order[f:f + k]]
            assert np.array_equal(nd["aabb"][:3], items[:, :3].min(0).astype(np.float32))
            assert np.array_equal(nd["aabb"][3:], items[:, 3:].max(0).astype(np.float32))
            depth_max = max(depth_max, depth)
            return items[:, :3].min(0), items[:, 3:].max(0)
        f = nd["first_child_id"]
        assert f % 2 == 1 and f + 1 < count
        assert nodes[f]["depth"] == depth + 1 and nodes[f + 1]["depth"] == depth + 1
        a, b = walk(f, depth + 1), walk(f + 1, depth + 1)
        lo, hi = np.minimum(a[0], b[0]), np.maximum(a[1], b[1])
        assert np.array_equal(nd["aabb"][:3], lo.astype(np.float32)) and np.array_equal(nd["aabb"][3:], hi.astype(np.float32))
        return lo, hi

    walk(0, 0)
    assert np.all(covered == 1)
    assert height == max(depth_max, 1)


@pytest.mark.parametrize("which", ["implicit16", "area", "mesh"])
def test_pick_matches_reference(which):
    """manipulateSelection's picking ray (viewport/manipulation.h:55-123): the oracle's pick equals
    the reference's own hitPrimitives + glow-sphere sequence bit for bit, on scattered pixels and on
    pixels that hit a light."""
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    if which == "implicit16":
        sd, cam = scenes.implicit16_scene()
    elif which == "area":
        sd, cam = scenes.example_area_lights()
    else:
        sd, cam = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="ref")
    H.tlas_sah(sd, "ref")
    w, h = 160, 120
    rng = np.random.default_rng(11)
    coords = [tuple(c) for c in rng.integers(0, [w, h], (60, 2))]
    lights = H.light_coords(sd, cam, w, h) if len(sd.lights) else []
    coords += lights[:10]
    a = [H.pick_key(r) for r in H.picks(sd, cam, w, h, coords, "orc")]
    b = [H.pick_key(r) for r in H.picks(sd, cam, w, h, coords, "ref")]
    assert a == b
    assert any(k[0] for k in a)
    if which == "implicit16":
        assert any(k[1] == 6 for k in a), "no pixel hit a light"


def test_projection_matrix_matches_begin_drawing():
    """scenes.set_projection_matrix equals the matrix the reference's beginDrawing leaves
    (setProjectionMatrix, viewport/viewport.h:95), bit for bit, with and without cube NDC."""
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    ref = oracle.reference()
    sd, cam = scenes.implicit16_scene()
    for cube in (0, 1):
        fr = scenes.Frame(200, 150, cam, with_pixels=False)
        fr.viewport.settings.use_cube_NDC = cube
        scenes.set_projection_matrix(fr.viewport, fr.camera, fr.grid.dimensions)
        mine = bytes(fr.viewport.projection_matrix)
        ref.ref_begin_drawing(C.byref(fr.viewport))
        assert bytes(fr.viewport.projection_matrix) == mine


@pytest.mark.parametrize("which", ["implicit16", "area", "mesh", "inside", "inside_mesh"])
def test_overlays_match_reference(which):
    """drawBVH and drawSSB (render/raytracer.h:46, render/SSB.h:175): the oracle's overlays leave
    the float grid byte-identical to the reference's own drawing over the same render, for the
    BVH alone, the SSB alone and both."""
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    sd, cam = H.overlay_scene(which)
    H.tlas_sah(sd, "ref")
    for what in (1, 2, 3):
        a = H.overlay_frame(sd, cam, 160, 120, what, "orc")
        b = H.overlay_frame(sd, cam, 160, 120, what, "ref")
        assert a.float_pixels.tobytes() == b.float_pixels.tobytes()
        changed = np.count_nonzero(a.float_pixels.view(np.uint8).reshape(len(a.float_pixels), -1)
                                   != a.base.view(np.uint8).reshape(len(a.base), -1), axis=1)
        assert np.count_nonzero(changed) > 100, "the overlay drew almost nothing"


def test_overlays_far_plane_matches_reference():
    """drawBVH / drawSSB with a far clipping plane inside the scene (cullAndClipEdge's far branch,
    shapes/edge.h:23-29): the oracle still equals the reference's own drawing."""
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    sd, cam = H.overlay_scene("implicit16")
    H.tlas_sah(sd, "ref")
    out = {}
    for which in ("orc", "ref"):
        fr = H.oracle_frame(sd, cam, 160, 120, depth=1)
        fr.viewport.settings.far_clipping_plane_distance = np.float32(16.0)
        scenes.set_projection_matrix(fr.viewport, fr.camera, fr.grid.dimensions)
        base = fr.float_pixels.copy()
        lib = oracle.restatement() if which == "orc" else oracle.reference()
        d = sd.copy()
        sc, keep = d.to_ctypes()
        (lib.orc_update_scene_ssb if which == "orc" else lib.ref_update_scene_ssb)(C.byref(sc), C.byref(fr.viewport))
        if which == "orc":
            lib.orc_draw_overlays(C.byref(sc), C.byref(fr.viewport), 3)
        else:
            assert lib.ref_draw_overlays(C.byref(sc), C.byref(fr.viewport), 3) == 0
        out[which] = fr.float_pixels.copy()
        assert np.count_nonzero(out[which].view(np.uint8) != base.view(np.uint8)) > 100
    assert out["orc"].tobytes() == out["ref"].tobytes()


def _deepest(nodes, count):
    """Depth of the deepest node reachable from the root (root = 0), walking child pairs."""
    deepest, stack = 0, [(0, 0)]
    while stack:
        i, d = stack.pop()
        deepest = max(deepest, d)
        if not nodes[i]["child_count"] and count > 1:
            f = int(nodes[i]["first_child_id"])
            stack += [(f, d + 1), (f + 1, d + 1)]
    return deepest


def test_project_builders_state_exact_heights():
    """LBVH30 and binned SAH (the project's builders): the stated height is the depth of the deepest
    leaf (1 for a root leaf) and every node's depth field is its depth from the root."""
    rng = np.random.default_rng(9)
    for builder in ("lbvh", "binned_sah"):
        for n, leaf in ((1, 2), (5, 2), (2000, 2), (3000, 4)):
            c = rng.uniform(-10, 10, (n, 3))
            boxes = np.concatenate([c - 0.1, c + 0.1], 1)
            _, _, nodes, _, cnt, height = _lbvh(boxes, leaf, builder)
            assert height == max(_deepest(nodes, cnt), 1), (builder, n)
            stack = [(0, 0)]
            while stack:
                i, d = stack.pop()
                assert nodes[i]["depth"] == d, (builder, n, i)
                if not nodes[i]["child_count"] and cnt > 1:
                    f = int(nodes[i]["first_child_id"])
                    stack += [(f, d + 1), (f + 1, d + 1)]


@pytest.mark.parametrize("which", ["orc", "ref"])
def test_reference_sah_understates_heights(which):
    """The reference's top-down SAH (builder_top_down.h:204; the oracle restates it) states heights
    and node depth fields below the depth its trees reach, so the library bounds its traversal
    stacks by the walked depth: st_validate_bvh accepts these trees and measures them itself."""
    if which == "ref" and not oracle.reference_available():
        pytest.skip("reference harness not built")
    L = api.lib()
    seen = []
    for count in (16, 300, 4096):
        sd, _ = scenes.moving_scene(count=count)
        H.tlas_sah(sd, which)
        n = sd.tlas_node_count
        deepest = _deepest(sd.tlas_nodes, n)
        assert deepest >= sd.tlas_height and int(sd.tlas_nodes[:n]["depth"].max()) <= deepest
        seen.append(deepest - sd.tlas_height)
        assert L.st_validate_bvh(sd.tlas_nodes.ctypes.data, n, count, sd.tlas_height) == api.ST_OK
    for sub in (2, 4):
        md = H.blas_sah(scenes.displaced_icosphere(sub, seed=3), which)
        deepest = _deepest(md.nodes, md.node_count)
        assert deepest >= md.height
        seen.append(deepest - md.height)
        assert L.st_validate_bvh(md.nodes.ctypes.data, md.node_count, md.triangle_count, md.height) == api.ST_OK
    assert max(seen) >= 2          # 4096 primitives: height 11, walked depth 15
