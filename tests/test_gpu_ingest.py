"""Device texture baking (st_bake_texture, loadTexture bmp2texture.c:324) against the oracle's
baker and the reference's own, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

import oracle
from slimtracin_b200 import api, scenes, structs as S
from tests.test_io import _texture_bytes, _texture_ctypes

pytestmark = pytest.mark.gpu

CASES = [(64, 48, 1, 1, 24), (32, 32, 0, 1, 24), (20, 12, 1, 0, 24), (33, 17, 0, 1, 32), (2, 2, 1, 1, 24),
         (1024, 1024, 1, 1, 24), (640, 200, 0, 1, 32)]


def device_bake(renderer, comps, w, h, bits, wrap, mip):
    L = renderer.L
    need = L.st_texture_bytes(w, h, mip)
    mem = np.zeros(need, dtype=np.uint8)
    tex = S.Texture()
    assert L.st_bake_texture(renderer.ctx, comps.ctypes.data, w, h, bits, wrap, mip, C.byref(tex), mem.ctypes.data,
                             need - 1) == api.ST_ERR_BUDGET
    st = L.st_bake_texture(renderer.ctx, comps.ctypes.data, w, h, bits, wrap, mip, C.byref(tex), mem.ctypes.data, need)
    assert st == 0, st
    return tex, mem


@pytest.mark.parametrize("w,h,wrap,mip,bits", CASES)
def test_bake_equals_oracle_and_reference(renderer, w, h, wrap, mip, bits):
    rng = np.random.default_rng(w * 131 + h)
    comps = rng.integers(0, 256, (h, w, bits // 8), dtype=np.uint8)
    tex, mem = device_bake(renderer, comps, w, h, bits, wrap, mip)
    keep = []
    want = _texture_ctypes(scenes.bake_texture(comps[..., :3], bool(wrap), bool(mip)), keep)
    assert _texture_bytes(tex) == _texture_bytes(want)
    if oracle.reference_available():
        ref = oracle.reference()
        rt = S.Texture()
        ref.ref_load_texture(C.byref(rt), w, h, wrap, mip, comps.ctypes.data, bits)
        try:
            assert _texture_bytes(tex) == _texture_bytes(rt)
        finally:
            ref.ref_free_texture(C.byref(rt))


def test_bake_refuses_bad_arguments(renderer):
    L = renderer.L
    comps = np.zeros(64 * 3, dtype=np.uint8)
    mem = np.zeros(1 << 16, dtype=np.uint8)
    tex = S.Texture()
    for w, h, bits in ((1, 8, 24), (8, 1, 24), (8, 8, 16)):
        assert L.st_bake_texture(renderer.ctx, comps.ctypes.data, w, h, bits, 1, 1, C.byref(tex), mem.ctypes.data,
                                 mem.nbytes) == api.ST_ERR_INVALID_ARG


def write_obj(path, md, invert=False):
    """A Wavefront OBJ with positions, uvs, normals and "f v/t/n" faces (9 significant digits, so
    every float reads back exactly), placed off the origin so that obj2mesh recentres it."""
    lines = []
    for p in md.positions:
        lines.append("v %.9g %.9g %.9g" % (p[0] + 1.25, p[1] - 0.5, p[2] + 3.0))
    for t in md.uvs:
        lines.append("vt %.9g %.9g" % (t[0], t[1]))
    for n in md.normals:
        lines.append("vn %.9g %.9g %.9g" % tuple(n))
    lines.append("# comment, ignored")
    for a, b, c in md.indices + 1:
        lines.append("f %d/%d/%d %d/%d/%d %d/%d/%d" % (a, a, a, b, b, b, c, c, c))
    open(path, "w").write("\n".join(lines) + "\n")


def obj_mesh(renderer, path, invert, mode):
    L = renderer.L
    need = L.st_obj_mesh_bytes(path.encode())
    assert need > 0
    mem = np.zeros(need, dtype=np.uint8)
    m = S.Mesh()
    st = L.st_obj_to_mesh(renderer.ctx, path.encode(), int(invert), mode, C.byref(m), mem.ctypes.data, need)
    assert st == 0, st
    return m, mem


@pytest.mark.parametrize("invert", [0, 1])
def test_obj_to_mesh_matches_obj2mesh(renderer, tmp_path, invert):
    """obj2mesh (obj2mesh.c:25): the reference's converter and st_obj_to_mesh agree on the AABB,
    every vertex, uv and normal, every face index (winding inverted or not) and the edge list in
    first-appearance order; the BLAS is the device build of st_update_mesh_bvh over those arrays."""
    from tests.test_io import _mesh_arrays
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    md = scenes.displaced_icosphere(2, 7)
    obj = str(tmp_path / "a.obj")
    write_obj(obj, md)
    m, mem = obj_mesh(renderer, obj, invert, api.ST_BVH_BINNED_SAH)
    ref = oracle.reference()
    out = str(tmp_path / "ref.mesh").encode()
    assert ref.obj2mesh(obj.encode(), out, bool(invert)) == 0
    theirs = S.Mesh()
    arena = ref.ref_load_mesh(out, C.byref(theirs))
    try:
        a, b = _mesh_arrays(m), _mesh_arrays(theirs)
        for key in ("positions", "position_ids", "edges", "uvs", "uv_ids", "normals", "normal_ids"):
            assert a[key] == b[key], key
        assert bytes(m.aabb) == bytes(theirs.aabb)
        assert (m.vertex_count, m.triangle_count, m.edge_count) == (theirs.vertex_count, theirs.triangle_count,
                                                                     theirs.edge_count)
    finally:
        ref.ref_free(arena)
    # the BLAS equals the device build over the same arrays
    again = S.Mesh.from_buffer_copy(m)
    nodes = np.zeros(2 * m.triangle_count, dtype=S.BVHNODE_DT)
    leaf = np.zeros(m.triangle_count, dtype=np.uint32)
    tris = np.zeros(m.triangle_count, dtype=S.TRIANGLE_DT)
    again.bvh.nodes, again.bvh.leaf_ids, again.triangles = nodes.ctypes.data, leaf.ctypes.data, tris.ctypes.data
    assert renderer.L.st_update_mesh_bvh(renderer.ctx, C.byref(again), api.ST_BVH_BINNED_SAH) == 0
    assert C.string_at(m.bvh.nodes, 32 * m.bvh.node_count) == nodes[:again.bvh.node_count].tobytes()
    assert C.string_at(m.triangles, 128 * m.triangle_count) == tris.tobytes()


def test_obj_edges_on_a_large_mesh(renderer, tmp_path):
    """The device's edge list on a 20,480-triangle mesh equals first-appearance order computed on
    the host (a closed icosphere has 3/2 edges per triangle)."""
    md = scenes.displaced_icosphere(5, 3)
    obj = str(tmp_path / "b.obj")
    write_obj(obj, md)
    m, mem = obj_mesh(renderer, obj, 0, api.ST_BVH_LBVH30)
    ids = np.frombuffer(C.string_at(m.vertex_position_indices, 12 * m.triangle_count), dtype=np.uint32).reshape(-1, 3)
    seen, want = set(), []
    for t in ids:
        for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            e = (min(a, b), max(a, b))
            if e not in seen:
                seen.add(e)
                want.append(e)
    got = np.frombuffer(C.string_at(m.edge_vertex_indices, 8 * m.edge_count), dtype=np.uint32).reshape(-1, 2)
    assert m.edge_count == len(want) == 3 * m.triangle_count // 2
    assert np.array_equal(got, np.array(want, dtype=np.uint32))


def test_obj_refuses_other_face_layouts(renderer, tmp_path):
    obj = str(tmp_path / "c.obj")
    open(obj, "w").write("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    need = renderer.L.st_obj_mesh_bytes(obj.encode())
    mem = np.zeros(max(need, 64), dtype=np.uint8)
    m = S.Mesh()
    assert renderer.L.st_obj_to_mesh(renderer.ctx, obj.encode(), 0, api.ST_BVH_LBVH30, C.byref(m), mem.ctypes.data,
                                     mem.nbytes) == api.ST_ERR_BAD_SCENE
    assert renderer.L.st_obj_mesh_bytes(str(tmp_path / "none.obj").encode()) == -1
