"""The reference's file formats through the library (st_io.cu): .mesh, .texture and .scene files
written by the library are byte-identical to the reference's writers' (saveMeshToFile,
bmp2texture, saveSceneToFile), and the library reads what the reference writes.  Host code only:
no GPU is needed."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

import oracle
from slimtracin_b200 import api, scenes, structs as S
from tests import helpers as H

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


def _mesh():
    """A small displaced icosphere with its BLAS (the oracle's SAH) and a few edges."""
    sd, cam = scenes.mesh_scene(subdivisions=2, texture_size=8)
    md = sd.meshes[0]
    H.blas_sah(md, "orc")
    keep = []
    m = md.to_ctypes(keep)
    edges = np.arange(40, dtype=np.uint32).reshape(20, 2) % max(len(md.positions), 1)
    keep.append(edges)
    m.edge_count = len(edges)
    m.edge_vertex_indices = edges.ctypes.data
    return md, m, keep


def _mesh_arrays(m):
    """Every array of a ctypes Mesh as bytes, keyed by name."""
    def arr(ptr, nbytes):
        return C.string_at(ptr, nbytes) if nbytes else b""
    t = m.triangle_count
    return {
        "header": bytes(m.aabb) + struct.pack("7I", m.vertex_count, t, m.edge_count, m.uvs_count, m.normals_count,
                                              m.bvh.node_count, m.bvh.height),
        "positions": arr(m.vertex_positions, 12 * m.vertex_count),
        "position_ids": arr(m.vertex_position_indices, 12 * t),
        "edges": arr(m.edge_vertex_indices, 8 * m.edge_count),
        "uvs": arr(m.vertex_uvs, 8 * m.uvs_count), "uv_ids": arr(m.vertex_uvs_indices, 12 * t if m.uvs_count else 0),
        "normals": arr(m.vertex_normals, 12 * m.normals_count),
        "normal_ids": arr(m.vertex_normal_indices, 12 * t if m.normals_count else 0),
        "triangles": arr(m.triangles, 128 * t), "nodes": arr(m.bvh.nodes, 32 * m.bvh.node_count),
        "leaf_ids": arr(m.bvh.leaf_ids, 4 * t),
    }


def test_mesh_file_round_trip(tmp_path):
    """st_write_mesh_file -> st_read_mesh_file gives back every array; size queries and refusals."""
    L = api.lib()
    md, m, keep = _mesh()
    path = str(tmp_path / "a.mesh").encode()
    assert L.st_write_mesh_file(path, C.byref(m)) == 0
    need = L.st_mesh_file_bytes(path)
    assert need > 0
    mem = np.zeros(need, dtype=np.uint8)
    out = S.Mesh()
    assert L.st_read_mesh_file(path, C.byref(out), mem.ctypes.data, need - 1) == api.ST_ERR_BUDGET
    assert L.st_read_mesh_file(path, C.byref(out), mem.ctypes.data, need) == 0
    assert _mesh_arrays(out) == _mesh_arrays(m)
    # a truncated file and a missing file
    data = open(path, "rb").read()
    short = str(tmp_path / "short.mesh").encode()
    open(short, "wb").write(data[:-7])
    assert L.st_read_mesh_file(short, C.byref(out), mem.ctypes.data, need) == api.ST_ERR_IO
    assert L.st_mesh_file_bytes(str(tmp_path / "none.mesh").encode()) == -1
    assert L.st_read_mesh_file(str(tmp_path / "none.mesh").encode(), C.byref(out), mem.ctypes.data, need) == api.ST_ERR_IO


@needs_ref
def test_mesh_file_matches_reference(tmp_path):
    """Byte-identical to saveMeshToFile (scene/io.h:145); loadMeshFromFile (:95) reads it back."""
    L, ref = api.lib(), oracle.reference()
    md, m, keep = _mesh()
    ours, theirs = str(tmp_path / "ours.mesh").encode(), str(tmp_path / "ref.mesh").encode()
    assert L.st_write_mesh_file(ours, C.byref(m)) == 0
    ref.ref_save_mesh(C.byref(m), theirs)
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    back = S.Mesh()
    arena = ref.ref_load_mesh(ours, C.byref(back))
    try:
        assert _mesh_arrays(back) == _mesh_arrays(m)
    finally:
        ref.ref_free(arena)


@needs_ref
def test_reads_the_reference_monkey_mesh():
    """The one .mesh file the reference ships (src/examples/monkey.mesh) reads like
    loadMeshFromFile reads it."""
    from tests.golden import make_golden as G
    path = G.MONKEY
    if not os.path.exists(path):
        pytest.skip("reference sources not present")
    L, ref = api.lib(), oracle.reference()
    need = L.st_mesh_file_bytes(path.encode())
    mem = np.zeros(need, dtype=np.uint8)
    ours = S.Mesh()
    assert L.st_read_mesh_file(path.encode(), C.byref(ours), mem.ctypes.data, need) == 0
    theirs = S.Mesh()
    arena = ref.ref_load_mesh(path.encode(), C.byref(theirs))
    try:
        assert _mesh_arrays(ours) == _mesh_arrays(theirs)
    finally:
        ref.ref_free(arena)


def _texture_ctypes(td, keep):
    tex = S.Texture()
    tex.width, tex.height, tex.wrap, tex.mipmap = td.width, td.height, td.wrap, td.mipmap
    mips = (S.TextureMip * len(td.mips))()
    for k, (w, h, quads) in enumerate(td.mips):
        mips[k].width, mips[k].height = w, h
        mips[k].texel_quads = quads.ctypes.data
        keep.append(quads)
    keep.append(mips)
    tex.mip_count = len(td.mips)
    tex.mips = C.cast(mips, C.POINTER(S.TextureMip))
    return tex


def _texture_bytes(t):
    out = struct.pack("<HH??B", t.width, t.height, t.mipmap, t.wrap, t.mip_count)
    for k in range(t.mip_count):
        mip = t.mips[k]
        out += struct.pack("<HH", mip.width, mip.height) + C.string_at(mip.texel_quads, 12 * (mip.width + 1) * (mip.height + 1))
    return out


def write_bmp(path, rgb):
    """A 24-bit BMP with the rows in file order as given and BGR pixels (what LoadBitmapFile,
    bmp2texture.c:45, expects: it reads biSizeImage bytes and swaps B and R)."""
    h, w = rgb.shape[:2]
    assert (3 * w) % 4 == 0
    data = np.ascontiguousarray(rgb[..., ::-1]).tobytes()
    header = struct.pack("<2sIHHI", b"BM", 54 + len(data), 0, 0, 54)
    info = struct.pack("<IiiHHIIiiII", 40, w, h, 1, 24, 0, len(data), 0, 0, 0, 0)
    open(path, "wb").write(header + info + data)


@pytest.mark.parametrize("w,h,wrap,mip", [(64, 48, 1, 1), (32, 32, 0, 1), (20, 12, 1, 0)])
def test_texture_file_round_trip(tmp_path, w, h, wrap, mip):
    """st_write_texture_file -> st_read_texture_file gives back the texture; the file is the
    reference's layout."""
    L = api.lib()
    rng = np.random.default_rng(w * h)
    td = scenes.bake_texture(rng.integers(0, 256, (h, w, 3), dtype=np.uint8), bool(wrap), bool(mip))
    keep = []
    tex = _texture_ctypes(td, keep)
    path = str(tmp_path / "t.texture").encode()
    assert L.st_write_texture_file(path, C.byref(tex)) == 0
    assert open(path, "rb").read() == _texture_bytes(tex)
    need = L.st_texture_file_bytes(path)
    mem = np.zeros(need, dtype=np.uint8)
    back = S.Texture()
    assert L.st_read_texture_file(path, C.byref(back), mem.ctypes.data, need) == 0
    assert _texture_bytes(back) == _texture_bytes(tex)


@needs_ref
@pytest.mark.parametrize("w,h,wrap,mip", [(64, 48, 1, 1), (32, 32, 0, 1), (20, 12, 1, 0), (36, 64, 0, 0)])
def test_texture_file_matches_bmp2texture(tmp_path, w, h, wrap, mip):
    """The reference's bmp2texture tool (bmp2texture.c:364) on a BMP file writes the same bytes as
    st_write_texture_file of the same image baked by scenes.bake_texture; loadTextureFromFile
    (scene/io.h:34) reads the library's file back."""
    L, ref = api.lib(), oracle.reference()
    rng = np.random.default_rng(w + 7 * h)
    rgb = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
    bmp = str(tmp_path / "in.bmp")
    write_bmp(bmp, rgb)
    theirs = str(tmp_path / "ref.texture").encode()
    assert ref.bmp2texture(bmp.encode(), theirs, bool(mip), bool(wrap)) == 0
    keep = []
    tex = _texture_ctypes(scenes.bake_texture(rgb, bool(wrap), bool(mip)), keep)
    ours = str(tmp_path / "ours.texture").encode()
    assert L.st_write_texture_file(ours, C.byref(tex)) == 0
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    back = S.Texture()
    arena = ref.ref_load_texture_file(C.byref(back), ours, L.st_texture_file_bytes(ours) + 4096)
    try:
        assert _texture_bytes(back) == _texture_bytes(tex)
    finally:
        ref.ref_free(arena)


def _scene_file_scene():
    """The 16-primitive scene with its camera (a scene file holds settings, cameras and primitives)."""
    sd, spec = scenes.implicit16_scene()
    sc, keep = sd.to_ctypes()
    cams = (S.Camera * 1)()
    scenes.fill_camera(cams[0], spec)
    keep = [keep, cams]
    sc.cameras = C.addressof(cams)
    sc.settings.cameras = 1
    return sd, sc, keep


def test_scene_file_round_trip(tmp_path):
    """st_write_scene_file -> st_read_scene_file restores counts, cameras and primitives and keeps
    the reader's own pointers; too-small arrays are refused."""
    L = api.lib()
    sd, sc, keep = _scene_file_scene()
    path = str(tmp_path / "a.scene").encode()
    assert L.st_write_scene_file(path, C.byref(sc)) == 0
    n = sc.settings.primitives
    prims = (S.Primitive * n)()
    cams = (S.Camera * 1)()
    target = S.Scene()
    target.primitives = C.addressof(prims)
    target.cameras = C.addressof(cams)
    assert L.st_read_scene_file(path, C.byref(target), 1, n - 1) == api.ST_ERR_BUDGET
    assert L.st_read_scene_file(path, C.byref(target), 1, n) == 0
    assert target.settings.primitives == n and target.settings.cameras == sc.settings.cameras
    assert bytes(prims) == C.string_at(sc.primitives, 72 * n)
    cam = cams[0]
    src = S.Camera.from_address(sc.cameras)
    assert cam.focal_length == src.focal_length and bytes(cam.transform.rotation) == bytes(src.transform.rotation)
    right = cam.transform.right_direction
    assert C.addressof(cam.transform.rotation_matrix.X) == (right if isinstance(right, int) else C.cast(right, C.c_void_p).value)


@needs_ref
def test_scene_file_matches_reference(tmp_path):
    """Byte-identical to saveSceneToFile (scene/io.h:199); loadSceneFromFile (:178) reads it."""
    L, ref = api.lib(), oracle.reference()
    sd, sc, keep = _scene_file_scene()
    ours, theirs = str(tmp_path / "ours.scene").encode(), str(tmp_path / "ref.scene").encode()
    assert L.st_write_scene_file(ours, C.byref(sc)) == 0
    ref.ref_save_scene(C.byref(sc), theirs)
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    n = sc.settings.primitives
    prims = (S.Primitive * n)()
    cams = (S.Camera * 1)()
    target = S.Scene()
    target.primitives = C.addressof(prims)
    target.cameras = C.addressof(cams)
    ref.ref_load_scene(C.byref(target), ours)
    assert bytes(prims) == C.string_at(sc.primitives, 72 * n)


def test_texture_file_refusals(tmp_path):
    """Truncated texture files (inside the header, a mip's size, its quads), a missing file and a
    destination one byte too small are refused, never read past."""
    L = api.lib()
    rng = np.random.default_rng(5)
    keep = []
    tex = _texture_ctypes(scenes.bake_texture(rng.integers(0, 256, (24, 16, 3), dtype=np.uint8), True, True), keep)
    path = str(tmp_path / "t.texture").encode()
    assert L.st_write_texture_file(path, C.byref(tex)) == 0
    data = open(path, "rb").read()
    need = L.st_texture_file_bytes(path)
    mem = np.zeros(need + 64, dtype=np.uint8)
    back = S.Texture()
    assert L.st_read_texture_file(path, C.byref(back), mem.ctypes.data, need - 1) == api.ST_ERR_BUDGET
    for cut in (3, 9, len(data) // 2, len(data) - 1):
        short = str(tmp_path / f"short{cut}.texture").encode()
        open(short, "wb").write(data[:cut])
        got = L.st_texture_file_bytes(short)
        if got < 0:
            assert L.st_read_texture_file(short, C.byref(back), mem.ctypes.data, need) == api.ST_ERR_IO, cut
        else:
            assert L.st_read_texture_file(short, C.byref(back), mem.ctypes.data, len(mem)) == api.ST_ERR_IO, cut
    none = str(tmp_path / "none.texture").encode()
    assert L.st_texture_file_bytes(none) == -1
    assert L.st_read_texture_file(none, C.byref(back), mem.ctypes.data, need) == api.ST_ERR_IO


def test_scene_file_refusals(tmp_path):
    """Truncated scene files and a missing file are refused with ST_ERR_IO."""
    L = api.lib()
    sd, sc, keep = _scene_file_scene()
    path = str(tmp_path / "a.scene").encode()
    assert L.st_write_scene_file(path, C.byref(sc)) == 0
    data = open(path, "rb").read()
    n = sc.settings.primitives
    prims = (S.Primitive * n)()
    cams = (S.Camera * 1)()
    for cut in (5, len(data) // 2, len(data) - 1):
        short = str(tmp_path / f"short{cut}.scene").encode()
        open(short, "wb").write(data[:cut])
        target = S.Scene()
        target.primitives = C.addressof(prims)
        target.cameras = C.addressof(cams)
        assert L.st_read_scene_file(short, C.byref(target), 1, n) == api.ST_ERR_IO, cut
    target = S.Scene()
    target.primitives = C.addressof(prims)
    target.cameras = C.addressof(cams)
    assert L.st_read_scene_file(str(tmp_path / "none.scene").encode(), C.byref(target), 1, n) == api.ST_ERR_IO
