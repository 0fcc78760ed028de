"""Device path vs the oracle at the benchmarked sizes, through the C ABI.

* the 1080p PBR mesh scene exactly as the benchmark renders it: the 1,310,720-triangle displaced
  icosphere with its device binned-SAH BLAS (compared byte for byte with the oracle's build of the
  same boxes), 8 instances under a device LBVH30 TLAS, 1024^2 textures with 9 mips, 1921x1081 QCAA
  grid, depth 4, in every render mode, with and without ray-cone mip selection;
* the moving scene of 4096 implicit primitives at 1280x720, depth 2, with its TLAS rebuilt on the
  device by LBVH30 and by binned SAH, at frame 0 and after 30 frames of motion;
* a glass and mirror view of the 327,680-triangle mesh scene at 1920x1080, depth 6.

The oracle is given the trees the device built (their bytes are checked against the oracle's own
builders first), so every traversal step can be compared: work counters must be equal, primary-hit
ids and the non-beauty modes byte-identical, beauty within the stated tolerances (the libm calls
powf/acosf round differently in CUDA and glibc)."""
import ctypes as C

import numpy as np
import pytest

from slimtracin_b200 import api, scenes, structs as S
from tests import helpers as H

pytestmark = pytest.mark.gpu

SLOT_MESH, SLOT_MOVING, SLOT_GLASS = 14, 15, 15


def _mesh_identical(a, b):
    n = a.triangle_count
    return ((a.node_count, a.height) == (b.node_count, b.height)
            and a.nodes[:a.node_count].tobytes() == b.nodes[:b.node_count].tobytes()
            and np.array_equal(a.leaf_ids[:n], b.leaf_ids[:n])
            and a.triangles.tobytes() == b.triangles.tobytes())


@pytest.fixture(scope="module")
def bench_scene(renderer):
    """The benchmark's scene, built as bench.py builds it: device binned-SAH BLAS, device LBVH30 TLAS."""
    sd, cam = scenes.mesh_scene()
    for md in sd.meshes:
        renderer.build_blas(md, api.ST_BVH_BINNED_SAH)
    renderer.upload(SLOT_MESH, sd, tlas=None)
    renderer.build_tlas(SLOT_MESH, sd, api.ST_BVH_LBVH30)
    yield sd, cam
    renderer.free(SLOT_MESH)


def test_fullsize_blas_and_tlas_equal_the_oracle_builds(bench_scene):
    """The 1.31M-triangle BLAS: nodes, leaf ids and every Triangle record byte-identical to the
    oracle's binned-SAH updateMeshBVH of the same mesh; the TLAS to the oracle's LBVH30."""
    sd, _ = bench_scene
    md = sd.meshes[0]
    assert md.triangle_count == 1310720
    ref, _ = scenes.mesh_scene()
    H.blas_sah(ref.meshes[0], "binned")
    assert _mesh_identical(md, ref.meshes[0])
    assert md.height + 2 <= 64
    t = sd.copy()
    H.tlas_lbvh(t)
    assert H.same_tlas(sd, t)


@pytest.mark.parametrize("mode", [S.RM_BEAUTY, S.RM_DEPTH, S.RM_NORMALS, S.RM_UVS])
def test_fullsize_mesh_frame(renderer, bench_scene, mode):
    sd, cam = bench_scene
    g = H.gpu_frame(renderer, SLOT_MESH, sd, cam, 1920, 1080, depth=4, mode=mode, counters=True)
    o = H.oracle_frame(sd, cam, 1920, 1080, depth=4, mode=mode)
    m = H.compare(g, o, mode)
    print("mesh 1080p", mode, m, g.counters[:11])
    assert np.array_equal(g.counters[:11], o.counters[:11]), (g.counters[:11], o.counters[:11])
    assert np.array_equal(g.prim_ids, o.prim_ids)
    H.assert_parity(m, mode)
    if mode != S.RM_BEAUTY:
        assert m["exact"] == 1.0, m


@pytest.mark.parametrize("mode", [S.RM_BEAUTY, S.RM_NORMALS])
def test_fullsize_mesh_frame_ray_cone_mips(renderer, bench_scene, mode):
    """cone_angle = atan(2 / (H * focal_length)): mips above 0 of the 1024^2 textures are sampled."""
    sd, cam = bench_scene
    cone = H.cone_angle_for(1080, cam.focal_length)
    g = H.gpu_frame(renderer, SLOT_MESH, sd, cam, 1920, 1080, depth=4, mode=mode, cone_angle=cone, counters=True)
    o = H.oracle_frame(sd, cam, 1920, 1080, depth=4, mode=mode, cone_angle=cone)
    m = H.compare(g, o, mode)
    print("mesh 1080p cones", mode, m, g.counters[:11])
    assert np.array_equal(g.counters[:11], o.counters[:11]), (g.counters[:11], o.counters[:11])
    assert g.counters[10] > 0
    H.assert_parity(m, mode)
    if mode != S.RM_BEAUTY:
        assert m["exact"] == 1.0, m


@pytest.mark.parametrize("mode", [api.ST_BVH_LBVH30, api.ST_BVH_BINNED_SAH])
def test_moving_scene_720p_rebuilt_every_frame(renderer, mode):
    """4096 moving primitives at 1280x720, depth 2: the device TLAS equals the oracle's build of the
    same boxes at frame 0 and after 30 frames of motion, and the frames equal the oracle's."""
    sd, cam = scenes.moving_scene()
    assert len(sd.primitives) == 4096
    renderer.upload(SLOT_MOVING, sd, tlas=None)
    try:
        for frame in (0, 30):
            if frame:
                scenes.advance_moving_scene(sd, frame)
                sc, keep = sd.to_ctypes()
                renderer._check(renderer.L.st_upload_primitives(renderer.ctx, SLOT_MOVING, C.byref(sc)), "st_upload_primitives")
            renderer.build_tlas(SLOT_MOVING, sd, mode)
            t = sd.copy()
            (H.tlas_lbvh if mode == api.ST_BVH_LBVH30 else H.tlas_binned)(t)
            assert H.same_tlas(sd, t), frame
            g = H.gpu_frame(renderer, SLOT_MOVING, sd, cam, 1280, 720, depth=2, counters=True)
            o = H.oracle_frame(sd, cam, 1280, 720, depth=2)
            m = H.compare(g, o, S.RM_BEAUTY)
            print("moving 720p", mode, frame, m)
            # primary rays walk the TLAS with the screen-space cull here (more than 64 primitives)
            # where the reference loops over every primitive, so the box, primitive-test and leaf
            # counters differ by design; the rays, shading and texture counters do not
            same = [0, 1, 2, 7, 8, 9, 10]
            assert np.array_equal(g.counters[same], o.counters[same]), (g.counters[:11], o.counters[:11])
            assert np.array_equal(g.prim_ids, o.prim_ids)
            H.assert_parity(m, S.RM_BEAUTY)
    finally:
        renderer.free(SLOT_MOVING)


def test_glass_mirror_1080p_depth6(renderer):
    """The 327,680-triangle mesh scene of the mixed set (device binned-SAH BLAS and TLAS), 1080p,
    six bounces: long glass and mirror paths, deep BLAS walks from every bounce."""
    sd, cam = scenes.mesh_scene(seed_offset=207, subdivisions=7)
    renderer.build_blas(sd.meshes[0], api.ST_BVH_BINNED_SAH)
    ref, _ = scenes.mesh_scene(seed_offset=207, subdivisions=7)
    H.blas_sah(ref.meshes[0], "binned")
    assert _mesh_identical(sd.meshes[0], ref.meshes[0])
    renderer.upload(SLOT_GLASS, sd, tlas=None)
    try:
        renderer.build_tlas(SLOT_GLASS, sd, api.ST_BVH_BINNED_SAH)
        g = H.gpu_frame(renderer, SLOT_GLASS, sd, cam, 1920, 1080, depth=6, counters=True)
        o = H.oracle_frame(sd, cam, 1920, 1080, depth=6)
        m = H.compare(g, o, S.RM_BEAUTY)
        print("glass/mirror 1080p depth 6", m, g.counters[:11])
        assert g.counters[2] > 1_000_000              # bounce rays
        assert np.array_equal(g.counters[:11], o.counters[:11]), (g.counters[:11], o.counters[:11])
        assert np.array_equal(g.prim_ids, o.prim_ids)
        H.assert_parity(m, S.RM_BEAUTY)
    finally:
        renderer.free(SLOT_GLASS)
