"""The drop-in: a host compiled from the reference's own headers (oracle/dropin.c) — its scene and
camera code, its top-down SAH TLAS build, its per-frame sequence updateSceneSSB, beginDrawing,
renderScene, drawViewportToWindowContent — with the GPU seams bound to libslimtracin_b200 through
the C ABI.  Its GPU frames equal its own CPU frames (the reference's renderSceneOnCPU) within the
parity tolerances."""
import ctypes as C

import pytest

import oracle
from slimtracin_b200 import scenes, structs as S
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin():
    if not oracle.dropin_available():
        pytest.skip("oracle/_ref/libdropin.so is not built (needs the reference sources)")
    lib = oracle.dropin()
    yield lib
    lib.dropin_shutdown()


def _frames(lib, sd, cam, w, h, depth, mode):
    out = []
    for use_gpu in (1, 0):
        d = sd.copy()
        sc, keep = d.to_ctypes()
        fr = scenes.Frame(w, h, cam, depth=depth, mode=mode)
        assert lib.dropin_frame(C.byref(sc), C.byref(fr.viewport), use_gpu, 1) == 0
        out.append(fr)
    return out


@pytest.mark.parametrize("which,mode", [("implicit16", S.RM_BEAUTY), ("implicit16", S.RM_NORMALS), ("area", S.RM_BEAUTY),
                                        ("mesh", S.RM_BEAUTY), ("mesh", S.RM_UVS)])
def test_dropin_host_gpu_equals_its_cpu(dropin, which, mode):
    if which == "implicit16":
        sd, cam = scenes.implicit16_scene()
        depth = 2
    elif which == "area":
        sd, cam = scenes.example_area_lights()
        depth = 2
    else:
        sd, cam = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="ref")
        depth = 4
    gpu, cpu = _frames(dropin, sd, cam, 320, 240, depth, mode)
    m = H.compare(gpu, cpu, mode)
    H.assert_parity(m, mode)
    if mode != S.RM_BEAUTY:
        assert m["exact"] == 1.0, m
