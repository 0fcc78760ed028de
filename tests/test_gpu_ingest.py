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
