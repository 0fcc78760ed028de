"""Slot state after a failed TLAS rebuild, through the C ABI.

A rebuild (LBVH30 or binned SAH) overwrites the slot's node and leaf arrays before it can check the
new tree, so a rebuild that fails part way must leave no TLAS that a render or a refit could use:
both report ST_ERR_NOT_RESIDENT until a later build succeeds.  The failure is made on the host: a
context whose device-memory budget holds the scene and an LBVH30 build but not the binned-SAH
builder's scratch refuses the binned build with ST_ERR_BUDGET."""
import ctypes as C

import numpy as np
import pytest

from slimtracin_b200 import api, scenes
from tests import helpers as H

pytestmark = pytest.mark.gpu

ST_ERR_NOT_RESIDENT = 8


def _prepare(r, sd, cam):
    """Upload, an LBVH30 TLAS and one render: every allocation the test's context makes first."""
    r.upload(0, sd, tlas=None)
    r.build_tlas(0, sd, api.ST_BVH_LBVH30)
    return H.gpu_frame(r, 0, sd, cam, 128, 72, depth=2)


def test_failed_rebuild_leaves_no_usable_tlas():
    sd, cam = scenes.moving_scene(count=1024)
    with api.Renderer(device=0) as probe:
        _prepare(probe, sd.copy(), cam)
        need = int(probe.L.st_device_bytes_in_use(probe.ctx))
    # the same calls in a context whose budget ends 4 KB above what they hold
    with api.Renderer(device=0, memory_budget=need + 4096) as r:
        work = sd.copy()
        g = _prepare(r, work, cam)
        assert np.isfinite(g.float_pixels["depth"]).any()
        sc, keep = work.to_ctypes()
        L = r.L
        assert L.st_update_scene_bvh(r.ctx, 0, C.byref(sc), api.ST_BVH_BINNED_SAH) == api.ST_ERR_BUDGET
        assert L.st_update_scene_bvh(r.ctx, 0, None, api.ST_BVH_REFIT) == ST_ERR_NOT_RESIDENT
        fr = scenes.Frame(128, 72, cam, depth=2)
        opt = api.st_render_options()
        assert L.st_render_ex(r.ctx, 0, C.byref(sc), C.byref(fr.viewport), C.byref(opt)) == ST_ERR_NOT_RESIDENT
        # a build that succeeds makes the slot renderable again, with the frame it had before
        assert L.st_update_scene_bvh(r.ctx, 0, C.byref(sc), api.ST_BVH_LBVH30) == api.ST_OK
        g2 = H.gpu_frame(r, 0, work, cam, 128, 72, depth=2)
        assert g2.float_pixels.tobytes() == g.float_pixels.tobytes()
