"""Warp-vote ray compaction in st_render_batch's persistent kernel, through the C ABI: at a bounce, a
warp whose lanes still tracing number fewer than the threshold parks their paths in a queue, and a
second persistent pass traces them to the end.  A parked path runs the same steps as one traced in
place, so every view's float grid and u8 frame must equal the per-frame render's, byte for byte, at
every threshold, tile shape, stack placement, with and without the CUDA graph; the batch reports how
many paths it parked."""
import numpy as np
import pytest

from slimtracin_b200 import api, scenes, structs as S
from tests import helpers as H

pytestmark = pytest.mark.gpu


def test_compacted_batch_equals_per_frame_renders(renderer):
    c0, cam0 = scenes.implicit16_scene()
    H.tlas_sah(c0)
    renderer.upload(11, c0, tlas="host")
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    renderer.upload(12, c1, tlas="host")
    c2, cam2 = scenes.moving_scene(count=300)
    H.tlas_sah(c2)
    renderer.upload(13, c2, tlas="host")
    # the glass and mirror instances of the mesh scene bounce; the others end at the first hit
    specs = [(11, c0, cam0, 96, 64, 2, S.RM_BEAUTY), (12, c1, cam1, 320, 180, 6, S.RM_BEAUTY),
             (13, c2, cam2, 64, 48, 1, S.RM_BEAUTY), (12, c1, cam1, 80, 60, 4, S.RM_NORMALS),
             (12, c1, cam1, 160, 90, 3, S.RM_BEAUTY), (11, c0, cam0, 33, 17, 3, S.RM_DEPTH)]
    singles = [H.gpu_frame(renderer, slot, sd, cam, w, h, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
    for threshold in (8, 32):
        for tile in (0, 2):
            for stack in (0, 1):
                for graph in (False, True, True):
                    frames = [scenes.Frame(w, h, cam, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
                    opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)],
                                           tile_shape=tile, stack_placement=stack, use_graph=graph, chunk=1,
                                           launch_mode=api.LAUNCH_PERSISTENT, compaction_threshold=threshold)
                    key = (threshold, tile, stack, graph)
                    assert opt.compaction_threshold_used == threshold, key
                    for a, b in zip(frames, singles):
                        assert np.array_equal(a.float_pixels.view(np.uint8), b.float_pixels.view(np.uint8)), key
                        assert np.array_equal(a.pixels.view(np.uint8), b.pixels.view(np.uint8)), key
                    if threshold == 32:
                        assert opt.parked_rays > 0, key        # a warp short of 32 lanes parks its paths
    # without compaction nothing is parked; autotuned, the chosen threshold is reported
    frames = [scenes.Frame(w, h, cam, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
    opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)], tile_shape=0,
                           stack_placement=0, chunk=1, launch_mode=api.LAUNCH_PERSISTENT, compaction_threshold=0)
    assert opt.parked_rays == 0 and opt.compaction_threshold_used == 0
    frames = [scenes.Frame(w, h, cam, depth=d, mode=m) for slot, sd, cam, w, h, d, m in specs]
    opt = api.render_batch(renderer, [(sp[0], sp[1], fr) for sp, fr in zip(specs, frames)],
                           launch_mode=api.LAUNCH_PERSISTENT, compaction_threshold=-1)
    assert opt.compaction_threshold_used in (0, 8, 16, 24)
    for a, b in zip(frames, singles):
        assert np.array_equal(a.float_pixels.view(np.uint8), b.float_pixels.view(np.uint8))


def test_context_shutdown_returns_the_ray_queue():
    """A compacting batch reserves the parked-ray queue (96 MB for a launch group of a million rays or
    more); shutting the context down gives it back with everything else the context holds."""
    import torch
    c0, cam0 = scenes.implicit16_scene()
    H.tlas_sah(c0)
    warm = api.Renderer(device=0)          # the library's modules load once, outside the measurement
    warm.close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    r = api.Renderer(device=0)
    r.upload(3, c0, tlas="host")
    fr = scenes.Frame(1920, 1080, cam0, depth=3, mode=S.RM_BEAUTY)
    opt = api.render_batch(r, [(3, c0, fr)], tile_shape=0, stack_placement=0, chunk=1,
                           launch_mode=api.LAUNCH_PERSISTENT, compaction_threshold=32)
    assert opt.compaction_threshold_used == 32
    r.close()
    torch.cuda.synchronize()
    assert free0 - torch.cuda.mem_get_info()[0] < (16 << 20)
