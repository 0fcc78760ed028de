"""The serving loop (st_serve_start / st_submit / st_wait) through the C ABI: every served view equals
the same view rendered alone by st_render_scene after the same sequence of transform updates and
TLAS maintenance, whatever batches the server formed."""
import numpy as np
import pytest

from slimtracin_b200 import api, scenes, structs as S
from tests import helpers as H

pytestmark = pytest.mark.gpu

REFIT_FRACTION = 0.25


def _scenes():
    c0, cam0 = scenes.implicit16_scene()
    H.tlas_sah(c0)
    c1, cam1 = H.small_mesh_scene(subdivisions=3, texture_size=64, blas="orc")
    H.tlas_sah(c1)
    c2, cam2 = scenes.moving_scene(count=300)
    return [(c0, cam0, "host"), (c1, cam1, "host"), (c2, cam2, "lbvh")]


def _requests(c2, seed=7):
    """A stream of (scene index, w, h, depth, mode, moved ids) with transform updates of scene 2:
    small ones (refit) and large ones (rebuild)."""
    rng = np.random.default_rng(seed)
    out = []
    n2 = len(c2.primitives)
    for k in range(40):
        si = int(rng.integers(0, 3))
        w, h = int(rng.integers(24, 120)), int(rng.integers(16, 90))
        depth = int(rng.integers(1, 4))
        mode = [S.RM_BEAUTY, S.RM_BEAUTY, S.RM_NORMALS, S.RM_DEPTH][int(rng.integers(0, 4))]
        moved = None
        if si == 2 and k % 3 == 0:
            count = int(rng.integers(1, 20)) if k % 2 else int(rng.integers(100, n2))
            moved = np.sort(rng.choice(n2, count, replace=False)).astype(np.uint32)
        out.append((si, w, h, depth, mode, moved))
    return out


def test_served_views_equal_views_rendered_alone():
    scn = _scenes()
    reqs = _requests(scn[2][0])
    # the motion applied with each mutating request, precomputed on the host
    motion = scenes.SceneData.copy(scn[2][0])
    updates = []
    for si, w, h, d, m, moved in reqs:
        if moved is None:
            updates.append(None)
        else:
            scenes.advance_moving_scene(motion, 1)
            updates.append(motion.primitives[moved].copy())

    served = api.Renderer(device=0)
    alone = api.Renderer(device=0)
    try:
        for k, (sd, cam, tlas) in enumerate(scn):
            served.upload(k, sd.copy(), tlas=tlas)
            alone.upload(k, sd.copy(), tlas=tlas)
        srv = api.Server(served, max_in_flight=3, max_views_per_batch=8, refit_fraction=REFIT_FRACTION)
        frames, tickets = [], []
        try:
            for (si, w, h, d, m, moved), upd in zip(reqs, updates):
                sd, cam, _ = scn[si]
                fr = scenes.Frame(w, h, cam, depth=d, mode=m)
                frames.append(fr)
                tickets.append(srv.submit(si, sd, fr, moved=upd, moved_ids=moved))
            results = [srv.wait(t, timeout=120) for t in tickets]
        finally:
            srv.stop()
        assert all(r.status == api.ST_OK for r in results), [r.status for r in results]
        assert max(r.batch_size for r in results) > 1            # the server did batch
        for r in results:
            assert r.arrival_time <= r.launch_time <= r.completion_time
        # the same sequence, one request at a time
        n2 = len(scn[2][0].primitives)
        moved_since_build = 0          # the server refits while this stays below the fraction
        for (si, w, h, d, m, moved), upd, fr, res in zip(reqs, updates, frames, results):
            sd, cam, _ = scn[si]
            if moved is not None:
                alone.update_primitives(2, upd, moved)
                moved_since_build += len(moved)
                mode = api.ST_BVH_REFIT if moved_since_build < REFIT_FRACTION * n2 else api.ST_BVH_LBVH30
                if mode != api.ST_BVH_REFIT:
                    moved_since_build = 0
                alone.build_tlas(2, sd.copy(), mode)
            ref = scenes.Frame(w, h, cam, depth=d, mode=m)
            alone.render(si, sd, ref)
            assert res.rays == ref.rays
            assert np.array_equal(fr.float_pixels.view(np.uint8), ref.float_pixels.view(np.uint8)), (si, w, h, d, m)
            assert np.array_equal(fr.pixels.view(np.uint8), ref.pixels.view(np.uint8))
    finally:
        served.close()
        alone.close()


def test_request_over_frame_budget_is_refused():
    sd, cam = scenes.implicit16_scene()
    H.tlas_sah(sd)
    r = api.Renderer(device=0)
    try:
        r.upload(0, sd, tlas="host")
        srv = api.Server(r, frame_budget=4096)
        try:
            fr = scenes.Frame(320, 240, cam)
            res = srv.wait(srv.submit(0, sd, fr), timeout=60)
        finally:
            srv.stop()
        assert res.status == 5   # ST_ERR_BUDGET: a 320x240 grid never fits in 4 KiB
    finally:
        r.close()


def test_served_views_into_page_locked_buffers():
    """Requests whose output frames are page-locked are resolved straight into them (no staging);
    each equals the same view rendered alone."""
    import torch
    sd, cam = scenes.implicit16_scene()
    H.tlas_sah(sd)
    r = api.Renderer(device=0)
    try:
        r.upload(0, sd, tlas="host")
        sizes = [(64, 48), (96, 64), (33, 17), (128, 96)]
        frames, bufs = [], []
        for w, h in sizes:
            fr = scenes.Frame(w, h, cam, depth=2, with_pixels=False)
            buf = torch.zeros(w * h * 4, dtype=torch.uint8, pin_memory=True)
            fr.grid.pixels = buf.data_ptr()
            frames.append(fr)
            bufs.append(buf)
        srv = api.Server(r, max_in_flight=2, max_views_per_batch=4)
        try:
            tickets = [srv.submit(0, sd, fr) for fr in frames]
            results = [srv.wait(t, timeout=60) for t in tickets]
        finally:
            srv.stop()
        assert all(res.status == api.ST_OK for res in results)
        for (w, h), fr, buf in zip(sizes, frames, bufs):
            alone = scenes.Frame(w, h, cam, depth=2)
            r.render(0, sd, alone)
            assert np.array_equal(buf.numpy(), alone.pixels.view(np.uint8))
            assert np.array_equal(fr.float_pixels.view(np.uint8), alone.float_pixels.view(np.uint8))
    finally:
        r.close()
