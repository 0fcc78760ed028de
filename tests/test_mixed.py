"""Host logic of the mixed-request workloads (slimtracin_b200/mixed.py): the seeded generators the
batched and served measurements draw from, and the latency summary they are reported through."""
import math

import numpy as np

from slimtracin_b200 import mixed as MX, scenes


def _resident(seed_offset=0):
    sd, _ = scenes.implicit16_scene(seed_offset=seed_offset)
    return MX.Resident("implicit16", sd, (0.0, 0.0, 0.0), 15.0, 2.0, "sah")


def test_poisson_arrivals_are_seeded_and_have_the_rate():
    a = MX.poisson_arrivals(np.random.default_rng(7), 1000.0, 20000)
    b = MX.poisson_arrivals(np.random.default_rng(7), 1000.0, 20000)
    assert np.array_equal(a, b)
    gaps = np.diff(np.concatenate([[0.0], a]))
    assert (gaps > 0).all()
    assert abs(gaps.mean() - 1e-3) < 0.03e-3          # mean inter-arrival 1/rate within 3 %
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential: coefficient of variation 1


def test_random_views_cover_the_stated_sets():
    rng = np.random.default_rng(3)
    views = [MX.random_view(rng, 8) for _ in range(4000)]
    assert {v[0] for v in views} == set(range(8))
    assert {(v[1], v[2]) for v in views} == set(MX.RESOLUTIONS)
    assert {v[3] for v in views} == set(range(1, 7))


def test_random_camera_orbits_the_target():
    res = _resident()
    rng = np.random.default_rng(5)
    for _ in range(200):
        cam = MX.random_camera(rng, res)
        p = np.array(cam.position)
        horiz = math.hypot(p[0] - res.target[0], p[2] - res.target[2])
        assert 0.8 * res.radius - 1e-9 <= horiz <= 1.2 * res.radius + 1e-9
        assert 0.5 * res.height - 1e-9 <= p[1] - res.target[1] <= res.height + 1e-9
        # looks at the target: the camera's forward column points from the position to it
        fwd = cam.matrix_cols()[:, 2]
        d = np.array(res.target) - p
        assert np.allclose(fwd, d / np.linalg.norm(d), atol=1e-9)


def test_random_update_moves_only_the_returned_primitives():
    res = _resident()
    before = res.sd.primitives.copy()
    rng = np.random.default_rng(11)
    seen_empty = seen_some = False
    for _ in range(60):
        prev = res.sd.primitives.copy()
        recs, ids = MX.random_update(rng, res, max_count=8, step=0.05)
        if recs is None:
            seen_empty = True
            assert np.array_equal(res.sd.primitives, prev)
            continue
        seen_some = True
        n = len(prev)
        assert 1 <= len(ids) <= 8 and ids.dtype == np.uint32
        assert np.array_equal(ids, np.unique(ids)) and ids.max() < n
        # the records are the scene's host rows after the move
        assert np.array_equal(recs, res.sd.primitives[ids])
        others = np.setdiff1d(np.arange(n), ids)
        assert np.array_equal(res.sd.primitives[others], prev[others])
        moved = res.sd.primitives[ids]
        assert (np.abs(moved["position"] - prev[ids]["position"]) <= 0.05 + 1e-6).all()
        q = moved["rotation"].astype(np.float64)
        assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-6)
        # a small rotation: the angle between old and new orientation is at most `step`
        dots = np.abs((q * prev[ids]["rotation"].astype(np.float64)).sum(1))
        assert (2 * np.arccos(np.minimum(dots, 1.0)) <= 0.05 + 1e-5).all()
        # nothing but position and rotation changes
        for f in before.dtype.names:
            if f not in ("position", "rotation"):
                assert np.array_equal(moved[f], prev[ids][f]), f
    assert seen_empty and seen_some


def test_latency_summary():
    # (arrival, completion, rays, status, width, height, batch size)
    res = [(float(k), float(k) + (k + 1) * 1e-3, 1000, 0, 640, 480, 2) for k in range(99)]
    res.append((99.0, 99.5, 2_000_000, 0, 1920, 1080, 4))
    res.append((100.0, 100.010, 500, 5, 256, 256, 1))     # refused: counted in latency, not in rays
    s = MX.latency_summary(res)
    lat = np.array([(c - a) * 1e3 for a, c, *_ in res])
    assert s["requests"] == 101
    assert math.isclose(s["accepted"], 100 / 101)
    assert math.isclose(s["p50_ms"], float(np.percentile(lat, 50)))
    assert math.isclose(s["p99_ms"], float(np.percentile(lat, 99)))
    assert math.isclose(s["p99_1080p_ms"], 500.0)
    span = 100.010 - 0.0
    assert math.isclose(s["mrays_s"], (99 * 1000 + 2_000_000) / span / 1e6)
    assert math.isclose(s["mean_batch"], (99 * 2 + 4 + 1) / 101)
