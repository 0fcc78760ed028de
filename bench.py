"""Benchmark: Mrays/s of the 1080p PBR mesh scene on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one step = one frame): 1920x1080 viewport = 1921x1081 QCAA grid of primary rays,
trace.depth 4, one displaced icosphere of 1,310,720 triangles in 8 instances (4 Cook-Torrance,
2 glass, 2 mirror), two 1024^2 textures with 9-level mip chains, 2 emissive quads.  Seeded
synthetic data (scenes.mesh_scene); the BLAS is built on the device (binned SAH) once, before timing.

value      primary rays of all ranks / (max over ranks of the device time of K renders), inputs
           resident, outputs to device buffers; L2 flushed (256 MiB write) before every step,
           outside the timed events
e2e        the same through st_render_scene with host buffers: each step uploads the primitive
           records (H2D) and reads back the float grid and the u8 frame (D2H)
roofline   the trace kernel: algorithmic bytes per frame (device event counters on the reference
           traversal times the bytes per event of BYTES below: 32 per AABB test, 64 per triangle
           test, 72 per implicit-primitive test, 4 per leaf id, 148 per shaded hit, 12 per texel
           fetch, 24 per primary ray) / its CUDA-event time, against the measured HBM copy
           bandwidth and the L2 read rate measured in the same run (csrc/st_peaks.cu); the
           measured L2 and DRAM bytes of one launch come from the ncu capture in profiles/
cpu_baseline / --impl reference
           the reference's own renderer (oracle/_ref, compiled from the reference sources) on the
           same scene bytes, all host threads, over a bounded sample of rows
implicit16 16 implicit primitives, 3 point lights, 640x480, depth 2: the device frame beside
           the reference's CPU renderer (all host threads, and one thread)
dynamic    4096 moving primitives, TLAS rebuilt (LBVH30, binned SAH, the reference's SAH) or refit
           every frame, 1280x720 depth 2, 300 frames: build ms (API wall time) and trace ms (device
           events)
batched    64 views (resolutions from 256x256 to 1920x1080, 1-6 bounces) over 8 resident scenes:
           one st_render_batch call (launch mode, tile shape, queue depth, stack placement and
           compaction threshold autotuned, CUDA graph) against one st_render_ex call per view, both
           timed with device events around the whole sequence, and how busy the device is during
           the per-view loop
served     Poisson request streams (--rates) over the same 8 scenes, each request a view plus a
           transform update of 0-64 primitives, u8 frames to host: the library's server against
           the same requests one at a time; p50/p99 latency from arrival to completion (library
           clock) and Mrays/s over the stream
ray_segments
           primary + point-light shadow + bounce rays per frame (device counters of the same frame)
           and the value and e2e rates restated in those segments
ingest     texture baking (st_bake_texture, 1024x1024) and OBJ conversion (st_obj_to_mesh at 20,480
           and 327,680 triangles) beside the reference's loadTexture and obj2mesh on the host
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from slimtracin_b200 import dist as D, scenes, structs as S  # noqa: E402

WIDTH, HEIGHT, DEPTH = 1920, 1080, 4
METRIC = "Mrays/s at 1080p PBR mesh scene; p50/p99 latency, served vs per-frame launch"
# bytes per event of the algorithmic traffic model (reference traversal, counted on the device)
BYTES = {"aabb_tests": 32, "triangle_tests": 64, "primitive_tests": 72, "leaf_id_reads": 4,
         "shaded_hits": 84 + 64, "texel_fetches": 12, "primary_rays": 24}


def build_scene(seed_offset=0):
    sd, cam = scenes.mesh_scene(seed_offset=seed_offset)
    return sd, cam


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) >= 9 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) >= 9 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            if len(s) >= 9:
                for k, n in enumerate(names):
                    if s[5 + k].lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def reference_frame_setup(sd, cam, width=WIDTH, height=HEIGHT, depth=DEPTH):
    """The reference's per-frame set-up on a private copy of the scene: updateSceneSSB, beginDrawing."""
    import oracle
    ref = oracle.reference()
    d = sd.copy()
    sc, keep = d.to_ctypes()
    fr = scenes.Frame(width, height, cam, depth=depth)
    ref.ref_update_scene_ssb(C.byref(sc), C.byref(fr.viewport))
    ref.ref_begin_drawing(C.byref(fr.viewport))
    return ref, sc, fr, (d, keep)


def cpu_reference_sample(sd, cam, threads, budget_s, width=WIDTH, height=HEIGHT, depth=DEPTH):
    """The reference's renderer (oracle/_ref) on whole frames of the same scene bytes, repeated until
    about budget_s seconds have passed.  Returns (rays, seconds, frames)."""
    ref, sc, fr, keep = reference_frame_setup(sd, cam, width, height, depth)
    rays, total, frames = 0, 0.0, 0
    while total < budget_s or frames == 0:
        t = time.perf_counter()
        ref.ref_render_rows(C.byref(sc), C.byref(fr.viewport), threads, 0, 1, fr.grid_h)
        total += time.perf_counter() - t
        rays += fr.rays
        frames += 1
    return rays, total, frames


def bench_config(world, triangles, grid):
    """The workload both arms report, key for key: the same scene bytes, BVHs and frame."""
    return {"workload": "1080p PBR mesh scene, depth 4, 1.31M-triangle BLAS x 8 instances",
            "width": WIDTH, "height": HEIGHT, "depth": DEPTH, "rays_per_frame": grid,
            "triangles": triangles, "instances": 8, "parallelism": f"replicas x{world}",
            "l2": "device arm: 256 MiB written before every step, outside the timed events; "
                  "reference arm: host caches as they are",
            "blas": "binned SAH, the same node and Triangle bytes in both arms",
            "tlas": "LBVH30, the same node bytes in both arms"}


def reference_scene():
    """The benchmark scene with its BLAS and TLAS built on the host by the oracle's binned-SAH and
    LBVH30 builders, which give the bytes the device builders give (the full-size BLAS is compared
    byte for byte on the GPU).  The reference's own full-sweep SAH over 1.31M triangles takes more
    than ten minutes, so it is not the arm's input."""
    import tests.helpers as H
    sd, cam = build_scene()
    for md in sd.meshes:
        H.blas_sah(md, "binned")
    H.tlas_lbvh(sd)
    return sd, cam


def run_reference_arm(args):
    rank, world, _ = D.env()
    if rank != 0:
        return 0
    import oracle
    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libslimref.so is not built"}))
        return 0
    threads = os.cpu_count() or 1
    sd, cam = reference_scene()
    ref, sc, fr, keep = reference_frame_setup(sd, cam)

    def frame():
        ref.ref_render_rows(C.byref(sc), C.byref(fr.viewport), threads, 0, 1, fr.grid_h)

    # untimed warm-up frames; the last one's time caps the steps so that the timed region stays
    # near two minutes at most
    for _ in range(args.warmup):
        t0 = time.perf_counter()
        frame()
        frame_s = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(120.0 / max(frame_s, 1e-3))))
    total, rays = 0.0, 0
    for _ in range(steps):
        t = time.perf_counter()
        frame()
        total += time.perf_counter() - t
        rays += fr.rays
    value = rays / total / 1e6
    grid = (WIDTH + 1) * (HEIGHT + 1)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded mesh scene: displaced icosphere, Perlin textures; no dataset)",
            "config": bench_config(world, sd.meshes[0].triangle_count, grid),
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                             "sample": f"{steps} whole 1921x1081 frames, the reference's rayTrace "
                                       f"(render/raytracer.h:81) per grid point on {threads} host threads, "
                                       f"{total:.1f} s; {args.warmup} untimed frames before"},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def mixed_workloads(r, big_sd, stream, rates):
    """The batched-views workload (64 views over 8 resident scenes, one graph-launched
    st_render_batch call with its launch mode autotuned vs one st_render_ex per view) and the served stream (Poisson arrivals at `rates` with
    transform updates, the library's server vs one request at a time), both with device-event or
    library-clock timing."""
    import torch
    from slimtracin_b200 import api, mixed as MX
    residents = MX.resident_scenes(big=big_sd)
    slots = MX.upload(r, residents, first_slot=1)
    rng = np.random.default_rng(1234)
    views = []
    for _ in range(64):
        si, w, h, d = MX.random_view(rng, len(residents))
        views.append((slots[si], residents[si], scenes.Frame(w, h, MX.random_camera(rng, residents[si]), depth=d,
                                                             with_pixels=False, with_float=False)))
    rays = sum(fr.rays for _, _, fr in views)
    biggest = max(fr.rays for _, _, fr in views)
    # per-view device outputs for the batch; one shared pair for the per-frame loop
    f_sizes = [fr.rays * 24 for _, _, fr in views]
    u_sizes = [fr.width * fr.height * 4 for _, _, fr in views]
    fbuf = torch.empty(sum(f_sizes), dtype=torch.uint8, device="cuda")
    ubuf = torch.empty(sum(u_sizes), dtype=torch.uint8, device="cuda")
    fptr = fbuf.data_ptr() + np.concatenate([[0], np.cumsum(f_sizes)[:-1]]).astype(np.int64)
    uptr = ubuf.data_ptr() + np.concatenate([[0], np.cumsum(u_sizes)[:-1]]).astype(np.int64)
    one_f = torch.empty(biggest * 24, dtype=torch.uint8, device="cuda")
    one_u = torch.empty(biggest * 4, dtype=torch.uint8, device="cuda")
    per_frame = MX.PerFrame(r, views, one_f.data_ptr(), one_u.data_ptr())
    batch = MX.Batch(r, views, [int(x) for x in fptr], [int(x) for x in uptr], use_graph=True)

    def timed(fn, reps=3):
        fn()                      # warm-up (and, for the batch, autotuning and graph capture)
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
            fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return float(np.median(out))

    pf_ms = timed(per_frame.run)
    # how busy the device is while the per-frame loop runs: if the views' renders already fill most
    # of the elapsed time, no batching of the same rays can go faster than the busy time allows
    pf_busy_ms, pf_trace_ms = per_frame.device_ms()
    b_ms = timed(batch.run)
    batched = {"views": len(views), "scenes": [x.name for x in residents], "rays": rays,
               "per_frame_ms": pf_ms, "batch_ms": b_ms,
               "per_frame_mrays_s": rays / pf_ms / 1e3, "batch_mrays_s": rays / b_ms / 1e3,
               "speedup": pf_ms / b_ms,
               "per_frame_busy_fraction": pf_busy_ms / pf_ms, "per_frame_trace_fraction": pf_trace_ms / pf_ms,
               "speedup_bound_if_gaps_removed": pf_ms / pf_trace_ms,
               "tile_shape": batch.opt.tile_shape_used,
               "stack_placement": batch.opt.stack_placement_used, "launch_mode": batch.opt.launch_mode_used,
               "chunk": batch.opt.chunk_used, "graph_replayed": batch.opt.graph_replayed,
               "compaction_threshold": batch.opt.compaction_threshold_used, "parked_rays": batch.opt.parked_rays}
    del fbuf, ubuf, one_f, one_u
    served = []
    if rates:
        # a short stream first: the server's staging, arenas and scene versions reach their sizes
        MX.Stream(residents, slots, 200.0, 60, seed=499).serve(r)
    for k, rate in enumerate(rates):
        count = int(min(max(rate * 3.0, 60), 1500))
        stream_k = MX.Stream(residents, slots, rate, count, seed=500 + k)
        srv = MX.latency_summary(stream_k.serve(r))
        pf = MX.latency_summary(stream_k.per_frame(r))
        served.append({"rate_req_s": rate, "requests": count, "served": srv, "per_frame": pf})
    # the highest swept rate at which 1080p requests still finish within 33 ms at the 99th percentile
    ok = [x["rate_req_s"] for x in served if x["served"].get("p99_1080p_ms", 0.0) <= 33.0]
    knee = {"served_max_rate_p99_1080p_le_33ms": max(ok) if ok else None,
            "per_frame_max_rate_p99_1080p_le_33ms":
                max([x["rate_req_s"] for x in served if x["per_frame"].get("p99_1080p_ms", 0.0) <= 33.0], default=None)}
    return {"batched": batched, "served": served, "served_knee": knee}


def dynamic_tlas(r, frames, cpu_reference):
    """The moving scene: 4096 implicit primitives, the TLAS rebuilt (LBVH30, binned SAH, or the
    reference's own SAH on the first 30 frames) or refit every frame, 1280x720 depth 2.  Per frame: the primitive records go up (whole array), the TLAS
    is updated through st_update_scene_bvh (wall time of the call, which includes its validity
    check of the new node array), and the frame is traced (device events)."""
    import torch
    from slimtracin_b200 import api
    L = api.lib()
    out = {"primitives": 4096, "frames": frames, "width": 1280, "height": 720, "depth": 2}
    slot = 12
    # the reference's own SAH (ST_BVH_REF_SAH) is a parity mode, timed on the first 30 frames
    for name, mode, n_frames in (("lbvh30", api.ST_BVH_LBVH30, frames), ("binned_sah", api.ST_BVH_BINNED_SAH, frames),
                                 ("refit", api.ST_BVH_REFIT, frames), ("ref_sah", api.ST_BVH_REF_SAH, min(frames, 30))):
        sd, cam = scenes.moving_scene()
        r.upload(slot, sd, tlas=None)
        r.build_tlas(slot, sd, api.ST_BVH_LBVH30)     # the topology a refit keeps
        fr = scenes.Frame(1280, 720, cam, depth=2, with_pixels=False, with_float=False)
        dev_f = torch.empty(fr.rays * 24, dtype=torch.uint8, device="cuda")
        dev_u = torch.empty(1280 * 720 * 4, dtype=torch.uint8, device="cuda")
        sc, keep = sd.to_ctypes()
        opt = api.st_render_options()
        opt.device_outputs, opt.out_float, opt.out_u8 = 1, dev_f.data_ptr(), dev_u.data_ptr()
        up_ms, build_ms, trace_ms = [], [], []
        for _ in range(n_frames):
            scenes.advance_moving_scene(sd, 1)           # in place: sc.primitives sees the new records
            t0 = time.perf_counter()
            r._check(L.st_upload_primitives(r.ctx, slot, C.byref(sc)), "st_upload_primitives")
            t1 = time.perf_counter()
            r._check(L.st_update_scene_bvh(r.ctx, slot, None, mode), "st_update_scene_bvh")
            t2 = time.perf_counter()
            r._check(L.st_render_ex(r.ctx, slot, C.byref(sc), C.byref(fr.viewport), C.byref(opt)), "st_render_ex")
            up_ms.append((t1 - t0) * 1e3)
            build_ms.append((t2 - t1) * 1e3)
            trace_ms.append(opt.trace_ms)
        out[name] = {"frames": n_frames, "build_ms_p50": float(np.median(build_ms)),
                     "build_ms_p99": float(np.percentile(build_ms, 99)),
                     "upload_ms_p50": float(np.median(up_ms)),
                     "trace_ms_p50": float(np.median(trace_ms)), "trace_ms_last": float(trace_ms[-1]),
                     "mrays_s": fr.rays / (float(np.median(trace_ms)) / 1e3) / 1e6}
        r.free(slot)
    if cpu_reference:
        # the reference's own updateSceneBVH (top-down SAH on one host thread), a bounded sample
        try:
            import oracle
            if oracle.reference_available():
                ref = oracle.reference()
                sd, _ = scenes.moving_scene()
                sc, keep = sd.to_ctypes()
                ts = []
                for _ in range(5):
                    scenes.advance_moving_scene(sd, 1)
                    t = time.perf_counter()
                    ref.ref_update_scene_bvh(C.byref(sc))
                    ts.append((time.perf_counter() - t) * 1e3)
                out["reference_cpu_build_ms_p50"] = float(np.median(ts))
        except Exception as ex:  # reported, never required
            out["reference_cpu_build_ms_p50"] = f"failed: {ex}"
    return out


def implicit16_section(r, cpu_reference):
    """The implicit16 scene (16 implicit primitives, 3 point lights, 640x480, depth 2): the device
    frame (device outputs, trace kernel by CUDA events) beside the reference's CPU renderer on the
    same scene."""
    import torch
    from slimtracin_b200 import api
    sd, cam = scenes.implicit16_scene()
    slot = 13
    r.upload(slot, sd, tlas=None)
    r.build_tlas(slot, sd, api.ST_BVH_BINNED_SAH)
    fr = scenes.Frame(640, 480, cam, depth=2, with_pixels=False, with_float=False)
    dev_f = torch.empty(fr.rays * 24, dtype=torch.uint8, device="cuda")
    dev_u = torch.empty(640 * 480 * 4, dtype=torch.uint8, device="cuda")
    for _ in range(5):
        r.render_device(slot, sd, fr, dev_f.data_ptr(), dev_u.data_ptr())
    trace = [r.render_device(slot, sd, fr, dev_f.data_ptr(), dev_u.data_ptr()).trace_ms for _ in range(50)]
    out = {"width": 640, "height": 480, "depth": 2, "rays_per_frame": fr.rays,
           "gpu_trace_ms_p50": float(np.median(trace)), "gpu_mrays_s": fr.rays / float(np.median(trace)) / 1e3}
    r.free(slot)
    if cpu_reference:
        try:
            import oracle
            if oracle.reference_available():
                import tests.helpers as H
                ref_sd = sd.copy()
                H.tlas_sah(ref_sd, "ref")
                threads = os.cpu_count() or 1
                rays, dt, frames = cpu_reference_sample(ref_sd, cam, threads, 3.0, 640, 480, 2)
                rays1, dt1, frames1 = cpu_reference_sample(ref_sd, cam, 1, 0.0, 640, 480, 2)
                out.update({"cpu_mrays_s": rays / dt / 1e6, "cpu_threads": threads,
                            "cpu_1thread_frame_ms": dt1 / frames1 * 1e3})
        except Exception as ex:  # reported, never required
            out["cpu_mrays_s"] = f"failed: {ex}"
    return out


def ingest_section(r, cpu_reference):
    """Texture ingestion: loadTexture (bmp2texture.c:324) of the 1024x1024 RGB texture the mesh scene uses,
    on the device through st_bake_texture (API wall time: image upload, bake, quads download into
    host memory) beside the reference's CPU baker on one thread."""
    import ctypes as C
    L = r.L
    rgb = scenes.perlin_textures(1024, 0x5EED0001)[0]
    comps = np.ascontiguousarray(rgb[..., :3])
    need = L.st_texture_bytes(1024, 1024, 1)
    mem = np.zeros(need, dtype=np.uint8)
    tex = S.Texture()
    ts = []
    for k in range(8):
        t0 = time.perf_counter()
        st = L.st_bake_texture(r.ctx, comps.ctypes.data, 1024, 1024, 24, 1, 1, C.byref(tex), mem.ctypes.data, need)
        ts.append((time.perf_counter() - t0) * 1e3)
        if st != 0:
            return {"texture_bake": f"failed: status {st}"}
    out = {"texture": "1024x1024 RGB, wrap, 9 mips", "bytes_out": int(need),
           "device_bake_ms_p50": float(np.median(ts[3:]))}
    # obj2mesh: a displaced icosphere written as OBJ text (positions, uvs, normals), converted on
    # the device (parse on the host's threads, device edges and binned-SAH BLAS) and by the
    # reference's converter (full-sweep SAH, quadratic edge search) at the size it finishes in
    import tempfile
    tmp = tempfile.mkdtemp()

    def write_obj(path, md):
        with open(path, "w") as f:
            f.write("\n".join("v %.9g %.9g %.9g" % tuple(p) for p in md.positions) + "\n")
            f.write("\n".join("vt %.9g %.9g" % tuple(t) for t in md.uvs) + "\n")
            f.write("\n".join("vn %.9g %.9g %.9g" % tuple(n) for n in md.normals) + "\n")
            f.write("\n".join("f %d/%d/%d %d/%d/%d %d/%d/%d" % (a, a, a, b, b, b, c, c, c)
                               for a, b, c in md.indices + 1) + "\n")

    objs = {}
    for sub in (5, 7):
        md = scenes.displaced_icosphere(sub, 0x5EED0001)
        path = os.path.join(tmp, f"ico{sub}.obj")
        write_obj(path, md)
        need = L.st_obj_mesh_bytes(path.encode())
        omem = np.zeros(need, dtype=np.uint8)
        m = S.Mesh()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            st = L.st_obj_to_mesh(r.ctx, path.encode(), 0, 2, C.byref(m), omem.ctypes.data, need)
            ts.append((time.perf_counter() - t0) * 1e3)
        objs[sub] = path
        out[f"obj_{len(md.indices)}_triangles_device_ms_p50"] = float(np.median(ts)) if st == 0 else f"failed: status {st}"
    if cpu_reference:
        try:
            import oracle
            if oracle.reference_available():
                ref = oracle.reference()
                t0 = time.perf_counter()
                ref.obj2mesh(objs[5].encode(), os.path.join(tmp, "ref.mesh").encode(), False)
                out["obj_20480_triangles_reference_cpu_ms"] = (time.perf_counter() - t0) * 1e3
        except Exception as ex:  # reported, never required
            out["obj_20480_triangles_reference_cpu_ms"] = f"failed: {ex}"
    if cpu_reference:
        try:
            import oracle
            if oracle.reference_available():
                ref = oracle.reference()
                rts = []
                for _ in range(3):
                    rt = S.Texture()
                    t0 = time.perf_counter()
                    ref.ref_load_texture(C.byref(rt), 1024, 1024, 1, 1, comps.ctypes.data, 24)
                    rts.append((time.perf_counter() - t0) * 1e3)
                    ref.ref_free_texture(C.byref(rt))
                out["reference_cpu_bake_ms_p50"] = float(np.median(rts))
        except Exception as ex:  # reported, never required
            out["reference_cpu_bake_ms_p50"] = f"failed: {ex}"
    return out


def measure_l2_gbs(device):
    """The L2 read rate: libst_peaks.so's kernel (csrc/st_peaks.cu) reads a 48 MB buffer, which stays
    in the 126 MB L2, 400 times in one launch with 128-bit L1-bypassing loads (CUDA events).  The
    denominator of the trace kernel's L2 fraction."""
    from slimtracin_b200 import build
    L = C.CDLL(build.PEAKS_LIB)
    L.st_peak_l2_read_gbs.argtypes = [C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_double)]
    L.st_peak_l2_read_gbs.restype = C.c_int
    best = 0.0
    for _ in range(3):
        g = C.c_double()
        st = L.st_peak_l2_read_gbs(device, 48 << 20, 400, C.byref(g))
        if st != 0:
            return None
        best = max(best, g.value)
    return best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the batched-views and served-stream sections")
    ap.add_argument("--rates", default="50,100,200,500,1000,2000", help="served-stream arrival rates (req/s)")
    ap.add_argument("--dynamic-frames", type=int, default=300, help="config-2 frames (0 skips the section)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    from slimtracin_b200 import api, build

    rank, world, local = D.env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    build.build()

    # ---- scene (seeded; every rank renders its own replica) -----------------------------------
    sd, cam = build_scene()
    r = api.Renderer(device=local)
    for md in sd.meshes:
        r.build_blas(md, api.ST_BVH_BINNED_SAH)
        md.device_built = True
    r.upload(0, sd, tlas=None)
    r.build_tlas(0, sd, api.ST_BVH_LBVH30)
    frame = scenes.Frame(WIDTH, HEIGHT, cam, depth=DEPTH)
    grid = frame.rays

    stream = torch.cuda.ExternalStream(r.stream)
    out_float = torch.empty(grid * 24, dtype=torch.uint8, device="cuda")
    out_u8 = torch.empty(WIDTH * HEIGHT * 4, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # ---- work counters (instrumented kernel, untimed) -----------------------------------------
    ctr_frame = scenes.Frame(WIDTH, HEIGHT, cam, depth=DEPTH)
    opt = r.render(0, sd, ctr_frame, count_work=True, skip_float_copy=True)
    counters = api.counters_dict(opt)
    bytes_alg = sum(BYTES[k] * counters[k] for k in BYTES)
    segments = counters["primary_rays"] + counters["shadow_rays"] + counters["bounce_rays"]

    # the call's arguments are built once, so that a step times st_render_ex and not Python
    L = api.lib()
    scene_args, scene_keep = sd.to_ctypes()
    dev_opt = api.st_render_options()
    dev_opt.device_outputs, dev_opt.out_float, dev_opt.out_u8 = 1, out_float.data_ptr(), out_u8.data_ptr()
    dev_call = (r.ctx, 0, C.byref(scene_args), C.byref(frame.viewport), C.byref(dev_opt))

    def render_dev():
        st = L.st_render_ex(*dev_call)
        assert st == 0, st
        return dev_opt.trace_ms

    def step():
        with torch.cuda.stream(stream):
            flush.zero_()
        return render_dev()

    trace_ms = []
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        # clocks are sampled from the warm-up on, so short timed regions still get samples under load
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            evs[k][0].record(stream)
            t_ms = render_dev()
            evs[k][1].record(stream)
            trace_ms.append(t_ms)
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = D.max_over_ranks(sum(step_ms), device="cuda")       # the slowest rank's device time
    if world > 1:
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * grid / (ms_per_step / 1e3) / 1e6

    # ---- end to end through st_render_scene with pinned host buffers ----------------------------
    pinned_float = torch.empty(grid * 24, dtype=torch.uint8, pin_memory=True)
    pinned_u8 = torch.empty(WIDTH * HEIGHT * 4, dtype=torch.uint8, pin_memory=True)
    e2e_frame = scenes.Frame(WIDTH, HEIGHT, cam, depth=DEPTH)
    e2e_frame.grid.float_pixels = pinned_float.data_ptr()
    e2e_frame.grid.pixels = pinned_u8.data_ptr()
    prims_pinned = torch.from_numpy(sd.primitives.view(np.uint8).copy()).pin_memory()
    prim_view = prims_pinned.numpy().view(S.PRIMITIVE_DT)
    sc, keep = sd.to_ctypes()
    sc.primitives = prims_pinned.data_ptr()
    L = api.lib()

    def e2e_step():
        st = L.st_upload_primitives(r.ctx, 0, C.byref(sc))
        st |= L.st_render_scene(r.ctx, 0, C.byref(sc), C.byref(e2e_frame.viewport))
        assert st == 0, st

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = D.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    e2e_value = world * grid * args.steps / (e2e_ms / 1e3) / 1e6
    h2d = len(prim_view) * S.PRIMITIVE_DT.itemsize
    d2h = grid * 24 + WIDTH * HEIGHT * 4

    mixed = None if args.no_mixed else mixed_workloads(r, sd, stream, [float(x) for x in args.rates.split(",") if x])
    dynamic = dynamic_tlas(r, args.dynamic_frames, rank == 0 and world == 1 and not args.no_cpu_baseline) \
        if args.dynamic_frames > 0 else None
    l2_gbs = measure_l2_gbs(local)
    implicit16 = implicit16_section(r, rank == 0 and world == 1 and not args.no_cpu_baseline)
    ingest = ingest_section(r, rank == 0 and world == 1 and not args.no_cpu_baseline)

    # ---- roofline of the trace kernel -----------------------------------------------------------
    trace_avg_ms = sum(trace_ms) / len(trace_ms)
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks and "hbm_gbs" in peaks else 6650.0
    achieved = bytes_alg / (trace_avg_ms / 1e3) / 1e9
    traffic, l2_traffic = None, None
    prof = os.path.join(ROOT, "profiles", "trace_kernel_mesh_1080p_traffic.json")
    if os.path.exists(prof):
        try:
            pj = json.load(open(prof))
            traffic, l2_traffic = pj.get("dram_bytes_per_launch"), pj.get("l2_bytes_per_launch")
        except Exception:
            traffic = None

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                import oracle
                if oracle.reference_available():
                    threads = os.cpu_count() or 1
                    # the device-built BLAS and TLAS as read back: the frame the device traced
                    rays, dt, frames = cpu_reference_sample(sd, cam, threads, 10.0)
                    cpu = {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
                           "sample": f"{frames} whole 1921x1081 frames of the same scene bytes, "
                                     f"{dt:.1f} s on {threads} host threads"}
            except Exception as ex:  # the baseline is reported, never required
                cpu = {"value": None, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"failed: {ex}"}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded mesh scene: displaced icosphere, Perlin textures; no dataset)",
            "config": bench_config(world, sd.meshes[0].triangle_count, grid),
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "api": "st_upload_primitives + st_render_scene, pinned host buffers"},
            "gpu_launches": 4 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "trace_kernel", "kernel_ms": trace_avg_ms,
                         "bytes_alg_per_launch": bytes_alg,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6.65 TB/s",
                         "l2_peak": l2_gbs, "l2_frac": achieved / l2_gbs if l2_gbs else None,
                         "l2_traffic_frac": (l2_traffic / (trace_avg_ms / 1e3) / 1e9 / l2_gbs)
                         if (l2_gbs and l2_traffic) else None,
                         "l2_traffic": l2_traffic,
                         "l2_peak_source": "48 MB L2-resident buffer read 400 times in one launch "
                                           "(csrc/st_peaks.cu, CUDA events), measured in this run"},
            "counters": counters,
            "ray_segments": {"per_frame": segments, "mrays_s": value * segments / grid,
                             "e2e_mrays_s": e2e_value * segments / grid,
                             "counted": "primary + point-light shadow + bounce rays, device counters"},
            "implicit16": implicit16,
            "dynamic_tlas": dynamic,
            "ingest": ingest,
            "batched": mixed["batched"] if mixed else None,
            "served": mixed["served"] if mixed else None,
            "served_knee": mixed["served_knee"] if mixed else None,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    r.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
