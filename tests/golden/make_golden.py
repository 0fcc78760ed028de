"""Generate the golden fixtures from the reference's own code (oracle/_ref/libslimref.so, built in
place from the reference sources by oracle/Makefile).

    python tests/golden/make_golden.py

Writes tests/golden/golden.json (digests and small tables) and tests/golden/frames.npz (resolved
u8 frames of small renders).  Every figure comes from the reference: its renderer
(render/raytracer.h:136 via rayTrace, viewport/viewport.h:12), its SAH builders
(builder_top_down.h:272,366), its texture baker (bmp2texture.c:324) and its mesh loader
(scene/io.h:95) on the one fixture the reference ships, src/examples/monkey.mesh.
"""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from slimtracin_b200 import scenes, structs as S  # noqa: E402
from tests import helpers as H  # noqa: E402

# the reference's src/ directory: $ST_REFERENCE_SRC, else a reference checkout beside this repository
REF_SRC = os.environ.get("ST_REFERENCE_SRC") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))), "reference", "src")
MONKEY = os.path.join(REF_SRC, "examples", "monkey.mesh")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def render_cases():
    """(name, scene builder, camera, w, h, depth, mode) of the golden renders."""
    cases = []
    for mode, mname in ((S.RM_BEAUTY, "beauty"), (S.RM_DEPTH, "depth"), (S.RM_NORMALS, "normals"), (S.RM_UVS, "uvs")):
        cases.append((f"implicit16_{mname}", "implicit16", 96, 72, 2, mode))
    cases.append(("area_lights_beauty_d3", "area", 96, 72, 3, S.RM_BEAUTY))
    cases.append(("mesh_tiny_beauty_d4", "mesh_tiny", 96, 54, 4, S.RM_BEAUTY))
    cases.append(("mesh_tiny_normals", "mesh_tiny", 96, 54, 4, S.RM_NORMALS))
    cases.append(("moving256_beauty", "moving256", 96, 54, 2, S.RM_BEAUTY))
    return cases


def make_scene(kind, which="ref"):
    if kind == "implicit16":
        sd, cam = scenes.implicit16_scene()
    elif kind == "area":
        sd, cam = scenes.example_area_lights()
    elif kind == "mesh_tiny":
        sd, cam = scenes.mesh_scene(subdivisions=2, texture_size=32)
        H.blas_sah(sd.meshes[0], which)
    elif kind == "moving256":
        sd, cam = scenes.moving_scene(count=256)
    else:
        raise ValueError(kind)
    H.tlas_sah(sd, which)
    return sd, cam


def main():
    oracle.build()
    ref = oracle.reference()
    out = {"renders": {}, "tlas": {}, "textures": {}, "monkey": None}
    frames = {}
    for name, kind, w, h, depth, mode in render_cases():
        sd, cam = make_scene(kind, "ref")
        fr = H.reference_frame(sd, cam, w, h, depth=depth, mode=mode, threads=8)
        out["renders"][name] = {"kind": kind, "w": w, "h": h, "depth": depth, "mode": mode,
                                "float_sha256": sha(fr.float_pixels),
                                "tlas_sha256": sha(sd.tlas_nodes[:sd.tlas_node_count])}
        frames[name] = np.stack([fr.pixels["R"], fr.pixels["G"], fr.pixels["B"]], -1).reshape(h, w, 3)
    for kind in ("implicit16", "moving256"):
        sd, _ = make_scene(kind, "ref")
        out["tlas"][kind] = {"node_count": int(sd.tlas_node_count), "height": int(sd.tlas_height),
                             "nodes_sha256": sha(sd.tlas_nodes[:sd.tlas_node_count]),
                             "leaf_ids_sha256": sha(sd.tlas_leaf_ids)}
    rng = np.random.default_rng(1234)
    for (w, h, wrap, mip) in ((8, 8, 1, 1), (16, 8, 0, 1), (12, 10, 1, 1), (33, 17, 0, 0), (64, 64, 1, 1)):
        img = rng.integers(0, 256, size=(h, w, 3), dtype=np.uint8)
        tex = S.Texture()
        ref.ref_load_texture(C.byref(tex), w, h, wrap, mip, img.ctypes.data, 24)
        digests = []
        for m in range(tex.mip_count):
            mp = tex.mips[m]
            n = (mp.width + 1) * (mp.height + 1)
            q = np.ctypeslib.as_array((C.c_uint8 * (12 * n)).from_address(mp.texel_quads))
            digests.append([int(mp.width), int(mp.height), hashlib.sha256(q.tobytes()).hexdigest()])
        ref.ref_free_texture(C.byref(tex))
        out["textures"][f"{w}x{h}_w{wrap}_m{mip}"] = {"seed": 1234, "mips": digests}
    if os.path.exists(MONKEY):
        m = S.Mesh()
        arena = ref.ref_load_mesh(MONKEY.encode(), C.byref(m))
        t = m.triangle_count
        nodes = np.ctypeslib.as_array((C.c_uint8 * (32 * m.bvh.node_count)).from_address(m.bvh.nodes))
        leaf = np.ctypeslib.as_array((C.c_uint8 * (4 * t)).from_address(m.bvh.leaf_ids))
        tris = np.ctypeslib.as_array((C.c_uint8 * (128 * t)).from_address(m.triangles))
        out["monkey"] = {"triangles": int(t), "vertices": int(m.vertex_count), "node_count": int(m.bvh.node_count),
                         "height": int(m.bvh.height), "nodes_sha256": hashlib.sha256(nodes.tobytes()).hexdigest(),
                         "leaf_ids_sha256": hashlib.sha256(leaf.tobytes()).hexdigest(),
                         "triangles_sha256": hashlib.sha256(tris.tobytes()).hexdigest()}
        ref.ref_free(arena)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "frames.npz"), **frames)
    print("wrote", len(out["renders"]), "renders,", len(out["textures"]), "textures")


if __name__ == "__main__":
    main()
