"""TEST INFRASTRUCTURE — the oracle.

Two CPU checkers for the tracing path, loaded with ctypes:
  * `restatement()` — liboracle.so, this directory's C restatement of the reference's algorithm
    (oracle.c, each function citing the reference file:line it follows);
  * `reference()`   — _ref/libslimref.so, the reference's own code compiled in place by
    ref_harness.c; used to pin the restatement and as the timed CPU baseline.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arms may import this
package.  The product (slimtracin_b200) never does.
"""
import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def build(quiet=True):
    """Build liboracle.so and, where the reference sources exist, _ref/libslimref.so."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _load(name, path):
    if name not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C {HERE}`)")
        _libs[name] = C.CDLL(path)
    return _libs[name]


def dropin():
    """oracle/_ref/libdropin.so: a host built from the reference's headers whose GPU seams call
    libslimtracin_b200 (dropin.c)."""
    lib = _load("dropin", os.path.join(HERE, "_ref", "libdropin.so"))
    lib.dropin_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    lib.dropin_frame.restype = C.c_int
    lib.dropin_shutdown.argtypes = []
    lib.dropin_shutdown.restype = None
    return lib


def dropin_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libdropin.so"))


def reference_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libslimref.so"))


def reference():
    lib = _load("ref", os.path.join(HERE, "_ref", "libslimref.so"))
    lib.ref_layout_query.restype = C.c_long
    lib.ref_layout_query.argtypes = [C.c_char_p]
    lib.ref_render_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    lib.ref_render_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32]
    lib.ref_begin_drawing.argtypes = [C.c_void_p]
    lib.ref_update_scene_ssb.argtypes = [C.c_void_p, C.c_void_p]
    lib.ref_pick.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.ref_pick.restype = C.c_int
    lib.ref_resolve.argtypes = [C.c_void_p]
    lib.ref_update_scene_bvh.argtypes = [C.c_void_p]
    lib.ref_update_mesh_bvh.argtypes = [C.c_void_p]
    lib.ref_load_mesh.restype = C.c_void_p
    lib.ref_load_mesh.argtypes = [C.c_char_p, C.c_void_p]
    lib.ref_load_texture.argtypes = [C.c_void_p, C.c_uint16, C.c_uint16, C.c_int, C.c_int, C.c_void_p, C.c_int]
    lib.ref_free_texture.argtypes = [C.c_void_p]
    lib.ref_free.argtypes = [C.c_void_p]
    lib.ref_draw_overlays.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.ref_draw_overlays.restype = C.c_int
    lib.ref_save_mesh.argtypes = [C.c_void_p, C.c_char_p]
    lib.ref_save_scene.argtypes = [C.c_void_p, C.c_char_p]
    lib.ref_load_scene.argtypes = [C.c_void_p, C.c_char_p]
    lib.ref_load_texture_file.argtypes = [C.c_void_p, C.c_char_p, C.c_uint64]
    lib.ref_load_texture_file.restype = C.c_void_p
    lib.bmp2texture.argtypes = [C.c_char_p, C.c_char_p, C.c_bool, C.c_bool]   # bmp2texture.c:364
    lib.bmp2texture.restype = C.c_int
    lib.obj2mesh.argtypes = [C.c_char_p, C.c_char_p, C.c_bool]              # obj2mesh.c:25
    lib.obj2mesh.restype = C.c_int
    return lib


def restatement():
    lib = _load("oracle", os.path.join(HERE, "liboracle.so"))
    lib.orc_render_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.orc_update_scene_ssb.argtypes = [C.c_void_p, C.c_void_p]
    lib.orc_update_scene_bvh.argtypes = [C.c_void_p]
    lib.orc_update_mesh_bvh.argtypes = [C.c_void_p]
    lib.orc_lbvh30.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p]  # aabbs, n, max_leaf, codes, order, nodes, leaf_ids, info
    lib.orc_lbvh30.restype = C.c_int
    lib.orc_primitive_aabbs.argtypes = [C.c_void_p, C.c_void_p]
    lib.orc_binned_sah.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_binned_sah.restype = C.c_int
    lib.orc_update_mesh_bvh_binned.argtypes = [C.c_void_p]
    lib.orc_update_mesh_bvh_binned.restype = C.c_int
    lib.orc_pick.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.orc_pick.restype = C.c_int
    lib.orc_draw_overlays.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.orc_draw_overlays.restype = None
    return lib
