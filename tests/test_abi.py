"""The C ABI on a machine without a GPU: the library loads, exports every declared entry point,
agrees on the data-contract layout, and refuses cleanly when there is no device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from slimtracin_b200 import api, build, structs as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    build.build()
    return api.lib()


def test_every_declared_function_is_exported(L):
    names = api.declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def layout_names():
    text = open(os.path.join(ROOT, "include", "slimtracin_layout.h")).read()
    return re.findall(r"ST_LAYOUT_(?:STRUCT|FIELD)\(([A-Za-z]+)(?:, ([A-Za-z_]+))?\)", text)


def test_layout_matches_python_mirror(L):
    for name, cls in S.STRUCTS.items():
        assert L.st_layout_query(name.encode()) == C.sizeof(cls), name
    for s, f in layout_names():
        if f and s in S.STRUCTS:
            pyf = f if f != "is" else "is_"
            if pyf in dict(S.STRUCTS[s]._fields_):
                assert L.st_layout_query(f"{s}.{f}".encode()) == getattr(S.STRUCTS[s], pyf).offset, (s, f)


@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")
def test_layout_matches_reference_headers(L):
    ref = oracle.reference()
    names = layout_names()
    assert len(names) > 150
    for s, f in names:
        q = (s + ("." + f if f else "")).encode()
        assert L.st_layout_query(q) == ref.ref_layout_query(q), q


def test_status_strings(L):
    for code in range(0, 13):
        assert L.st_strerror(code) and L.st_strerror(code) != b"unknown status"
    assert L.st_strerror(99) == b"unknown status"


def test_init_without_device_reports_no_device(L):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    cfg = api.st_config(0, 0, 0, 0)
    assert L.st_init(C.byref(ctx), C.byref(cfg)) == 2   # ST_ERR_NO_DEVICE
    assert not ctx.value


def test_null_arguments_are_rejected(L):
    assert L.st_init(None, None) == 1                    # ST_ERR_INVALID_ARG
    assert L.st_render_scene(None, 0, None, None) == 1
    assert L.st_upload_scene(None, 0, None) == 1
    assert L.st_layout_query(None) == -1
    assert L.st_layout_query(b"NoSuchStruct") == -1
    # ingestion: host-side checks that need no device
    assert L.st_obj_mesh_bytes(b"/nonexistent/none.obj") == -1
    assert L.st_obj_mesh_bytes(None) == -1
    assert L.st_obj_to_mesh(None, b"x.obj", 0, api.ST_BVH_LBVH30, None, None, 0) == 1
    assert L.st_bake_texture(None, None, 4, 4, 24, 1, 1, None, None, 0) == 1


API_STRUCTS = ["st_config", "st_render_options", "st_view", "st_batch_options", "st_serve_config", "st_request",
               "st_result", "st_pick_result"]


def _header_enums():
    """Every `NAME = value` of the header's enums."""
    text = open(os.path.join(ROOT, "include", "slimtracin_b200.h")).read()
    out = {}
    for body in re.findall(r"enum \w+ \{(.*?)\};", text, re.S):
        for name, value in re.findall(r"(ST_\w+)\s*=\s*(-?\d+)", body):
            out[name] = int(value)
    return out


def test_api_structs_and_enums_match_the_header(tmp_path):
    """The ctypes mirror of the entry points' own structs (api.py) against the header compiled by gcc:
    every size and field offset, and every enum constant the binding names."""
    lines = []
    for s in API_STRUCTS:
        cls = getattr(api, s)
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    src = tmp_path / "probe.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "slimtracin_b200.h"\nint main(void) {\n'
                   + "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "probe"
    assert os.system(f"gcc -std=c11 -I{ROOT}/include {src} -o {exe}") == 0
    got = dict(line.split() for line in os.popen(str(exe)).read().splitlines())
    for s in API_STRUCTS:
        cls = getattr(api, s)
        assert int(got[s]) == C.sizeof(cls), s
        for f, _ in cls._fields_:
            assert int(got[f"{s}.{f}"]) == getattr(cls, f).offset, (s, f)
    enums = _header_enums()
    py = {"ST_OK": api.ST_OK, "ST_ERR_INVALID_ARG": api.ST_ERR_INVALID_ARG, "ST_ERR_BUDGET": api.ST_ERR_BUDGET,
          "ST_ERR_BAD_SCENE": api.ST_ERR_BAD_SCENE, "ST_ERR_IO": api.ST_ERR_IO,
          "ST_ERR_NOT_READY": api.ST_ERR_NOT_READY, "ST_ERR_TIMEOUT": api.ST_ERR_TIMEOUT,
          "ST_BVH_LBVH30": api.ST_BVH_LBVH30, "ST_BVH_BINNED_SAH": api.ST_BVH_BINNED_SAH,
          "ST_BVH_REFIT": api.ST_BVH_REFIT, "ST_BVH_REF_SAH": api.ST_BVH_REF_SAH, "ST_OVERLAY_BVH": api.OVERLAY_BVH, "ST_OVERLAY_SSB": api.OVERLAY_SSB,
          "ST_LAUNCH_AUTOTUNED": api.LAUNCH_AUTOTUNED, "ST_LAUNCH_PER_VIEW": api.LAUNCH_PER_VIEW,
          "ST_LAUNCH_PERSISTENT": api.LAUNCH_PERSISTENT}
    for name, value in py.items():
        assert enums[name] == value, name
    counters = sorted((v, k) for k, v in enums.items() if k.startswith("ST_CNT_") and k != "ST_CNT_COUNT")
    assert [k[len("ST_CNT_"):].lower() for _, k in counters] == api.COUNTER_NAMES[:len(counters)]


def test_renderer_is_a_context_manager(L):
    """Without a device the constructor raises STError (ST_ERR_NO_DEVICE); the with-statement
    protocol closes a context exactly once."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.STError):
        api.Renderer(device=0)
    r = api.Renderer.__new__(api.Renderer)
    r.L, r.ctx = L, C.c_void_p()
    with r as same:
        assert same is r
    r.close()                       # idempotent on a closed context
    assert not r.ctx


def _chain(depth):
    """A reference-layout BVH whose every internal node has a one-item leaf on the left and the next
    internal node on the right, down to depth `depth` (its last pair is two leaves)."""
    nodes = np.zeros(1 + 2 * depth, dtype=S.BVHNODE_DT)
    item = 0
    for d in range(depth):
        f = 1 + 2 * d
        nodes[2 * d if d else 0]["first_child_id"] = f
        nodes[f]["first_child_id"], nodes[f]["child_count"] = item, 1
        item += 1
    nodes[2 * depth]["first_child_id"], nodes[2 * depth]["child_count"] = item, 1
    return nodes, item + 1


def test_validate_bvh(L):
    """st_validate_bvh: the host-side check the uploads make, without a device."""
    ok = api.ST_OK
    bad = api.ST_ERR_BAD_SCENE
    nodes, items = _chain(5)
    assert L.st_validate_bvh(nodes.ctypes.data, len(nodes), items, 5) == ok
    assert L.st_validate_bvh(None, len(nodes), items, 5) == api.ST_ERR_INVALID_ARG
    assert L.st_validate_bvh(nodes.ctypes.data, 0, items, 5) == bad
    assert L.st_validate_bvh(nodes.ctypes.data, len(nodes), items - 1, 5) == bad      # a leaf past the items
    assert L.st_validate_bvh(nodes.ctypes.data, len(nodes), items, 63) == bad         # stated height too large
    broken = nodes.copy()
    broken[2]["first_child_id"] = len(nodes) - 1                                      # a pair past the array
    assert L.st_validate_bvh(broken.ctypes.data, len(nodes), items, 5) == bad
    shared = nodes.copy()
    shared[2]["first_child_id"] = 1                                                   # a cycle back to pair 1
    assert L.st_validate_bvh(shared.ctypes.data, len(nodes), items, 5) == bad
    even = nodes.copy()
    even[0]["first_child_id"] = 2                                                     # pairs start at odd slots
    assert L.st_validate_bvh(even.ctypes.data, len(nodes), items, 5) == bad
    # the walked depth bounds the stacks whatever height is stated: 62 levels fit, 63 do not
    deep, n_items = _chain(62)
    assert L.st_validate_bvh(deep.ctypes.data, len(deep), n_items, 3) == ok
    deeper, n_items = _chain(63)
    assert L.st_validate_bvh(deeper.ctypes.data, len(deeper), n_items, 3) == bad
    # words that are no tree at all (a node array read back before anything wrote it): refused
    rng = np.random.default_rng(7)
    for _ in range(4):
        junk = np.frombuffer(rng.integers(0, 2**32, size=len(nodes) * 8, dtype=np.uint32).tobytes(),
                             dtype=S.BVHNODE_DT).copy()
        assert L.st_validate_bvh(junk.ctypes.data, len(junk), items, 5) == bad
    # a root leaf
    leaf = np.zeros(1, dtype=S.BVHNODE_DT)
    leaf[0]["child_count"] = 2
    assert L.st_validate_bvh(leaf.ctypes.data, 1, 2, 1) == ok
    assert L.st_validate_bvh(leaf.ctypes.data, 1, 1, 1) == bad
