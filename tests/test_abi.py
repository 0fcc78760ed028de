"""The C ABI on a machine without a GPU: the library loads, exports every declared entry point,
agrees on the data-contract layout, and refuses cleanly when there is no device."""
import ctypes as C
import os
import re

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
