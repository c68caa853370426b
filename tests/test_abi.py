"""CPU tests of the boundary: the library loads, exports every symbol the header declares,
and rejects bad arguments without needing a GPU."""
import ctypes
import os
import re
from ctypes import byref, c_void_p

from eos_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "eos_c.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eos_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = L.load()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    bound = {s[0] for s in L.SIGNATURES}
    assert set(names) == bound


def test_struct_layouts_match_header():
    assert ctypes.sizeof(L.Material) == 40
    assert ctypes.sizeof(L.Light) == 24
    assert ctypes.sizeof(L.Camera) == 56
    assert ctypes.sizeof(L.RenderParams) == 44
    assert ctypes.sizeof(L.BuildParams) == 16
    assert ctypes.sizeof(L.Tuning) == 28
    assert ctypes.sizeof(L.SceneInfo) == 56
    assert ctypes.sizeof(L.PathRecord) == 64
    assert ctypes.sizeof(L.Job) == 8 + 56 + 16 + 24 + 8


def test_status_strings_and_version():
    lib = L.load()
    assert lib.eos_abi_version() == 1
    for code in range(11):
        assert lib.eos_status_string(code)


def test_null_arguments_are_rejected_without_device_work():
    lib = L.load()
    assert lib.eos_ctx_create(0, None) == 1
    assert lib.eos_ctx_destroy(None) == 1
    assert lib.eos_scene_destroy(None) == 1
    assert lib.eos_render(None, None, None, None, None, None, None, None, None) == 1
    assert lib.eos_render_batch(None, None, 0, None, None) == 1
    assert lib.eos_trace_closest(None, None, None, 0, None, None) == 1
    assert lib.eos_scene_save(None, b"x.eos") == 1
    assert lib.eos_scene_load(None, b"x.eos", None) == 1


def test_no_device_reports_status_not_crash():
    import torch
    if torch.cuda.is_available():
        return
    lib = L.load()
    h = c_void_p()
    assert lib.eos_ctx_create(0, byref(h)) == 8  # EOS_ERR_NO_DEVICE


def test_python_package_fails_loudly_without_library(tmp_path):
    import pytest
    saved = L._lib
    try:
        L._lib = None
        with pytest.raises(RuntimeError):
            L.load(str(tmp_path / "missing.so"))
    finally:
        L._lib = saved


def test_context_close_destroys_its_scenes_first():
    """Scenes still alive when their Context closes (e.g. held by a traceback) are destroyed
    before the context, never after it."""
    import weakref

    from eos_b200 import api
    calls = []

    class FakeLib:
        def eos_scene_destroy(self, h):
            calls.append(("scene", h))

        def eos_ctx_destroy(self, h):
            calls.append(("ctx", h))

    ctx = api.Context.__new__(api.Context)
    ctx.lib, ctx.h, ctx._scenes = FakeLib(), "C", weakref.WeakSet()
    scs = []
    for k in range(2):
        sc = api.DeviceScene.__new__(api.DeviceScene)
        sc.lib, sc.h = ctx.lib, f"S{k}"
        ctx._scenes.add(sc)
        scs.append(sc)
    ctx.close()
    assert sorted(calls[:2]) == [("scene", "S0"), ("scene", "S1")] and calls[2] == ("ctx", "C")
    ctx.close()
    for sc in scs:
        sc.close()
    assert len(calls) == 3
