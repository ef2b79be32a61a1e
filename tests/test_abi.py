"""The C-ABI library loads and exports every entry point include/sortgpu.h declares."""
import ctypes
import os
import re

import numpy as np

from conftest import ROOT
from sort_b200 import _lib


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sortgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_declared_symbols():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.exported_symbols())


def test_version_and_errors():
    lib = _lib.load()
    assert b"sm_100a" in lib.sg_version()
    st = lib.sg_scene_create(None, 1, None, ctypes.byref(ctypes.c_void_p()))
    assert st == 1 and b"opts" in lib.sg_last_error()
    o = _lib.BuildOpts()
    lib.sg_default_build_opts(ctypes.byref(o))
    assert (o.width, o.max_depth, o.max_leaf) == (8, 16, 8)
    o.width = 3
    tri = np.zeros((1, 9), np.float32)
    st = lib.sg_scene_create(tri.ctypes.data, 1, ctypes.byref(o), ctypes.byref(ctypes.c_void_p()))
    assert st == 1
    assert lib.sg_trace_closest(None, None, 0, None, None) == 1
    assert lib.sg_scene_destroy(None) == 0


def test_server_option_layout():
    """sg_server_opts / sg_server_stats as the Python mirror lays them out:
    the defaults the library writes land in the right fields."""
    lib = _lib.load()
    o = _lib.ServerOpts()
    o.solo_pixels = -7
    lib.sg_default_server_opts(ctypes.byref(o))
    assert (o.device, o.max_requests, o.path_slots, o.pixel_budget) == (0, 1024, 1 << 20, 1 << 24)
    assert (o.steps_per_poll, o.samples_per_claim, o.solo_pixels) == (4, 1, 0)
    assert ctypes.sizeof(_lib.ServerOpts) == 40 and ctypes.sizeof(_lib.ServerStats) == 8 * 8
