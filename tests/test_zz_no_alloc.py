"""sg_trace_closest_host_static: the allocation-free host-buffer query.

Callers that cannot call cudaMalloc while they query (a host that owns the
whole GPU memory budget, a real-time loop that must not take the allocator's
locks) use this entry point; it stages rays and hits in an array compiled into the
library. Its results must equal sg_trace_closest_host's bit for bit, on two
calls in a row (the second call reuses the array the first one left behind).
This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import same_bits

pytestmark = pytest.mark.gpu

MAX_STATIC_RAYS = 524288


def _call_static(lib, handle, rays):
    n = rays.shape[1]
    prim = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    u = np.empty(n, np.float32)
    v = np.empty(n, np.float32)
    st = lib.sg_trace_closest_host_static(handle, rays.ctypes.data, n, prim.ctypes.data, t.ctypes.data,
                                          u.ctypes.data, v.ctypes.data, None)
    return st, (prim, t, u, v)


def test_static_entry_point_matches_host_entry_point():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import Obvh, _lib, scenes

    lib = _lib.load()
    acc = Obvh()
    acc.Build(scenes.sphere_field(32, 3, seed=31))
    batches = [np.ascontiguousarray(scenes.random_rays(200_000, seed=32)),
               np.ascontiguousarray(np.concatenate([scenes.camera_rays(300, 300, seed=33),
                                                    scenes.random_rays(50_000, seed=34)], axis=1))]
    for rays in batches:  # two calls in a row on the shared array
        st, (prim, t, u, v) = _call_static(lib, acc._h, rays)
        assert st == 0, lib.sg_last_error()
        ref = acc.GetIntersect(rays)  # sg_trace_closest_host
        assert np.array_equal(prim, ref.prim) and same_bits(t, ref.t)
        assert same_bits(u, ref.u) and same_bits(v, ref.v)


def test_static_entry_point_rejects_oversized_batch():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import Obvh, _lib, scenes

    lib = _lib.load()
    acc = Obvh()
    acc.Build(scenes.sphere_field(2, 2, seed=35))
    rays = np.zeros((8, MAX_STATIC_RAYS + 1), np.float32)
    st, _ = _call_static(lib, acc._h, rays)
    assert st == 5 and b"524288" in lib.sg_last_error()
    assert lib.sg_trace_closest_host_static(acc._h, None, 1, None, None, None, None, None) == 1
    out = np.empty(1, np.int32)
    assert lib.sg_trace_closest_host_static(acc._h, rays.ctypes.data, 0, out.ctypes.data, out.ctypes.data,
                                            None, None, ctypes.c_void_p()) == 0


def test_static_entry_point_ignores_sorted_schedule():
    """A scene tuned to the sorted schedule (which takes key and permutation
    scratch from a pool) still runs allocation-free through this entry point:
    the call runs one ray per thread, and device memory in use does not move."""
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import Obvh, _lib, scenes

    lib = _lib.load()
    acc = Obvh()
    acc.Build(scenes.sphere_field(32, 3, seed=36))
    acc.SetTuning(schedule=4)  # SG_SCHEDULE_SORTED: sorts batches of 65,536 rays or more
    rays = np.ascontiguousarray(scenes.random_rays(300_000, seed=37))
    st, first = _call_static(lib, acc._h, rays)  # loads the kernel the call uses
    assert st == 0, lib.sg_last_error()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    st, (prim, t, u, v) = _call_static(lib, acc._h, rays)
    assert st == 0, lib.sg_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    ref = acc.GetIntersect(rays)  # sg_trace_closest_host, sorted schedule
    assert np.array_equal(prim, ref.prim) and same_bits(t, ref.t)
    assert same_bits(u, ref.u) and same_bits(v, ref.v)
    assert all(np.array_equal(a.view(np.int32), b.view(np.int32)) for a, b in zip(first, (prim, t, u, v)))


def test_static_entry_point_rejects_hair_scene():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from conftest import golden
    from sort_b200 import Obvh, Scene, _lib

    lib = _lib.load()
    z = golden("hair")
    acc = Obvh()
    acc.Build(Scene(z["triangles"], z["lines"]))
    st, _ = _call_static(lib, acc._h, np.ascontiguousarray(z["rays"][:, :256]))
    assert st == 4 and b"hair" in lib.sg_last_error()
