"""Transparent-shadow query (sg_trace_attenuation) against SORT's own results.

tests/golden/attenuation.npz holds the rgb attenuation SORT's Scene::GetAttenuation
returns (Accelerator::GetAttenuation in a loop, with Fbvh's query_shadow
traversal) on a 48-sphere field with transparent and opaque materials, the
materials assigned by sphere and per triangle. The GPU must return it bit for
bit, through the device entry point and the host-buffer one. With only opaque
materials the query must agree with the any-hit query. Bad material ids and a
missing material table are reported, not faulted on.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _acc(width, tri, mat):
    from sort_b200 import Obvh, Qbvh
    acc = (Qbvh if width == 4 else Obvh)()
    acc.Build(tri)
    acc.SetMaterials(mat)
    return acc


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("assign", ["by_sphere", "per_tri"])
def test_attenuation_matches_sort(width, assign):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    z = golden("attenuation")
    acc = _acc(width, z["triangles"], z[assign])
    rays = torch.from_numpy(np.ascontiguousarray(z["rays"])).cuda()
    att = acc.GetAttenuationTransparent(rays, z["transparent"], z["rgb"])
    torch.cuda.synchronize()
    assert same_bits(att.cpu().numpy(), z[f"att{width}_{assign}"])


def test_attenuation_host_form_matches_device_form():
    from sort_b200 import _lib
    z = golden("attenuation")
    acc = _acc(8, z["triangles"], z["per_tri"])
    rays = np.ascontiguousarray(z["rays"])
    n = rays.shape[1]
    table = acc.transparency_table(z["transparent"], z["rgb"])
    out = np.empty((3, n), np.float32)
    lib = _lib.load()
    for _ in range(2):
        _lib.check(lib.sg_trace_attenuation_host(acc._h, rays.ctypes.data, n, table.ctypes.data, table.size,
                                                 out.ctypes.data))
        assert same_bits(out, z["att8_per_tri"])


def test_all_opaque_equals_any_hit():
    from sort_b200 import Obvh, scenes
    tri = scenes.sphere_field(64, 3, seed=5)
    rays = torch.from_numpy(np.ascontiguousarray(scenes.random_rays(50_000, seed=6))).cuda()
    acc = Obvh()
    acc.Build(tri)
    acc.SetMaterials(np.zeros(tri.shape[0], np.int32))
    att = acc.GetAttenuationTransparent(rays, [0], [[0.5, 0.5, 0.5]])
    occ = acc.GetAttenuation(rays)
    torch.cuda.synchronize()
    blocked = occ.cpu().numpy().astype(bool)
    a = att.cpu().numpy()
    assert (a[:, blocked] == 0).all() and (a[:, ~blocked] == 1).all()
    assert 0.05 < blocked.mean() < 0.95


def test_fully_transparent_scene_passes_everything():
    """Transparency 1 everywhere: every ray crosses all its surfaces unattenuated."""
    from sort_b200 import Qbvh, scenes
    tri = scenes.sphere_field(16, 2, seed=7)
    rays = torch.from_numpy(np.ascontiguousarray(scenes.random_rays(20_000, seed=8))).cuda()
    acc = Qbvh()
    acc.Build(tri)
    acc.SetMaterials(np.zeros(tri.shape[0], np.int32))
    att = acc.GetAttenuationTransparent(rays, [1], [[1.0, 1.0, 1.0]])
    torch.cuda.synchronize()
    assert (att.cpu().numpy() == 1.0).all()


def test_attenuation_errors_are_reported():
    from sort_b200 import Obvh, _lib, scenes
    tri = scenes.sphere_field(8, 2, seed=9)
    rays = np.ascontiguousarray(scenes.random_rays(4096, seed=10))
    n = rays.shape[1]
    out = np.empty((3, n), np.float32)
    lib = _lib.load()
    acc = Obvh()
    acc.Build(tri)
    table = acc.transparency_table([1, 0], [[0.5, 0.5, 0.5], [0, 0, 0]])
    st = lib.sg_trace_attenuation_host(acc._h, rays.ctypes.data, n, table.ctypes.data, table.size, out.ctypes.data)
    assert st == 1  # SG_ERR_INVALID_ARGUMENT: no primitive materials set yet
    acc.SetMaterials(np.full(tri.shape[0], 5, np.int32))  # outside the 2-entry table
    st = lib.sg_trace_attenuation_host(acc._h, rays.ctypes.data, n, table.ctypes.data, table.size, out.ctypes.data)
    assert st == 1
    assert b"material" in lib.sg_last_error()
    acc.SetMaterials(np.zeros(tri.shape[0], np.int32))  # the scene keeps answering after the error
    _lib.check(lib.sg_trace_attenuation_host(acc._h, rays.ctypes.data, n, table.ctypes.data, table.size,
                                             out.ctypes.data))
    nz = out[out != 0]  # 0 (opaque hit) or 0.5 to the number of transparent crossings
    assert np.array_equal(np.exp2(np.round(np.log2(nz))), nz) and (nz <= 1).all()
