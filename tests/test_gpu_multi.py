"""BSSRDF probe query (sg_trace_multi) against SORT's own results.

tests/golden/multi.npz holds what SORT's compiled Qbvh / Obvh return from
GetIntersect(ray, BSSRDFIntersections&, rc, matID) on a 48-sphere field: with
three materials (few hits per ray) and with one material (long rays collect
more than four hits, so SORT's overwrite-the-farthest rule and its maxt culling
decide what is kept). The GPU must return the same count and the same
(prim, t) in the same slots bit for bit; u, v by value (SORT passes them
through texture-coordinate interpolation, which maps -0 to +0).
"""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("materials", ["three", "one"])
def test_multi_matches_sort(width, materials):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import Obvh, Qbvh
    z = golden("multi")
    sfx = "" if materials == "three" else "_one"
    mat = z["mat_of_tri"] if materials == "three" else np.zeros_like(z["mat_of_tri"])
    ray_mat = z["ray_mat"] if materials == "three" else np.zeros_like(z["ray_mat"])
    acc = (Qbvh if width == 4 else Obvh)()
    acc.Build(z["triangles"])
    rays = torch.from_numpy(np.ascontiguousarray(z["rays"])).cuda()
    count, prim, t, u, v = acc.GetIntersectBSSRDF(rays, mat, ray_mat)
    torch.cuda.synchronize()
    assert np.array_equal(count.cpu().numpy(), z[f"count{width}{sfx}"])
    assert np.array_equal(prim.cpu().numpy(), z[f"prim{width}{sfx}"])
    assert same_bits(t.cpu().numpy(), z[f"t{width}{sfx}"])
    assert np.array_equal(u.cpu().numpy(), z[f"u{width}{sfx}"]) and np.array_equal(v.cpu().numpy(), z[f"v{width}{sfx}"])


def test_multi_kept_hits_are_hits_of_the_material():
    """Each kept hit is a genuine closest-style hit of its triangle (SORT's
    watertight test gives the same t), on a primitive of the ray's material."""
    from sort_b200 import Obvh, scenes
    from oracle.oracle import Port
    z = golden("multi")
    acc = Obvh()
    acc.Build(z["triangles"])
    rays = np.ascontiguousarray(z["rays"][:, :2000])
    count, prim, t, _, _ = acc.GetIntersectBSSRDF(torch.from_numpy(rays).cuda(), z["mat_of_tri"], z["ray_mat"][:2000])
    count, prim, t = count.cpu().numpy(), prim.cpu().numpy(), t.cpu().numpy()
    port = Port()
    for i in np.nonzero(count)[0][:300]:
        for k in range(count[i]):
            p = int(prim[i, k])
            assert z["mat_of_tri"][p] == z["ray_mat"][i]
            assert np.float32(port.tri_t(z["triangles"], p, rays, int(i))) == t[i, k]


def test_multi_host_form_matches_device_form():
    """sg_trace_multi_host (what the SORT adapter calls per ray) returns what the
    device form returns, with the scene's resident material table."""
    import ctypes
    from sort_b200 import Obvh, _lib
    z = golden("multi")
    acc = Obvh()
    acc.Build(z["triangles"])
    rays = np.ascontiguousarray(z["rays"])
    n = rays.shape[1]
    count_d, prim_d, t_d, u_d, v_d = acc.GetIntersectBSSRDF(torch.from_numpy(rays).cuda(), z["mat_of_tri"],
                                                            z["ray_mat"])
    lib = _lib.load()
    mats = np.ascontiguousarray(z["mat_of_tri"], np.int32)
    _lib.check(lib.sg_scene_set_materials(acc._h, mats.ctypes.data, mats.size))
    rm = np.ascontiguousarray(z["ray_mat"], np.int32)
    count = np.empty(n, np.int32)
    prim = np.empty((n, 4), np.int32)
    t, u, v = (np.empty((n, 4), np.float32) for _ in range(3))
    _lib.check(lib.sg_trace_multi_host(acc._h, rays.ctypes.data, n, rm.ctypes.data, count.ctypes.data,
                                       prim.ctypes.data, t.ctypes.data, u.ctypes.data, v.ctypes.data))
    assert np.array_equal(count, count_d.cpu().numpy()) and np.array_equal(prim, prim_d.cpu().numpy())
    assert same_bits(t, t_d.cpu().numpy()) and same_bits(u, u_d.cpu().numpy()) and same_bits(v, v_d.cpu().numpy())
    with pytest.raises(Exception):
        _lib.check(lib.sg_scene_set_materials(acc._h, mats.ctypes.data, mats.size - 1))
