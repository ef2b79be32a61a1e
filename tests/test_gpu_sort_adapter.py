"""SORT's own code on the GPU through the Gbvh adapter (sort_b200/integration/gbvh.h).

oracle/_ref/libsortref_gbvh.so is SORT's unmodified accelerator, scene,
integrator and BxDF code (the oracle harness) with every scene's accelerator
being Gbvh, the SORT-side adapter a maintainer adds, over this library. So
Accelerator::GetIntersect and GetAttenuation, Scene::GetIntersect /
GetAttenuation and PathTracing::Li run exactly as SORT runs them, one ray per
adapter call. Each query must answer as SORT's own Obvh / Qbvh answers the
same scene:

* closest hits and SurfaceInteraction u, v (SORT's interpolated texture
  coordinates) bit for bit on the golden edge cases, including rays whose
  tmax is exactly the hit distance (SORT's SIMD test keeps t == tmax, its
  scalar Triangle::GetIntersect would not, so the adapter fills the
  interaction from the GPU's t, u, v rather than re-running that test);
* any-hit through Accelerator::GetAttenuation;
* scenes with hair lines and area-light shapes, in SORT's primitive order;
* SORT's PathTracing::Li over the path-tracing scene (spheres with Lambert and
  GGX materials, the area light's Quad in the tree): the same image bits.
Skipped where the reference library was not built (SORT's sources absent).
"""
import os

import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def adapter():
    from oracle.oracle import REF_GBVH_LIB, Reference
    if not os.path.exists(REF_GBVH_LIB):
        pytest.skip("SORT reference library with the adapter (oracle/_ref) not built on this machine")
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    return Reference(adapter=True)


@pytest.mark.parametrize("case", ["edges", "spheres_1922", "edges_leaf1_depth4"])
@pytest.mark.parametrize("width", [4, 8])
def test_adapter_answers_as_sort(reference, adapter, case, width):
    z = golden(case)
    d, leaf = int(z["max_depth"]), int(z["max_leaf"])
    ref = reference.build(z["triangles"], width, d, leaf)
    ada = adapter.build(z["triangles"], width, d, leaf)
    rays = np.ascontiguousarray(z["rays"])
    rp, rt, ru, rv = ref.closest(rays)
    ap, at, au, av = ada.closest(rays)
    assert np.array_equal(ap, rp) and same_bits(at, rt)
    assert same_bits(au, ru) and same_bits(av, rv)
    assert np.array_equal(ada.any(rays), ref.any(rays))
    if case == "edges":  # the golden edge set has hits exactly at tmax
        assert ((rp >= 0) & (rt == rays[7])).sum() > 0


def test_adapter_shapes_and_lines(reference, adapter):
    from sort_b200 import SHAPE_DTYPE
    z = golden("shapes")
    shapes = np.ascontiguousarray(z["shapes"]).view(SHAPE_DTYPE).reshape(-1)
    rays = np.ascontiguousarray(z["rays"])
    first_shape = z["triangles"].shape[0] + z["lines"].shape[0]
    for order in (None, z["order_shuffled"]):
        ref = reference.build_shapes(z["triangles"], z["lines"], shapes, order, 8)
        ada = adapter.build_shapes(z["triangles"], z["lines"], shapes, order, 8)
        rp, rt, ru, rv = ref.closest(rays)
        ap, at, au, av = ada.closest(rays)
        assert np.array_equal(ap, rp) and same_bits(at, rt)
        # u, v of a shape hit are left over from the hit it replaced in SORT
        tri = (rp >= 0) & (rp < z["triangles"].shape[0])
        assert same_bits(au[tri], ru[tri]) and same_bits(av[tri], rv[tri])
        assert (rp >= first_shape).sum() > 1000
        assert np.array_equal(ada.any(rays), ref.any(rays))


def test_adapter_path_tracing_matches_sort():
    """SORT's PathTracing::Li (NEE with MIS, Lambert and GGX, Russian
    roulette) over the same scene and seeds: the image through the adapter is
    SORT's image, bit for bit."""
    from oracle.oracle import REF_GBVH_LIB, RefPathTracer, reference_available
    from sort_b200 import scenes
    if not (reference_available() and os.path.exists(REF_GBVH_LIB)):
        pytest.skip("SORT reference libraries (oracle/_ref) not built on this machine")
    tri, mat_of_tri, mats, light, _, _ = scenes.pt_scene(16, 2)
    sort_pt = RefPathTracer().build(tri, mat_of_tri, mats, light)
    ada_pt = RefPathTracer(adapter=True).build(tri, mat_of_tri, mats, light)
    a = sort_pt.render(scenes.CAMERA, 32, 32, 2, 5, seed=7)
    b = ada_pt.render(scenes.CAMERA, 32, 32, 2, 5, seed=7)
    assert a.mean() > 0.0
    assert np.array_equal(a.view(np.int32), b.view(np.int32))
