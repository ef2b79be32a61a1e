"""Area-light shapes in the accelerator, host side (no GPU): SORT's tree.

SORT puts each area light's Quad or Disk into the accelerator as a primitive
of the leaf's other_list (entity/light_entity.cpp:153-154,
accel/fast_bvh.hpp:244-247); the split rules see it as its box
(Quad::GetBBox / Disk::GetBBox). The host builder must give SORT's topology,
leaf by leaf, with each leaf listing its triangles, then its lines, then its
shapes, whatever order SORT's scene presents the primitives in
(tests/golden/shapes.npz was made by SORT's own Qbvh / Obvh).
"""
import numpy as np
import pytest

from conftest import golden

ORDERS = ["natural", "shapes_first", "shuffled"]


def _shapes(z):
    from sort_b200 import SHAPE_DTYPE
    return np.ascontiguousarray(z["shapes"]).view(SHAPE_DTYPE).reshape(-1)


def _order(z, name):
    return None if name == "natural" else z[f"order_{name}"]


@pytest.mark.parametrize("name", ORDERS)
@pytest.mark.parametrize("width", [4, 8])
def test_shapes_topology_matches_sort_golden(name, width):
    from sort_b200 import build_topology_host
    z = golden("shapes")
    topo, _ = build_topology_host(z["triangles"], width, lines=z["lines"], shapes=_shapes(z), order=_order(z, name))
    assert np.array_equal(topo, z[f"topology_{name}_{width}"])


def test_shapes_topology_matches_live_sort(reference):
    from sort_b200 import build_topology_host, scenes
    tri = scenes.sphere_field(24, 2, seed=71)
    shapes = scenes.random_area_shapes(40, seed=72, disk_fraction=0.5)
    n = tri.shape[0] + shapes.shape[0]
    order = np.random.default_rng(73).permutation(n).astype(np.int32)
    for width in (4, 8):
        for od in (None, order):
            ref = reference.build_shapes(tri, None, shapes, od, width).topology()
            ours, _ = build_topology_host(tri, width, shapes=shapes, order=od)
            assert np.array_equal(ours, ref)


def test_shapes_bad_input_is_rejected():
    from sort_b200 import _lib, build_topology_host, scenes
    tri = scenes.sphere_field(2, 1, seed=74)
    shapes = scenes.random_area_shapes(3, seed=75)
    n = tri.shape[0] + 3
    with pytest.raises(_lib.SortGpuError) as ex:  # not a permutation
        build_topology_host(tri, 8, shapes=shapes, order=np.zeros(n, np.int32))
    assert ex.value.status == 1
    bad = shapes.copy()
    bad["kind"][1] = 7
    lib = _lib.load()
    import ctypes
    from sort_b200 import Scene
    sc = Scene(tri, shapes=bad)
    o = _lib.BuildOpts()
    lib.sg_default_build_opts(ctypes.byref(o))
    h = ctypes.c_void_p()
    assert lib.sg_scene_create_shapes(ctypes.byref(sc._shapes_struct()), ctypes.byref(o), ctypes.byref(h)) == 1
