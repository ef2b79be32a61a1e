"""The restated CPU oracle (oracle/port) against SORT's own outputs.

Pins: tests/golden/*.npz hold what SORT's compiled Qbvh/Obvh returned
(tests/golden/make_golden.py). When the reference library is built on this
machine, random scenes are also compared live.
"""
import numpy as np
import pytest

from conftest import golden, same_bits

CASES = ["spheres_1922", "edges", "edges_leaf1_depth4"]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("width", [4, 8])
def test_port_matches_golden(port, case, width):
    z = golden(case)
    tree = port.build(z["triangles"], width, int(z["max_depth"]), int(z["max_leaf"]))
    assert np.array_equal(tree.topology(), z[f"w{width}_topology"])
    assert tree.depth() == int(z[f"w{width}_depth"])
    assert same_bits(tree.bbox(), z[f"w{width}_bbox"])
    prim, t, u, v = tree.closest(z["rays"])
    assert np.array_equal(prim, z[f"w{width}_prim"])
    assert same_bits(t, z[f"w{width}_t"])
    # SORT reports u, v through texture-coordinate interpolation (simd_triangle.h:336),
    # which turns a barycentric -0 into +0: compare by value.
    assert np.array_equal(u, z[f"w{width}_u"]) and np.array_equal(v, z[f"w{width}_v"])
    assert np.array_equal(tree.any(z["rays"]), z[f"w{width}_occ"])


def test_port_ray_prepare_matches_golden(port):
    z = golden("ray_prepare")
    for d, loc, sc in zip(z["dirs"], z["local"], z["scale"]):
        lx = np.zeros(3, np.int32)
        s = np.zeros(3, np.float32)
        d = np.ascontiguousarray(d)
        port.L.orc_ray_prepare(d.ctypes.data, lx.ctypes.data, s.ctypes.data)
        assert np.array_equal(lx, loc)
        assert same_bits(s, sc)


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("width", [4, 8])
def test_port_matches_reference_live(port, reference, seed, width):
    rng = np.random.default_rng(seed)
    ntri = 5000
    c = rng.uniform(-5, 5, (ntri, 1, 3))
    tri = (c + rng.normal(0, 0.5, (ntri, 3, 3))).astype(np.float32)
    tri[::7] = np.round(tri[::7])
    from sort_b200 import scenes
    rays = scenes.random_rays(20000, seed=seed + 10, box=8.0, axis_fraction=0.2)
    a, b = port.build(tri, width), reference.build(tri, width)
    assert np.array_equal(a.topology(), b.topology())
    pa, ta, ua, va = a.closest(rays)
    pb, tb, ub, vb = b.closest(rays)
    assert np.array_equal(pa, pb) and same_bits(ta, tb)
    assert np.array_equal(ua, ub) and np.array_equal(va, vb)
    assert np.array_equal(a.any(rays), b.any(rays))


def test_port_empty_scene(port):
    tree = port.build(np.zeros((0, 9), np.float32), 8)
    from sort_b200 import scenes
    prim, t, _, _ = tree.closest(scenes.random_rays(10))
    assert (prim == -1).all() and (t == np.float32(3.4028234663852886e38)).all()


@pytest.mark.parametrize("width", [4, 8])
def test_reference_multi_reproduces_golden(reference, width):
    """The committed BSSRDF probe fixture is what SORT's code returns (pins it)."""
    z = golden("multi")
    tree = reference.build_materials(z["triangles"], z["mat_of_tri"], 3, width)
    count, prim, t, u, v = tree.multi(z["rays"], z["ray_mat"])
    assert np.array_equal(count, z[f"count{width}"]) and np.array_equal(prim, z[f"prim{width}"])
    assert same_bits(t, z[f"t{width}"]) and same_bits(u, z[f"u{width}"]) and same_bits(v, z[f"v{width}"])


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("assign", ["by_sphere", "per_tri"])
def test_reference_attenuation_reproduces_golden(reference, width, assign):
    """The committed transparent-shadow fixture is what SORT's code returns (pins it)."""
    z = golden("attenuation")
    tree = reference.build_transparent(z["triangles"], z[assign], z["transparent"], z["rgb"], width)
    assert same_bits(tree.attenuation(z["rays"]), z[f"att{width}_{assign}"])


@pytest.mark.parametrize("width", [4, 8])
def test_reference_hair_reproduces_golden(reference, width):
    """The committed hair fixture is what SORT's code returns (pins it)."""
    z = golden("hair")
    tree = reference.build_hair(z["triangles"], z["lines"], width)
    prim, t, u, v = tree.closest(z["rays"])
    assert np.array_equal(prim, z[f"prim{width}"]) and same_bits(t, z[f"t{width}"])
    assert same_bits(u, z[f"u{width}"]) and same_bits(v, z[f"v{width}"])
    assert np.array_equal(tree.any(z["rays"]), z[f"occ{width}"])
