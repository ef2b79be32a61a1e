"""The product's host builder (libsortgpu, no GPU needed) builds SORT's tree.

Fbvh::Build (accel/fast_bvh.hpp:109-270) decides leaf membership, leaf order and
child order; the product must reproduce it exactly for hit IDs to match SORT at
exact-distance ties. Compared against SORT's own tree (golden fixtures and, when
built, the reference library) and against the restated oracle.
"""
import numpy as np
import pytest

from conftest import golden
from sort_b200 import build_topology_host, scenes


@pytest.mark.parametrize("case", ["spheres_1922", "edges", "edges_leaf1_depth4"])
@pytest.mark.parametrize("width", [4, 8])
def test_builder_matches_sort_golden(case, width):
    z = golden(case)
    topo, depth = build_topology_host(z["triangles"], width, int(z["max_depth"]), int(z["max_leaf"]))
    assert np.array_equal(topo, z[f"w{width}_topology"])
    assert depth == int(z[f"w{width}_depth"])


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("threads", [1, 8])
def test_builder_matches_oracle_spheres(port, width, threads):
    tri = scenes.sphere_field(64, 3, seed=1)  # the 81,922-triangle ray-cast scene
    topo, depth = build_topology_host(tri, width, threads=threads)
    ref = port.build(tri, width)
    assert np.array_equal(topo, ref.topology())
    assert depth == ref.depth()


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("max_depth,max_leaf", [(16, 8), (28, 16), (3, 2), (1, 8), (16, 1)])
def test_builder_params(port, width, max_depth, max_leaf):
    rng = np.random.default_rng(max_depth * 100 + max_leaf)
    n = 3000
    tri = (rng.uniform(-5, 5, (n, 1, 3)) + rng.normal(0, 0.3, (n, 3, 3))).astype(np.float32)
    tri[::5] = tri[0]  # many coincident centroids
    topo, depth = build_topology_host(tri, width, max_depth, max_leaf)
    ref = port.build(tri, width, max_depth, max_leaf)
    assert np.array_equal(topo, ref.topology())
    assert depth == ref.depth()


@pytest.mark.parametrize("ntri", [0, 1, 2, 8, 9])
def test_builder_small(port, ntri):
    rng = np.random.default_rng(ntri)
    tri = rng.normal(size=(ntri, 9)).astype(np.float32)
    topo, _ = build_topology_host(tri, 8)
    assert np.array_equal(topo, port.build(tri, 8).topology())


def test_builder_live_reference(reference):
    tri = scenes.sphere_field(16, 3, seed=4)
    for width in (4, 8):
        topo, depth = build_topology_host(tri, width)
        ref = reference.build(tri, width)
        assert np.array_equal(topo, ref.topology())
        assert depth == ref.depth()


def test_builder_rejects_bad_width():
    from sort_b200 import SortGpuError
    with pytest.raises(SortGpuError):
        build_topology_host(np.zeros((1, 9), np.float32), 5)
