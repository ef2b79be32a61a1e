"""Hair lines on the host: SORT's Line set-up and tree, without a GPU.

The split rules see a line as its box (Line::GetBBox, shape/line.cpp:98-106,
after Line::SetTransform), so building SORT's tree over triangles and lines
gives SORT's topology only if every line box is SORT's to the bit; the
topology lists each leaf's triangles before its lines, as SORT's leaf tests its
triangle packs before its line packs. Pinned against the committed fixture
(tests/golden/hair.npz, from SORT's own build) and, where the reference library
is built, against SORT directly on more strand sets and leaf sizes.
"""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("width", [4, 8])
def test_hair_topology_matches_golden(width):
    from sort_b200 import build_topology_host
    z = golden("hair")
    topo, _ = build_topology_host(z["triangles"], width, lines=z["lines"])
    assert np.array_equal(topo, z[f"topology{width}"])


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("leaf", [1, 3, 8, 16])
def test_hair_topology_matches_sort(reference, width, leaf):
    from sort_b200 import build_topology_host, scenes
    tri = scenes.sphere_field(16, 2, seed=3)
    for seed, steps in ((4, 8), (5, 3)):
        lines = scenes.hair_strands(150, steps, seed=seed)
        tree = reference.build_hair(tri, lines, width, 16, leaf)
        topo, depth = build_topology_host(tri, width, 16, leaf, lines=lines)
        assert np.array_equal(topo, tree.topology()) and depth == tree.depth()


def test_hair_only_scene_matches_sort(reference):
    from sort_b200 import build_topology_host, scenes
    lines = scenes.hair_strands(300, 6, seed=6)
    empty = np.zeros((0, 9), np.float32)
    for width in (4, 8):
        tree = reference.build_hair(empty, lines, width)
        topo, _ = build_topology_host(empty, width, lines=lines)
        assert np.array_equal(topo, tree.topology())
