"""A SORT scene stream traced on the GPU (sg_stream_scene_create).

The scene of tests/golden/scene.sort, built from the stream (its Obvh, or a
Qbvh when asked), must answer as SORT answers after reading the same entity
section with its own readers (tests/golden/stream.npz): closest hit (prim, t,
hair included) and any hit, bit for bit, through the host builder and the GPU
builder of SORT's tree, with the area lights' shapes in the tree in entity
order. u, v of a hair hit are SORT's; for a triangle SORT reports the
interpolated texture coordinates of its mesh (0.5, 0.5 in this file) where
this library reports barycentric weights, and a shape hit keeps the u, v of
the hit it replaced (so those follow the triangle rule).
"""
import os

import numpy as np
import pytest

from conftest import ROOT, golden, renumber_topology, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
GOLDEN = os.path.join(ROOT, "tests", "golden", "scene.sort")


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("builder", [0, 1])
def test_stream_scene_matches_sort(width, builder):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200.stream import SortStream
    z = golden("stream")
    s = SortStream(GOLDEN)
    acc = s.accelerator(builder=builder, width=None if width == 8 else 4)
    assert acc.info()["width"] == width
    assert acc.info()["triangles"] == s.info["triangles"] + s.info["lines"] + s.info["area_lights"]
    d = torch.from_numpy(np.ascontiguousarray(z["rays"])).cuda()
    h = acc.GetIntersect(d)
    occ = acc.GetAttenuation(d)
    torch.cuda.synchronize()
    # Our primitive ids number triangles, segments, then shapes; SORT's harness
    # numbers primitives in its iteration order (s.order lists ours in it).
    sort_index = np.argsort(s.order)
    ours = h.prim.cpu().numpy()
    assert np.array_equal(np.where(ours >= 0, sort_index[np.maximum(ours, 0)], -1), z[f"prim{width}"])
    assert same_bits(h.t.cpu().numpy(), z[f"t{width}"])
    p = ours
    nt, nl = s.info["triangles"], s.info["lines"]
    hair = (p >= nt) & (p < nt + nl)
    assert (p >= nt + nl).sum() > 100  # rays that end on the area lights' shapes
    u, v = h.u.cpu().numpy(), h.v.cpu().numpy()
    assert same_bits(u[hair], z[f"u{width}"][hair]) and same_bits(v[hair], z[f"v{width}"][hair])
    tri = (p >= 0) & (p < nt)
    assert (np.abs(z[f"u{width}"][tri] - 0.5) < 1e-6).all() and ((u[tri] >= 0) & (v[tri] >= 0) & (u[tri] + v[tri] <= 1.0001)).all()
    assert np.array_equal(occ.cpu().numpy(), z[f"occ{width}"])
    if builder == 0:
        assert np.array_equal(renumber_topology(acc.topology(), sort_index), z[f"topology{width}"])
