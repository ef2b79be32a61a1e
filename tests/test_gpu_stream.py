"""A SORT scene stream traced on the GPU (sg_stream_scene_create).

The scene of tests/golden/scene.sort, built from the stream (its Obvh, or a
Qbvh when asked), must answer as SORT answers after reading the same entity
section with its own readers (tests/golden/stream.npz): closest hit (prim, t,
hair included) and any hit, bit for bit, through the host builder and the GPU
builder of SORT's tree. u, v of a hair hit are SORT's; for a triangle SORT
reports the interpolated texture coordinates of its mesh (0.5, 0.5 in this
file) where this library reports barycentric weights.
"""
import os

import numpy as np
import pytest

from conftest import ROOT, golden, same_bits

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
    assert acc.info()["triangles"] == s.info["triangles"] + s.info["lines"]
    d = torch.from_numpy(np.ascontiguousarray(z["rays"])).cuda()
    h = acc.GetIntersect(d)
    occ = acc.GetAttenuation(d)
    torch.cuda.synchronize()
    assert np.array_equal(h.prim.cpu().numpy(), z[f"prim{width}"])
    assert same_bits(h.t.cpu().numpy(), z[f"t{width}"])
    hair = z[f"prim{width}"] >= s.info["triangles"]
    u, v = h.u.cpu().numpy(), h.v.cpu().numpy()
    assert same_bits(u[hair], z[f"u{width}"][hair]) and same_bits(v[hair], z[f"v{width}"][hair])
    tri = (z[f"prim{width}"] >= 0) & ~hair
    assert (np.abs(z[f"u{width}"][tri] - 0.5) < 1e-6).all() and ((u[tri] >= 0) & (v[tri] >= 0) & (u[tri] + v[tri] <= 1.0001)).all()
    assert np.array_equal(occ.cpu().numpy(), z[f"occ{width}"])
    if builder == 0:
        assert np.array_equal(acc.topology(), z[f"topology{width}"])
