"""Hair lines on the GPU (sg_scene_create_hair) against SORT's own answers.

tests/golden/hair.npz holds what SORT's Qbvh / Obvh return on 16 spheres and
400 hair strands (3,200 Line segments): closest hit (prim, t, u, v), many of
them on lines (intersectLine_SIMD, simd/simd_line.h:232-330), and the any-hit
answer. The GPU must return them bit for bit, through the host builder and the
GPU builder of SORT's tree; other queries on such a scene report
SG_ERR_UNSUPPORTED instead of answering without the lines.
"""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _scene(width, builder):
    from sort_b200 import Obvh, Qbvh, Scene
    z = golden("hair")
    acc = (Qbvh if width == 4 else Obvh)(builder=builder)
    acc.Build(Scene(z["triangles"], z["lines"]))
    return z, acc


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("builder", [0, 1])
def test_hair_matches_sort(width, builder):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    z, acc = _scene(width, builder)
    assert acc.info()["triangles"] == z["triangles"].shape[0] + z["lines"].shape[0]
    if builder == 0:
        assert np.array_equal(acc.topology(), z[f"topology{width}"])
    d = torch.from_numpy(np.ascontiguousarray(z["rays"])).cuda()
    h = acc.GetIntersect(d)
    occ = acc.GetAttenuation(d)
    torch.cuda.synchronize()
    assert np.array_equal(h.prim.cpu().numpy(), z[f"prim{width}"])
    assert same_bits(h.t.cpu().numpy(), z[f"t{width}"])
    assert same_bits(h.u.cpu().numpy(), z[f"u{width}"]) and same_bits(h.v.cpu().numpy(), z[f"v{width}"])
    assert np.array_equal(occ.cpu().numpy(), z[f"occ{width}"])


def test_hair_host_forms_match():
    z, acc = _scene(8, 0)
    h = acc.GetIntersect(np.ascontiguousarray(z["rays"]))  # host buffers: sg_trace_closest_host
    assert np.array_equal(np.asarray(h.prim), z["prim8"]) and same_bits(np.asarray(h.t), z["t8"])
    assert np.array_equal(np.asarray(acc.GetAttenuation(np.ascontiguousarray(z["rays"]))), z["occ8"])


def test_hair_unsupported_queries_are_reported():
    from sort_b200 import Obvh, Scene, _lib
    z, acc = _scene(8, 0)
    d = torch.from_numpy(np.ascontiguousarray(z["rays"][:, :1000])).cuda()
    with pytest.raises(_lib.SortGpuError) as ex:
        acc.TraceStats(d)
    assert ex.value.status == 4
    with pytest.raises(_lib.SortGpuError) as ex:
        acc.GetIntersectBSSRDF(d, np.zeros(acc.info()["triangles"], np.int32), np.zeros(1000, np.int32))
    assert ex.value.status == 4
    lb = Obvh(builder=_lib.SG_BUILDER_LBVH)
    with pytest.raises(_lib.SortGpuError) as ex:
        lb.Build(Scene(z["triangles"], z["lines"]))
    assert ex.value.status == 4
