"""Area-light shapes in the accelerator on the GPU, against SORT's answers.

tests/golden/shapes.npz holds what SORT's Qbvh / Obvh return on a scene of
triangles, hair lines and 26 area-light shapes (Quad and Disk, including a
quad on the ground plane and a disk on a square of triangles, where a ray
finds a triangle and a shape at the same t and SORT keeps the shape), in
three primitive orders. The GPU must return SORT's closest hits (prim, t, u, v:
a shape hit leaves u, v as the hit it replaced left them) and any-hit answers
bit for bit, through both builders of SORT's tree.
"""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ORDERS = ["natural", "shapes_first", "shuffled"]


def _scene(z, name):
    from sort_b200 import SHAPE_DTYPE, Scene
    shapes = np.ascontiguousarray(z["shapes"]).view(SHAPE_DTYPE).reshape(-1)
    order = None if name == "natural" else z[f"order_{name}"]
    return Scene(z["triangles"], z["lines"], shapes, order)


@pytest.mark.parametrize("name", ORDERS)
@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("builder", [0, 1])
def test_shapes_match_sort(name, width, builder):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import Obvh, Qbvh
    z = golden("shapes")
    acc = (Qbvh if width == 4 else Obvh)(builder=builder)
    acc.Build(_scene(z, name))
    key = f"{name}_{width}"
    assert np.array_equal(acc.topology(), z[f"topology_{key}"])
    d = torch.from_numpy(np.ascontiguousarray(z["rays"])).cuda()
    h = acc.GetIntersect(d)
    occ = acc.GetAttenuation(d)
    torch.cuda.synchronize()
    assert np.array_equal(h.prim.cpu().numpy(), z[f"prim_{key}"])
    assert same_bits(h.t.cpu().numpy(), z[f"t_{key}"])
    assert same_bits(h.u.cpu().numpy(), z[f"u_{key}"]) and same_bits(h.v.cpu().numpy(), z[f"v_{key}"])
    assert np.array_equal(occ.cpu().numpy(), z[f"occ_{key}"])


def test_shapes_host_forms_match():
    from sort_b200 import Obvh
    z = golden("shapes")
    acc = Obvh()
    acc.Build(_scene(z, "shuffled"))
    rays = np.ascontiguousarray(z["rays"])
    h = acc.GetIntersect(rays)
    assert np.array_equal(np.asarray(h.prim), z["prim_shuffled_8"]) and same_bits(np.asarray(h.t), z["t_shuffled_8"])
    assert np.array_equal(np.asarray(acc.GetAttenuation(rays)), z["occ_shuffled_8"])


def test_shapes_unsupported_queries_are_reported():
    from sort_b200 import Obvh, _lib
    z = golden("shapes")
    acc = Obvh()
    acc.Build(_scene(z, "natural"))
    d = torch.from_numpy(np.ascontiguousarray(z["rays"][:, :500])).cuda()
    with pytest.raises(_lib.SortGpuError) as ex:
        acc.TraceStats(d)
    assert ex.value.status == 4
    lb = Obvh(builder=_lib.SG_BUILDER_LBVH)
    with pytest.raises(_lib.SortGpuError) as ex:
        lb.Build(_scene(z, "natural"))
    assert ex.value.status == 4
