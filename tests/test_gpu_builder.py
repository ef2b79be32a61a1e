"""GPU builder (SG_BUILDER_GPU): the same tree as the host builder, which is
SORT's tree (tests/test_builder.py pins that against SORT's own build).

Compared: the pre-order topology (child counts, leaf membership and leaf
order), the recorded depth, and hits and distances of traces through both
trees, which also checks the stored child boxes. Scenes cover ties and
degenerate triangles (the golden edge scene), extreme build parameters and
sizes up to 1.3M triangles.
"""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def both(tri, width, **kw):
    from sort_b200 import Obvh, Qbvh, _lib
    cls = Qbvh if width == 4 else Obvh
    a = cls(builder=_lib.SG_BUILDER_HOST, **kw)
    a.Build(tri)
    b = cls(builder=_lib.SG_BUILDER_GPU, **kw)
    b.Build(tri)
    return a, b


def same_tree(a, b, rays):
    assert a.info()["depth"] == b.info()["depth"]
    assert a.info()["interior_nodes"] == b.info()["interior_nodes"] and a.info()["leaves"] == b.info()["leaves"]
    assert np.array_equal(a.topology(), b.topology())
    assert a.info()["bbox"] == b.info()["bbox"]
    d = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    ha, hb = a.GetIntersect(d), b.GetIntersect(d)
    assert torch.equal(ha.prim, hb.prim)
    assert same_bits(ha.t.cpu().numpy(), hb.t.cpu().numpy())
    assert torch.equal(a.GetAttenuation(d), b.GetAttenuation(d))
    na, pa = a.TraceStats(d)
    nb, pb = b.TraceStats(d)
    assert (na, pa) == (nb, pb)


@pytest.mark.parametrize("width", [4, 8])
def test_gpu_builder_sphere_fields(width):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import scenes
    for spheres, level, seed in ((64, 3, 1), (256, 4, 2)):
        tri = scenes.sphere_field(spheres, level, seed=seed)
        rays = np.concatenate([scenes.camera_rays(256, 256, seed=3), scenes.random_rays(50_000, seed=4)], axis=1)
        same_tree(*both(tri, width), rays)


@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("params", [{}, {"max_node_depth": 4, "max_pri_in_leaf": 1}, {"max_pri_in_leaf": 3}])
def test_gpu_builder_edge_scene(width, params):
    z = golden("edges")
    same_tree(*both(z["triangles"], width, **params), z["rays"])


def test_gpu_builder_random_soup_and_tiny_scenes():
    from sort_b200 import scenes
    rng = np.random.default_rng(7)
    c = rng.uniform(-5, 5, (20000, 1, 3))
    tri = (c + rng.normal(0, 0.5, (20000, 3, 3))).astype(np.float32).reshape(-1, 9)
    tri[::5] = np.round(tri[::5])  # repeated coordinates: equal centroids, zero-width bins
    rays = scenes.random_rays(20000, seed=8, box=8.0, axis_fraction=0.2)
    for width in (4, 8):
        same_tree(*both(tri, width), rays)
        for k in (1, 2, 9, 17):
            same_tree(*both(tri[:k], width), rays[:, :2000])


def test_gpu_builder_quantized_nodes_from_host_arrays():
    """8-bit nodes of a GPU-built tree come from its host arrays, as the host
    builder's do (the builder's device-written FP32 nodes are not used)."""
    from sort_b200 import _lib, scenes
    tri = scenes.sphere_field(64, 3, seed=5)
    rays = np.concatenate([scenes.camera_rays(128, 128, seed=6), scenes.random_rays(20_000, seed=7)], axis=1)
    for width in (4, 8):
        same_tree(*both(tri, width, node_format=_lib.SG_NODES_QUANT8), rays)
