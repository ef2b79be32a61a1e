"""SG_BUILDER_LBVH and SG_BUILDER_PLOC: the wide BVHs built on the GPU from
the Morton order (radix tree; parallel locally-ordered clustering).

Their trees are not SORT's, so the bar is the one for a different tree over the
same triangles: every ray's closest distance equals the one through SORT's
tree (the host builder's) bit for bit, the primitive is the same unless two
triangles are hit at exactly that distance, and the any-hit answer is the
same. Two exceptions come from the box arithmetic, not from a fault of either
tree. Near-ties: when two triangles are hit within rounding of each other, a
box entry distance that rounds above the first hit found culls the other, so
each tree may keep a different one. Rounding here is 1e-6 of the distance, or
a few float32 ulps of the vertices' offsets from the ray origin (the
watertight test works on those offsets, so its distance carries their
rounding; it dominates when the origin lies close to large triangles). And a
ray that
SORT's slab test (with its 1e-5 clamp of direction components,
simd/simd_ray_utils.h:61-64, and simd/simd_bbox.h:47-109) sends past a
triangle's own box by rounding reaches that triangle only through a larger
leaf box, so whether it is found depends on which triangles share its leaf;
such rays may differ, and the test checks that every difference is one.
Scenes cover ties and degenerate triangles (the golden edge scene), tiny and
empty scenes, leaf sizes 1 to 16, and both widths.
"""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


BUILDERS = ["lbvh", "ploc"]


def _code(builder):
    from sort_b200 import _lib
    return {"lbvh": _lib.SG_BUILDER_LBVH, "ploc": _lib.SG_BUILDER_PLOC}[builder]


def _pair(tri, width, builder="lbvh", **kw):
    from sort_b200 import Obvh, Qbvh, _lib
    cls = Qbvh if width == 4 else Obvh
    ref = cls(builder=_lib.SG_BUILDER_HOST, **kw)
    ref.Build(tri)
    lb = cls(builder=_code(builder), **kw)
    lb.Build(tri)
    return ref, lb


def _own_box_missed(tri, prim, rays, i):
    """SORT's slab test of ray i against triangle prim's own box (float32,
    multiply and add rounded separately, |d| < 1e-5 clamped): True if it fails."""
    f = np.float32
    v = np.asarray(tri[prim], f).reshape(3, 3)
    lo, hi = v.min(0), v.max(0)
    o = rays[0:3, i].astype(f)
    d = rays[3:6, i].astype(f)
    d = np.where(np.abs(d) < f(1e-5), np.where(d < 0, f(-1e-5), f(1e-5)), d).astype(f)
    rcp = (f(1) / d).astype(f)
    t1 = ((lo - o).astype(f) * rcp).astype(f)
    t2 = ((hi - o).astype(f) * rcp).astype(f)
    tmin = max(f(rays[6, i]), np.minimum(t1, t2).max())
    tmax = min(f(rays[7, i]), np.maximum(t1, t2).min())
    return not tmin <= tmax


def _t_slack(tri, prim, rays, i):
    """Rounding of the watertight distance from ray i to triangle prim: 8 float32
    ulps of the largest vertex offset from the origin, in units of the ray's
    largest direction component."""
    v = np.asarray(tri[prim], np.float64).reshape(3, 3)
    o = rays[0:3, i].astype(np.float64)
    d = rays[3:6, i].astype(np.float64)
    return 8.0 * 2.0 ** -24 * float(np.abs(v - o).max()) / float(np.abs(d).max())


def _same_hits(tri, ref, lb, rays, check_ties=True):
    from oracle.oracle import Port
    r = np.ascontiguousarray(rays)
    d = torch.from_numpy(r).cuda()
    ha, hb = ref.GetIntersect(d), lb.GetIntersect(d)
    pa, pb = ha.prim.cpu().numpy(), hb.prim.cpu().numpy()
    ta, tb = ha.t.cpu().numpy(), hb.t.cpu().numpy()
    moved = np.nonzero(ta.view(np.int32) != tb.view(np.int32))[0]
    for i in moved:  # a near-tie, or the nearer hit's own box is missed by the slab test
        near_tie = pa[i] >= 0 and pb[i] >= 0 and abs(float(ta[i]) - float(tb[i])) <= max(
            1e-6 * float(min(ta[i], tb[i])), _t_slack(tri, int(pa[i]), r, int(i)) + _t_slack(tri, int(pb[i]), r, int(i)))
        p = pa[i] if ta[i] < tb[i] else pb[i]
        assert near_tie or (p >= 0 and _own_box_missed(tri, int(p), r, int(i))), \
            f"ray {i}: {pa[i]}@{ta[i]} vs {pb[i]}@{tb[i]}"
    assert moved.size <= max(10, rays.shape[1] // 1000)
    same_t = np.ones(rays.shape[1], bool)
    same_t[moved] = False
    diff = np.nonzero((pa != pb) & same_t)[0]
    if check_ties and diff.size:
        port = Port()
        for i in diff[:50]:  # a tie: both triangles give the reported distance
            assert np.float32(port.tri_t(tri, int(pa[i]), r, int(i))) == ta[i]
            assert np.float32(port.tri_t(tri, int(pb[i]), r, int(i))) == ta[i]
    oa, ob = ref.GetAttenuation(d).cpu().numpy(), lb.GetAttenuation(d).cpu().numpy()
    assert np.array_equal(oa[same_t], ob[same_t])


@pytest.mark.parametrize("builder", BUILDERS)
@pytest.mark.parametrize("width", [4, 8])
def test_lbvh_sphere_fields(width, builder):
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import scenes
    for spheres, level, seed in ((64, 3, 1), (256, 4, 2)):
        tri = scenes.sphere_field(spheres, level, seed=seed)
        rays = np.concatenate([scenes.camera_rays(256, 256, seed=3), scenes.random_rays(50_000, seed=4)], axis=1)
        ref, lb = _pair(tri, width, builder)
        _same_hits(tri, ref, lb, rays)
        info = lb.info()
        assert info["triangles"] == tri.shape[0] and info["leaves"] > 0 and info["interior_nodes"] > 0
        assert info["bbox"] == ref.info()["bbox"]


@pytest.mark.parametrize("builder", BUILDERS)
@pytest.mark.parametrize("width", [4, 8])
@pytest.mark.parametrize("leaf", [1, 3, 8, 16])
def test_lbvh_edge_scene(width, leaf, builder):
    z = golden("edges")
    ref, lb = _pair(z["triangles"], width, builder, max_pri_in_leaf=leaf)
    _same_hits(z["triangles"], ref, lb, z["rays"])


@pytest.mark.parametrize("builder", BUILDERS)
def test_lbvh_random_soup_and_tiny_scenes(builder):
    from sort_b200 import scenes
    rng = np.random.default_rng(7)
    c = rng.uniform(-5, 5, (20000, 1, 3))
    tri = (c + rng.normal(0, 0.5, (20000, 3, 3))).astype(np.float32).reshape(-1, 9)
    tri[::5] = np.round(tri[::5])  # repeated coordinates: equal Morton codes
    rays = scenes.random_rays(20000, seed=8, box=8.0, axis_fraction=0.2)
    for width in (4, 8):
        ref, lb = _pair(tri, width, builder)
        _same_hits(tri, ref, lb, rays)
        for k in (1, 2, 9, 17):
            ref, lb = _pair(tri[:k], width, builder)
            _same_hits(tri[:k], ref, lb, rays[:, :2000])


def _leaf_prims(topo, width, max_leaf=8):
    """Primitive ids in leaf order from a pre-order topology (interior: child
    count then the children; leaf: 0, its count, its ids); checks the child
    counts and leaf sizes on the way."""
    out, pos = [], 0

    def walk():
        nonlocal pos
        c = int(topo[pos])
        pos += 1
        if c == 0:
            n = int(topo[pos])
            assert 0 < n <= max_leaf
            out.extend(int(x) for x in topo[pos + 1:pos + 1 + n])
            pos += 1 + n
            return 1
        assert 0 < c <= width
        return 1 + sum(walk() for _ in range(c))
    walk()
    assert pos == len(topo)
    return out


@pytest.mark.parametrize("builder", BUILDERS)
def test_lbvh_limits_are_reported(builder):
    """The topology export reads a device-built tree back from the device:
    every primitive in exactly one leaf, leaves of at most max_leaf, at most
    W children per node. 8-bit nodes are refused, an empty scene is invalid."""
    from sort_b200 import Obvh, _lib, scenes
    tri = scenes.sphere_field(8, 2, seed=9)
    acc = Obvh(builder=_code(builder))
    acc.Build(tri)
    topo = acc.topology()
    prims = _leaf_prims(topo, 8)
    assert sorted(prims) == list(range(tri.shape[0]))
    q8 = Obvh(builder=_code(builder), node_format=_lib.SG_NODES_QUANT8)
    with pytest.raises(_lib.SortGpuError) as ex:
        q8.Build(tri)
    assert ex.value.status == 4
    empty = Obvh(builder=_code(builder))
    empty.Build(np.zeros((0, 9), np.float32))
    assert not empty.GetIsValid()


@pytest.mark.parametrize("width", [4, 8])
def test_ploc_tree_is_tighter_than_lbvh(width):
    """The clustered tree's traversal does less work than the radix tree's on
    the same rays (SORT's counters: interior nodes box-tested and primitives
    tested per ray), and its build reports the clustering iterations."""
    from sort_b200 import scenes
    tri = scenes.sphere_field(256, 4, seed=2)
    rays = torch.from_numpy(np.ascontiguousarray(scenes.random_rays(100_000, seed=5))).cuda()
    work = {}
    for builder in BUILDERS:
        _, acc = _pair(tri, width, builder)
        nodes, prims = acc.TraceStats(rays, False)
        work[builder] = nodes * (width * 28) + prims * 36
        info = acc.info()
        assert info["build_rounds"] > 0 and info["build_launches"] > info["build_rounds"]
    assert work["ploc"] < work["lbvh"], work
