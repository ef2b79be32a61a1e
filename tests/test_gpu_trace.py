"""GPU parity of the closest-hit / any-hit kernels against SORT's results.

Bar: primitive ids and hit distances bit-identical to SORT's (FP32 nodes use
SORT's topology, visit order and rounding); u, v equal by value (SORT's own u, v
pass through texture-coordinate interpolation, which maps -0 to +0); any-hit
flags identical. Checked against the golden fixtures SORT produced, against the
restated oracle at the 81,922-triangle ray-cast size and on random rays, and
on the host-buffer forms. The 21M-triangle benchmark size is covered by
test_gpu_incoherent_21m.py.
"""
import numpy as np
import pytest

from conftest import golden, same_bits

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def cuda_device():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sort_b200 import _lib
    _lib.load()  # fails loudly if the extension is missing
    return torch.device("cuda:0")


def accel(width, **kw):
    from sort_b200 import Obvh, Qbvh
    return (Qbvh if width == 4 else Obvh)(**kw)


def run_device(acc, rays):
    d = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    h = acc.GetIntersect(d)
    occ = acc.GetAttenuation(d)
    torch.cuda.synchronize()
    return h.prim.cpu().numpy(), h.t.cpu().numpy(), h.u.cpu().numpy(), h.v.cpu().numpy(), occ.cpu().numpy()


@pytest.mark.parametrize("case", ["spheres_1922", "edges", "edges_leaf1_depth4"])
@pytest.mark.parametrize("width", [4, 8])
def test_gpu_matches_sort_golden(case, width):
    z = golden(case)
    acc = accel(width, max_node_depth=int(z["max_depth"]), max_pri_in_leaf=int(z["max_leaf"]))
    acc.Build(z["triangles"])
    assert np.array_equal(acc.topology(), z[f"w{width}_topology"])
    assert same_bits(np.array(acc.GetBBox(), np.float32), z[f"w{width}_bbox"])
    prim, t, u, v, occ = run_device(acc, z["rays"])
    assert np.array_equal(prim, z[f"w{width}_prim"])
    assert same_bits(t, z[f"w{width}_t"])
    assert np.array_equal(u, z[f"w{width}_u"]) and np.array_equal(v, z[f"w{width}_v"])
    assert np.array_equal(occ, z[f"w{width}_occ"])


@pytest.mark.parametrize("width", [4, 8])
def test_gpu_raycast_82k_matches_oracle(port, width):
    from sort_b200 import scenes
    tri = scenes.sphere_field(64, 3, seed=1)
    rays = scenes.camera_rays(1024, 1024, seed=7)
    acc = accel(width)
    acc.Build(tri)
    prim, t, u, v, occ = run_device(acc, rays)
    ref = port.build(tri, width)
    rp, rt, ru, rv = ref.closest(rays)
    assert np.array_equal(prim, rp)
    assert same_bits(t, rt) and same_bits(u, ru) and same_bits(v, rv)
    assert np.array_equal(occ, ref.any(rays))
    assert (prim >= 0).mean() > 0.2


@pytest.mark.parametrize("width", [4, 8])
def test_gpu_random_rays_matches_oracle(port, width):
    from sort_b200 import scenes
    tri = scenes.sphere_field(32, 3, seed=2)
    rays = scenes.random_rays(200_000, seed=8, axis_fraction=0.3)
    acc = accel(width)
    acc.Build(tri)
    prim, t, u, v, occ = run_device(acc, rays)
    ref = port.build(tri, width)
    rp, rt, ru, rv = ref.closest(rays)
    assert np.array_equal(prim, rp) and same_bits(t, rt)
    assert same_bits(u, ru) and same_bits(v, rv)
    assert np.array_equal(occ, ref.any(rays))


def test_gpu_host_entry_points_match_device(port):
    from sort_b200 import scenes
    tri = scenes.sphere_field(8, 3, seed=5)
    rays = scenes.random_rays(50_000, seed=6)
    acc = accel(8)
    acc.Build(tri)
    prim, t, u, v, occ = run_device(acc, rays)
    h = acc.GetIntersect(rays)           # numpy -> sg_trace_closest_host
    occ_h = acc.GetAttenuation(rays)     # numpy -> sg_trace_any_host
    assert np.array_equal(h.prim, prim) and same_bits(h.t, t)
    assert same_bits(h.u, u) and same_bits(h.v, v)
    assert np.array_equal(occ_h, occ)


@pytest.mark.parametrize("n", [1_048_576, 3_000_001])
def test_gpu_host_entry_points_pipelined_chunks(n):
    """Host-buffer calls large enough to be split into pipelined chunks (ragged
    last chunk included) return exactly the device-buffer results; u/v may be
    omitted."""
    from sort_b200 import _lib, scenes
    import ctypes
    tri = scenes.sphere_field(32, 3, seed=15)
    rays = np.ascontiguousarray(scenes.random_rays(n, seed=16))
    acc = accel(8)
    acc.Build(tri)
    prim, t, u, v, occ = run_device(acc, rays)
    h = acc.GetIntersect(rays)
    assert np.array_equal(h.prim, prim) and same_bits(h.t, t) and same_bits(h.u, u) and same_bits(h.v, v)
    assert np.array_equal(acc.GetAttenuation(rays), occ)
    p2, t2 = np.empty(n, np.int32), np.empty(n, np.float32)
    _lib.check(_lib.load().sg_trace_closest_host(acc._h, rays.ctypes.data, n, p2.ctypes.data, t2.ctypes.data,
                                                 None, None))
    assert np.array_equal(p2, prim) and same_bits(t2, t)


@pytest.mark.parametrize("n", [1, 31, 127, 128, 129, 1000, 4097])
def test_gpu_ragged_batches(n):
    from sort_b200 import scenes
    tri = scenes.sphere_field(8, 2, seed=9)
    rays = scenes.random_rays(5000, seed=10)
    acc = accel(4)
    acc.Build(tri)
    full = run_device(acc, rays)
    part = run_device(acc, rays[:, :n])
    for a, b in zip(full, part):
        assert np.array_equal(a[:n].view(np.uint8), b.view(np.uint8))


def test_gpu_empty_and_tiny_scenes(port):
    from sort_b200 import scenes
    rays = scenes.random_rays(1000, seed=12)
    acc = accel(8)
    acc.Build(np.zeros((0, 9), np.float32))
    assert not acc.GetIsValid()
    prim, t, _, _, occ = run_device(acc, rays)
    assert (prim == -1).all() and (t == np.float32(3.4028234663852886e38)).all() and (occ == 0).all()
    tri = np.array([[-1, -1, 0, 1, -1, 0, 0, 1, 0]], np.float32)
    acc.Build(tri)
    r = np.array([[0.1], [0.1], [5], [0], [0], [-1], [0], [3.4e38]], np.float32)
    prim, t, u, v, occ = run_device(acc, r)
    rp, rt, ru, rv = port.build(tri, 8).closest(r)
    assert prim[0] == 0 == rp[0] and same_bits(t, rt) and occ[0] == 1


def test_gpu_zero_rays_and_bad_input():
    from sort_b200 import SortGpuError
    acc = accel(8)
    acc.Build(np.random.default_rng(0).normal(size=(100, 9)).astype(np.float32))
    h = acc.GetIntersect(torch.zeros((8, 0), dtype=torch.float32, device="cuda"))
    assert h.prim.numel() == 0
    with pytest.raises(ValueError):
        acc.GetIntersect(torch.zeros((7, 10), dtype=torch.float32, device="cuda"))
    with pytest.raises(SortGpuError):
        accel(8, max_pri_in_leaf=0).Build(np.zeros((4, 9), np.float32))


def test_gpu_deep_tree_stack_bound(port):
    """max_depth 28 / leaf 16 (the exporter's UI defaults) needs the deeper stack."""
    from sort_b200 import scenes
    tri = scenes.sphere_field(16, 3, seed=13)
    rays = scenes.random_rays(20_000, seed=14)
    for width in (4, 8):
        acc = accel(width, max_node_depth=28, max_pri_in_leaf=2)
        acc.Build(tri)
        prim, t, _, _, occ = run_device(acc, rays)
        ref = port.build(tri, width, 28, 2)
        rp, rt, _, _ = ref.closest(rays)
        assert np.array_equal(prim, rp) and same_bits(t, rt)


@pytest.mark.parametrize("width", [4, 8])
def test_gpu_trace_stats_match_oracle_counters(port, width):
    """Node / primitive test counts of the GPU traversal equal the oracle's
    restatement of SORT's traversal (the counts behind the algorithmic-bytes figure)."""
    from sort_b200 import scenes
    tri = scenes.sphere_field(64, 3, seed=1)
    rays = scenes.camera_rays(256, 256, seed=3)
    acc = accel(width)
    acc.Build(tri)
    d = torch.from_numpy(rays).cuda()
    ref = port.build(tri, width)
    for any_hit in (False, True):
        assert acc.TraceStats(d, any_hit) == port.count(ref, rays, any_hit)


@pytest.mark.parametrize("width", [4, 8])
def test_gpu_schedules_give_identical_results(port, width):
    """The launch schedule (thread per ray, persistent warps with any refill
    threshold, while-while, speculative, rays sorted by a coherence key) never
    changes a result; the sorted schedule twice in a row (its scratch reused)."""
    from sort_b200 import scenes
    tri = scenes.sphere_field(32, 3, seed=15)
    rays = np.concatenate([scenes.camera_rays(200, 200, seed=16), scenes.random_rays(60_000, seed=17)], axis=1)
    acc = accel(width)
    acc.Build(tri)
    ref = port.build(tri, width)
    rp, rt, ru, rv = ref.closest(rays)
    ro = ref.any(rays)
    for schedule, refill in ((0, 1), (1, 1), (1, 8), (1, 16), (1, 32), (2, 8), (3, 8), (4, 8), (4, 8), (5, 8)):
        acc.SetTuning(schedule, refill)
        assert acc.GetTuning() == {"schedule": schedule, "refill_threshold": refill}
        prim, t, u, v, occ = run_device(acc, rays)
        assert np.array_equal(prim, rp) and same_bits(t, rt) and same_bits(u, ru) and same_bits(v, rv)
        assert np.array_equal(occ, ro)


@pytest.mark.parametrize("width", [4, 8])
def test_gpu_non_finite_rays_match_sort(port, width):
    """Rays with a NaN or infinite origin, direction, tmin or tmax component give
    SORT's answer (a miss, except an infinite tmax, which is an ordinary ray)
    under every schedule. Such rays can reach empty child slots, which the
    step-driven kernels pass over instead of testing each child for emptiness."""
    from sort_b200 import scenes
    tri = scenes.sphere_field(32, 3, seed=15)
    rng = np.random.default_rng(19)
    rays = scenes.random_rays(70_000, seed=18).copy()  # >= 2^16: the sorted schedule sorts
    vals = np.array([np.nan, np.inf, -np.inf], np.float32)
    k = 0
    for comp in range(8):
        for v in vals:
            rays[comp, k:k + 16] = v
            k += 16
    for j in range(k, 1024):  # several bad components at once
        comps = rng.choice(8, size=rng.integers(2, 5), replace=False)
        rays[comps, j] = rng.choice(vals, size=comps.size)
    acc = accel(width)
    acc.Build(tri)
    ref = port.build(tri, width)
    rp, rt, ru, rv = ref.closest(rays)
    ro = ref.any(rays)
    for schedule, refill in ((0, 1), (1, 8), (2, 8), (3, 8), (4, 8), (5, 8)):
        acc.SetTuning(schedule, refill)
        prim, t, u, v, occ = run_device(acc, rays)
        assert np.array_equal(prim, rp) and same_bits(t, rt)
        assert np.array_equal(occ, ro)
