"""8-bit child boxes (precision form): hits stay SORT's, except where SORT loses one.

The FP32-node traversal is bit-identical to SORT (test_gpu_trace.py), so it
stands in for SORT here. With 8-bit nodes every decoded child box contains the
FP32 box and the slab test uses SORT's monotonic formula, so the traversal
enters a superset of SORT's nodes. Allowed differences from SORT, per ray:
  * near-tie: both hit, |t_q8 - t_sort| <= 1e-6 * t_sort (visit order differs);
  * SORT lost a hit: the 8-bit traversal returns a nearer hit that SORT's own
    FP32 watertight test of that triangle confirms with the same t — a triangle
    SORT's FP32 box rounding culled or excluded. Required to be rare.
Everything else (a lost hit, a different t for the same triangle) fails.
"""
import numpy as np
import pytest

from conftest import same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

QUANT8 = 1


def trace(acc, rays):
    d = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    h = acc.GetIntersect(d)
    occ = acc.GetAttenuation(d)
    torch.cuda.synchronize()
    return h.prim.cpu().numpy(), h.t.cpu().numpy(), h.u.cpu().numpy(), h.v.cpu().numpy(), occ.cpu().numpy()


def check(port, tri, rays, width, max_lost_fraction=1e-4):
    from sort_b200 import Obvh, Qbvh
    cls = Qbvh if width == 4 else Obvh
    a = cls()
    a.Build(tri)
    b = cls(node_format=QUANT8)
    b.Build(tri)
    assert b.info()["node_format"] == QUANT8
    assert b.info()["device_bytes"] < a.info()["device_bytes"]
    pf, tf, uf, vf, of = trace(a, rays)
    pq, tq, uq, vq, oq = trace(b, rays)
    same = pf == pq
    assert same_bits(tf[same], tq[same]) and same_bits(uf[same], uq[same]) and same_bits(vf[same], vq[same])
    ties = lost = 0
    for i in np.nonzero(~same)[0]:
        if pf[i] >= 0 and pq[i] >= 0 and abs(float(tq[i]) - float(tf[i])) <= 1e-6 * float(tf[i]):
            ties += 1
            continue
        assert pq[i] >= 0 and (pf[i] < 0 or tq[i] < tf[i]), f"ray {i}: 8-bit nodes lost or worsened a hit"
        t = port.tri_t(tri, int(pq[i]), rays, int(i))
        assert t is not None and np.float32(t) == tq[i], f"ray {i}: hit not confirmed by SORT's triangle test"
        lost += 1
    assert lost <= max(2, max_lost_fraction * rays.shape[1]), lost
    # any-hit: a superset of SORT's occluded rays, each extra one a genuine hit
    assert not np.any(of & ~oq)
    for i in np.nonzero(oq & ~of)[0]:
        assert pq[i] >= 0 and rays[6, i] < tq[i] <= rays[7, i]
    return ties, lost


@pytest.mark.parametrize("width", [4, 8])
def test_quant8_raycast_82k(port, width):
    from sort_b200 import scenes
    tri = scenes.sphere_field(64, 3, seed=1)
    rays = np.concatenate([scenes.camera_rays(512, 512, seed=7), scenes.random_rays(100_000, seed=8)], axis=1)
    check(port, tri, rays, width)


def test_quant8_incoherent_1m(port):
    from sort_b200 import scenes
    tri = scenes.sphere_field(128, 4, seed=2)  # 327,682 triangles
    cam = scenes.camera_rays(512, 512, seed=9)
    from sort_b200 import Obvh
    a = Obvh()
    a.Build(tri)
    h = a.GetIntersect(torch.from_numpy(cam).cuda())
    diffuse, shadow = scenes.bounce_rays(tri, cam, h.prim.cpu().numpy(), h.t.cpu().numpy(), cam.shape[1], seed=10)
    check(port, tri, np.ascontiguousarray(np.concatenate([diffuse, shadow], axis=1)), 8)


def test_quant8_golden_edges(port):
    from conftest import golden
    z = golden("edges")
    check(port, z["triangles"], z["rays"], 8)
    check(port, z["triangles"], z["rays"], 4)
