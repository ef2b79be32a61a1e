"""Render server (sg_server): every request's image is bit-identical to
sg_pt_render of the same request, rendered alone or in a mix of requests that
share the path pool and wavefront queues, and whether or not it started in a
solo phase (whole-request waves while the server is idle) and joined the pool
part-way; admission, cancellation and limits.

The pools here are small (a few thousand path slots, a pixel budget below the
mix's total) so that slots are reused many times, requests wait for admission
and several scenes share each queue.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def tracers():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sort_b200 import scenes
    from sort_b200.pathtracer import PathTracer
    out = []
    for spheres, level, seed in ((16, 2, 1), (32, 3, 2), (8, 3, 3)):
        _, _, mats, light, tri, mat = scenes.pt_scene(spheres, level, seed=seed)
        out.append(PathTracer(tri, mat, mats, light))
    return out


def requests():
    from sort_b200 import scenes
    cam2 = [4.0, 6.0, 28.0, 0.0, -2.0, 0.0, 0.0, 1.0, 0.0, 40.0]
    return [  # scene, camera, width, height, spp, depth, seed
        (0, scenes.CAMERA, 64, 48, 4, 5, 11), (1, scenes.CAMERA, 96, 64, 2, 5, 12), (2, cam2, 33, 17, 7, 4, 13),
        (1, cam2, 128, 72, 1, 5, 14), (0, cam2, 16, 16, 16, 3, 15), (2, scenes.CAMERA, 80, 60, 3, 5, 16),
        (0, scenes.CAMERA, 1, 1, 5, 5, 17), (1, scenes.CAMERA, 200, 10, 2, 6, 18)]


def reference(tracers, req):
    sc, cam, w, h, spp, depth, seed = req
    img = tracers[sc].Render(cam, w, h, spp, depth, seed=seed)
    torch.cuda.synchronize()
    return img.cpu().numpy()


def loop_error(srv):
    """The error that stopped the server's loop (a submit after it reports it)."""
    from sort_b200 import scenes
    try:
        srv.submit(0, scenes.CAMERA, 1, 1, 1)
    except Exception as ex:  # noqa: BLE001 - the message is the point
        return str(ex)
    return "loop still running"


def server(tracers, **kw):
    from sort_b200.server import RenderServer
    srv = RenderServer(**kw)
    ids = [srv.add_scene(t) for t in tracers]
    assert ids == list(range(len(tracers)))
    return srv


@pytest.mark.parametrize("per_claim", [1, 3, 64])
def test_each_request_matches_single_render_alone_and_mixed(tracers, per_claim):
    reqs = requests()
    refs = [reference(tracers, r) for r in reqs]
    srv = server(tracers, path_slots=3000, pixel_budget=20_000, max_requests=4, samples_per_claim=per_claim)
    for r, ref in zip(reqs, refs):  # alone
        img, res = srv.wait(srv.submit(*r[:2], *r[2:6], seed=r[6]))
        assert res["status"] == 0, loop_error(srv)
        assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    tickets = [srv.submit(*r[:2], *r[2:6], seed=r[6]) for r in reqs[::-1]]  # mixed, reverse order
    for t, ref in zip(tickets, refs[::-1]):
        img, res = srv.wait(t)
        assert res["status"] == 0 and res["done_ns"] >= res["admit_ns"] >= res["submit_ns"]
        assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    st = srv.stats()
    assert st["requests_done"] == 2 * len(reqs)
    assert st["samples_done"] == 2 * sum(w * h * spp for _, _, w, h, spp, _, _ in reqs)
    assert st["queued"] == 0 and st["admitted"] == 0
    srv.close()


def test_solo_phase_and_handoff_give_the_same_image(tracers):
    """Large requests render every sample as whole-frame waves in the solo
    lanes, which scale and complete them, while smaller requests arriving
    meanwhile go to the pool. Images equal sg_pt_render's in every case, and
    with the lanes turned off."""
    import time

    from sort_b200 import scenes
    big = (1, scenes.CAMERA, 400, 300, 48, 5, 21)
    small = [(0, scenes.CAMERA, 64, 48, 4, 5, 22), (2, scenes.CAMERA, 33, 17, 7, 4, 23),
             (1, scenes.CAMERA, 200, 10, 2, 6, 24)]
    refs = [reference(tracers, r) for r in [big] + small]
    for solo in (1000, -1):
        srv = server(tracers, path_slots=50_000, pixel_budget=400_000, max_requests=8, samples_per_claim=8,
                     solo_pixels=solo)
        img, res = srv.wait(srv.submit(*big[:2], *big[2:6], seed=big[6]))  # alone: 48 waves in a lane
        assert res["status"] == 0, loop_error(srv)
        assert np.array_equal(img.view(np.uint32), refs[0].view(np.uint32))
        waves = srv.stats()["solo_waves"]
        assert waves == (big[4] if solo > 0 else 0)
        t_big = srv.submit(*big[:2], *big[2:6], seed=big[6])
        time.sleep(0.02)  # arrivals during the big request's waves
        tickets = [srv.submit(*r[:2], *r[2:6], seed=r[6]) for r in small]
        for t, ref in zip([t_big] + tickets, refs):
            img, res = srv.wait(t)
            assert res["status"] == 0 and np.array_equal(img.view(np.uint32), ref.view(np.uint32))
        lanes_take = [r for r in [big] + small if solo > 0 and r[2] * r[3] >= solo and r[4] >= 2]
        assert srv.stats()["solo_waves"] - waves == sum(r[4] for r in lanes_take)
        srv.close()


def test_cancel_leaves_others_unchanged(tracers):
    from sort_b200 import _lib, scenes
    reqs = requests()[:4]
    refs = [reference(tracers, r) for r in reqs]
    srv = server(tracers, path_slots=2048, pixel_budget=40_000, max_requests=8)
    big = srv.submit(1, scenes.CAMERA, 160, 120, 64, 5, seed=99)
    tickets = [srv.submit(*r[:2], *r[2:6], seed=r[6]) for r in reqs]
    queued = srv.submit(2, scenes.CAMERA, 150, 150, 8, 5, seed=98)  # waits for the pixel budget
    srv.cancel(big)
    srv.cancel(queued)
    for t, ref in zip(tickets, refs):
        img, res = srv.wait(t)
        assert res["status"] == 0 and np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    for t in (big, queued):
        img, res = srv.wait(t)
        assert img is None and res["status"] == _lib.SG_ERR_CANCELLED
    srv.close()


def test_limits_and_bad_requests(tracers):
    from sort_b200 import SortGpuError, scenes
    from sort_b200.pathtracer import PathTracer
    srv = server(tracers[:1], path_slots=1024, pixel_budget=10_000, max_requests=2)
    with pytest.raises(SortGpuError, match="LIMIT"):
        srv.submit(0, scenes.CAMERA, 200, 100, 1)
    with pytest.raises(SortGpuError, match="INVALID_ARGUMENT"):
        srv.submit(3, scenes.CAMERA, 10, 10, 1)
    with pytest.raises(SortGpuError, match="INVALID_ARGUMENT"):
        srv.submit(0, scenes.CAMERA, 10, 10, 0)
    _, _, mats, light, tri, mat = scenes.pt_scene(4, 1)
    q4 = PathTracer(tri, mat, mats, light, width=4)
    with pytest.raises(SortGpuError, match="UNSUPPORTED"):
        srv.add_scene(q4)
    # the server still serves after the refusals
    img, res = srv.wait(srv.submit(0, scenes.CAMERA, 20, 10, 2, seed=4))
    assert res["status"] == 0 and np.array_equal(img, reference(tracers, (0, scenes.CAMERA, 20, 10, 2, 5, 4)))
    srv.close()


def test_quantized_nodes_server(tracers):
    from sort_b200 import _lib, scenes
    from sort_b200.pathtracer import PathTracer
    _, _, mats, light, tri, mat = scenes.pt_scene(16, 3, seed=7)
    pt = PathTracer(tri, mat, mats, light, node_format=_lib.SG_NODES_QUANT8)
    srv = server([pt], path_slots=4096, pixel_budget=50_000)
    req = (0, scenes.CAMERA, 96, 54, 4, 5, 21)
    img, res = srv.wait(srv.submit(*req[:2], *req[2:6], seed=req[6]))
    assert res["status"] == 0
    assert np.array_equal(img.view(np.uint32), reference([pt], req).view(np.uint32))
    srv.close()


def test_replicated_server_front(tracers):
    """ReplicatedServer over one server per GPU (the scenes here live on GPU 0,
    so one replica): the same images as sg_pt_render, tickets and results of
    its own."""
    from sort_b200.replicas import ReplicatedServer
    front = ReplicatedServer([server(tracers, device=0, path_slots=4096, pixel_budget=40_000, max_requests=8)])
    reqs = requests()[:5]
    refs = [reference(tracers, r) for r in reqs]
    tickets = [front.submit(*r[:2], *r[2:6], seed=r[6]) for r in reqs]
    for t, ref in zip(tickets, refs):
        img, res = front.wait(t)
        assert res["status"] == 0 and res["ticket"] == t and res["replica"] == 0
        assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    assert front.stats()["requests_done"] == len(reqs)
    front.close()
