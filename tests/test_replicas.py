"""Multi-GPU work division, exercised as two gloo ranks on the CPU: shares of a
ray batch and of an image's tiles cover the work exactly once, a frame
rendered in bands of rows comes back whole and in order on every rank (also
when a rank has no rows), the timing reduction takes the slowest rank, and the
request router balances load."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")

from sort_b200.replicas import (ReplicaRouter, gather_rows, max_over_ranks, rank_tiles, render_sharded,  # noqa: E402
                                shard_range, tiles)


class _RowImage:
    """Stands in for PathTracer: a pixel's value is its index in the frame plus the seed."""
    device = torch.device("cpu")

    def Render(self, camera, width, height, spp, max_recursive_depth=5, seed=1, rows=None):
        r0, r1 = rows
        idx = torch.arange(r0 * width, r1 * width, dtype=torch.float32).reshape(r1 - r0, width, 1)
        return idx.repeat(1, 1, 3) + seed


def _frame(width, height, seed):
    return torch.arange(width * height, dtype=torch.float32).reshape(height, width, 1).repeat(1, 1, 3) + seed


def test_shard_range_partitions():
    for n in (0, 1, 7, 4_194_304, 4_194_305):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_tiles_cover_image_once():
    w, h = 1920, 1080
    seen = set()
    for r in range(3):
        for t in rank_tiles(w, h, r, 3):
            assert t not in seen
            seen.add(t)
    assert seen == set(tiles(w, h))
    assert sum((x1 - x0) * (y1 - y0) for x0, y0, x1, y1 in seen) == w * h


def test_router_balances_and_releases():
    rt = ReplicaRouter(2)
    a = rt.route("a", 100)
    b = rt.route("b", 10)
    c = rt.route("c", 10)
    assert (a, b, c) == (0, 1, 1)
    assert rt.route("d", 5) == 1 and rt.load == [100, 25]
    rt.done("a")
    assert rt.route("e", 1) == 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, stop = shard_range(n, rank, world)
        spans = [None] * world
        dist.all_gather_object(spans, (start, stop))
        slowest = max_over_ranks(1.0 + rank)  # rank 1 is "slower"
        mine = rank_tiles(640, 360, rank, world)
        all_tiles = [None] * world
        dist.all_gather_object(all_tiles, mine)
        frames = [bool(torch.equal(render_sharded(_RowImage(), None, w, h, 1, 5, seed=3), _frame(w, h, 3)))
                  for w, h in ((7, 5), (4, 1), (3, 2), (640, 361))]
        r0, r1 = shard_range(6, rank, world)
        band = torch.arange(r0, r1, dtype=torch.int64).reshape(-1, 1)
        frames.append(bool(torch.equal(gather_rows(band, 6), torch.arange(6).reshape(-1, 1))))
        if rank == 0:
            out.put((spans, slowest, all_tiles, frames))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    n = 1_000_003
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    spans, slowest, all_tiles, frames = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert spans[0] == (0, 500_002) and spans[1] == (500_002, n)
    assert slowest == 2.0
    flat = [t for ts in all_tiles for t in ts]
    assert len(flat) == len(set(flat)) == len(tiles(640, 360))
    assert all(frames), frames


def test_one_rank_renders_the_whole_frame():
    assert torch.equal(render_sharded(_RowImage(), None, 9, 4, 1, seed=2), _frame(9, 4, 2))


class _FakeServer:
    """Stands in for RenderServer: remembers what it was given."""

    def __init__(self):
        self.submitted, self.cancelled, self.closed, self.next = [], [], False, 100

    def submit(self, scene, camera, width, height, spp, max_depth=5, seed=1, image=None):
        self.next += 1
        self.submitted.append((self.next, scene, width, height, spp, seed))
        return self.next

    def wait(self, ticket, timeout=None):
        return "image-%d" % ticket, {"ticket": ticket, "status": 0}

    def cancel(self, ticket):
        self.cancelled.append(ticket)

    def stats(self):
        return {"requests_done": len(self.submitted), "samples_done": 7}

    def close(self):
        self.closed = True


def test_replicated_server_routes_by_outstanding_samples():
    from sort_b200.replicas import ReplicatedServer
    a, b = _FakeServer(), _FakeServer()
    srv = ReplicatedServer([a, b])
    t1 = srv.submit(0, None, 100, 100, 16)  # 160k samples -> a
    t2 = srv.submit(1, None, 10, 10, 4)     # -> b
    t3 = srv.submit(0, None, 20, 20, 4, seed=9)  # b still has less -> b
    assert [x[1:] for x in a.submitted] == [(0, 100, 100, 16, 1)]
    assert [x[1:] for x in b.submitted] == [(1, 10, 10, 4, 1), (0, 20, 20, 4, 9)]
    img, res = srv.wait(t1)  # a's load released: the next request goes to a
    assert img == "image-101" and res["ticket"] == t1 and res["replica"] == 0
    t4 = srv.submit(2, None, 8, 8, 1)
    assert a.submitted[-1][1:4] == (2, 8, 8)
    srv.cancel(t3)
    assert b.cancelled == [b.submitted[1][0]]
    st = srv.stats()
    assert st["requests_done"] == 4 and st["samples_done"] == 14 and len(st["replicas"]) == 2
    for t in (t2, t3, t4):
        srv.wait(t)
    assert srv.router.load == [0, 0]
    srv.close()
    assert a.closed and b.closed
