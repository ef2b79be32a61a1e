"""Multi-GPU work division for replicated scenes (one process per GPU).

Rays, paths and render requests are independent, so every GPU holds a full
replica of each scene's tree and takes a share of the work; no kernel reads
another GPU's memory and nothing on the data path needs a collective. This
module holds the host-side pieces: contiguous shares of a ray batch, tiles of
an image dealt round-robin, one frame rendered in bands of rows across the
ranks and gathered (bit-identical to a one-GPU render), a router that sends
each render request to the replica with the least outstanding work and a
server front that routes one request stream over one render server per GPU
with it, and the max-over-ranks reduction the timings use (torch.distributed,
NCCL on GPUs, gloo on CPU).

SORT's counterpart is its thread pool splitting one image into 64x64 tiles
(work/image_evaluation/image_evaluation.cpp:153-279); here the split is across
GPUs as well.
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous share of n items; shares differ by at most one."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need 0 <= rank < world and n >= 0")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def tiles(width: int, height: int, tile: int = 64) -> list[tuple[int, int, int, int]]:
    """The image's tiles (x0, y0, x1, y1) in row-major order."""
    if width <= 0 or height <= 0 or tile <= 0:
        raise ValueError("positive sizes required")
    return [(x, y, min(x + tile, width), min(y + tile, height))
            for y in range(0, height, tile) for x in range(0, width, tile)]


def rank_tiles(width: int, height: int, rank: int, world: int, tile: int = 64):
    """Tiles dealt round-robin, so every rank gets a spread of the image."""
    return tiles(width, height, tile)[rank::world]


class ReplicaRouter:
    """Sends each request to the replica with the least outstanding samples
    (ties: lowest index), and releases that load when the request completes."""

    def __init__(self, replicas: int):
        if replicas < 1:
            raise ValueError("at least one replica")
        self.load = [0] * replicas
        self.where = {}

    def route(self, request_id, samples: int) -> int:
        r = min(range(len(self.load)), key=lambda k: (self.load[k], k))
        self.load[r] += int(samples)
        self.where[request_id] = (r, int(samples))
        return r

    def done(self, request_id) -> int:
        r, samples = self.where.pop(request_id)
        self.load[r] -= samples
        return r


def _rank_world():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def gather_rows(band, height: int):
    """The whole image, on every rank, from each rank's band of rows: rank r
    holds rows shard_range(height, r, world) (possibly none). Bands are padded
    to the largest band for one all_gather (NCCL on GPU tensors, gloo on CPU)."""
    import torch
    import torch.distributed as dist
    rank, world = _rank_world()
    if world == 1:
        return band
    rows_max = -(-height // world)
    pad = torch.zeros((rows_max,) + tuple(band.shape[1:]), dtype=band.dtype, device=band.device)
    pad[:band.shape[0]] = band
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    return torch.cat([parts[r][:shard_range(height, r, world)[1] - shard_range(height, r, world)[0]]
                      for r in range(world)])


def render_sharded(pathtracer, camera, width: int, height: int, spp: int, max_recursive_depth: int = 5,
                   seed: int = 1):
    """One frame split across the ranks by rows (one process per GPU, each with
    its own replica of the scene): rank r renders its band with
    PathTracer.Render(rows=...), and the bands are gathered on every rank. The
    result is bit-identical to one GPU rendering the whole frame, because each
    pixel draws the random numbers of its place in the frame."""
    import torch
    rank, world = _rank_world()
    r0, r1 = shard_range(height, rank, world)
    if r1 > r0:
        band = pathtracer.Render(camera, width, height, spp, max_recursive_depth, seed, rows=(r0, r1))
    else:
        dev = pathtracer.device
        band = torch.empty((0, width, 3), dtype=torch.float32,
                           device=dev if isinstance(dev, torch.device) else torch.device("cuda", dev))
    return gather_rows(band, height)


def max_over_ranks(value: float, device=None) -> float:
    """The largest of every rank's value (the slowest rank's time); the value
    itself without an initialised process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ReplicatedServer:
    """Render servers on several GPUs of one node behind one request stream:
    each GPU runs its own sg_server (its own host loop, path pool and solo
    lanes) over its own replica of every scene, and each request goes to the
    replica with the least outstanding samples (ReplicaRouter). Tickets are
    the server's own; wait and cancel go to the replica that took the request.

    servers: one RenderServer-like object per GPU (add_scene, submit, wait,
    cancel, stats, close), already holding the same scenes in the same order.
    """

    def __init__(self, servers):
        if not servers:
            raise ValueError("at least one server")
        self.servers = list(servers)
        self.router = ReplicaRouter(len(self.servers))
        self._where = {}  # ticket -> (replica, the replica's ticket)
        self._next = 1

    def submit(self, scene: int, camera, width: int, height: int, spp: int, max_depth: int = 5, seed: int = 1,
               image=None) -> int:
        ticket = self._next
        self._next += 1
        r = self.router.route(ticket, int(width) * int(height) * int(spp))
        try:
            inner = self.servers[r].submit(scene, camera, width, height, spp, max_depth, seed=seed, image=image)
        except Exception:
            self.router.done(ticket)
            raise
        self._where[ticket] = (r, inner)
        return ticket

    def wait(self, ticket: int, timeout: float | None = None):
        r, inner = self._where[ticket]
        img, res = self.servers[r].wait(inner, timeout)
        del self._where[ticket]
        self.router.done(ticket)
        return img, dict(res, ticket=ticket, replica=r)

    def cancel(self, ticket: int) -> None:
        r, inner = self._where[ticket]
        self.servers[r].cancel(inner)

    def stats(self) -> dict:
        per = [s.stats() for s in self.servers]
        total = {k: sum(p[k] for p in per) for k in per[0]}
        total["replicas"] = per
        return total

    def close(self) -> None:
        for s in self.servers:
            s.close()
