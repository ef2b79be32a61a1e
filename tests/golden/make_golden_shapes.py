"""Generate tests/golden/shapes.npz: SORT's answers on scenes with area-light
shapes in the accelerator (oracle/_ref).

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden_shapes.py

16 level-2 icospheres plus a ground quad (triangles), 60 hair strands of 6
segments (SORT's Line shapes), 24 area-light shapes (SORT's Quad and Disk with
random rotations, entity/light_entity.cpp:112-154) and two shapes placed on
triangles' planes: a quad lying on the ground at y = -11 and a disk on a
ground-level square of two triangles, so that a ray can find a triangle and a
shape at the same distance (Quad::GetIntersect keeps a hit when t <= the
nearest t so far, shape/quad.cpp:72-74). Rays: aimed at random points of the
shapes (most hit one), aimed at the coplanar pair from above, random rays and
camera rays. Three primitive orders as SORT's scene would present them: the
natural one (triangles, lines, shapes), shapes first, and a shuffled one.
Stored per order and width (QBVH 4, OBVH 8): SORT's topology, the closest hit
(prim, t, u, v) and the any-hit answer.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from sort_b200 import area_shapes, scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def coplanar_shapes():
    """A quad on the ground plane (y = -11) and a disk on a small square at y = -5."""
    q_m = [1.0, 0.0, 0.0, 3.0, 0.0, 1.0, 0.0, -11.0, 0.0, 0.0, 1.0, -2.0, 0.0, 0.0, 0.0, 1.0]
    q_i = [1.0, 0.0, 0.0, -3.0, 0.0, 1.0, 0.0, 11.0, 0.0, 0.0, 1.0, 2.0, 0.0, 0.0, 0.0, 1.0]
    d_m = [1.0, 0.0, 0.0, -6.0, 0.0, 1.0, 0.0, -5.0, 0.0, 0.0, 1.0, 7.0, 0.0, 0.0, 0.0, 1.0]
    d_i = [1.0, 0.0, 0.0, 6.0, 0.0, 1.0, 0.0, 5.0, 0.0, 0.0, 1.0, -7.0, 0.0, 0.0, 0.0, 1.0]
    return area_shapes([0, 1], [[4.0, 3.0], [1.5, 0.0]], [q_m, d_m], [q_i, d_i])


def square_at(y, cx, cz, h):
    a, b, c, d = (cx - h, y, cz - h), (cx + h, y, cz - h), (cx + h, y, cz + h), (cx - h, y, cz + h)
    return np.array([[*a, *c, *b], [*a, *d, *c]], np.float32)


def aimed_rays(points, rng, spread=8.0, jitter=0.0):
    m = points.shape[0]
    tgt = points + rng.normal(scale=jitter, size=(m, 3))
    o = tgt + rng.normal(size=(m, 3)) * spread
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o.T, d.T, np.zeros((1, m)), np.full((1, m), 3.4e38)]).astype(np.float32)


def main():
    tri = np.ascontiguousarray(np.concatenate([scenes.sphere_field(16, 2, seed=61), square_at(-5.0, -6.0, 7.0, 2.0)]))
    lines = scenes.hair_strands(60, 6, seed=62)
    shapes = np.concatenate([scenes.random_area_shapes(24, seed=63), coplanar_shapes()])
    rng = np.random.default_rng(64)
    # Points on the shapes: a random point of the shape's plane inside it, to world space.
    k = rng.integers(0, shapes.shape[0], 6000)
    loc = np.stack([rng.uniform(-0.6, 0.6, k.size), np.zeros(k.size), rng.uniform(-0.6, 0.6, k.size),
                    np.ones(k.size)], axis=1)
    loc[:, 0] *= shapes["size"][k, 0]
    loc[:, 2] *= np.where(shapes["kind"][k] == 1, shapes["size"][k, 0], shapes["size"][k, 1])
    world = np.einsum("nij,nj->ni", shapes["matrix"][k].astype(np.float64).reshape(-1, 4, 4), loc)[:, :3]
    on_shapes = aimed_rays(world, rng, jitter=0.02)
    # Straight down onto the coplanar pairs (quad on the ground, disk on its square).
    m = 1500
    top = np.concatenate([np.stack([rng.uniform(0.0, 6.0, m), np.full(m, -1.0), rng.uniform(-4.0, 0.0, m)], 1),
                          np.stack([rng.uniform(-8.0, -4.0, m), np.full(m, 3.0), rng.uniform(5.0, 9.0, m)], 1)])
    down = np.concatenate([top.T, np.tile([[0.0], [-1.0], [0.0]], (1, 2 * m)), np.zeros((1, 2 * m)),
                           np.full((1, 2 * m), 3.4e38)]).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([on_shapes, down, scenes.random_rays(3000, seed=65),
                                                scenes.camera_rays(40, 40, seed=66)], axis=1))
    nall = tri.shape[0] + lines.shape[0] + shapes.shape[0]
    orders = {
        "natural": None,
        "shapes_first": np.concatenate([np.arange(tri.shape[0] + lines.shape[0], nall),
                                        np.arange(0, tri.shape[0] + lines.shape[0])]).astype(np.int32),
        "shuffled": np.random.default_rng(67).permutation(nall).astype(np.int32),
    }
    ref = Reference()
    out = {"triangles": tri, "lines": lines, "shapes": shapes.view(np.uint8).reshape(-1, 140), "rays": rays,
           "order_shapes_first": orders["shapes_first"], "order_shuffled": orders["shuffled"]}
    first_shape = tri.shape[0] + lines.shape[0]
    for name, order in orders.items():
        for w in (4, 8):
            tree = ref.build_shapes(tri, lines, shapes, order, w)
            prim, t, u, v = tree.closest(rays)
            key = f"{name}_{w}"
            out.update({f"prim_{key}": prim, f"t_{key}": t, f"u_{key}": u, f"v_{key}": v,
                        f"occ_{key}": tree.any(rays), f"topology_{key}": tree.topology()})
            print(f"{key}: hits {np.mean(prim >= 0):.3f}, on shapes {np.mean(prim >= first_shape):.3f}, "
                  f"occluded {np.mean(out[f'occ_{key}']):.3f}")
    np.savez_compressed(os.path.join(OUT, "shapes.npz"), **out)


if __name__ == "__main__":
    main()
