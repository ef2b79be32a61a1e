"""Generate tests/golden/multi.npz: SORT's BSSRDF probe query (oracle/_ref).

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden_multi.py

A 48-sphere field whose spheres carry materials 0..2 (by sphere) plus a
ground quad of material 0, queried with rays that cross many spheres (long
rays along the field, camera rays, random rays), each ray asking for one
material. Stored per width (QBVH 4, OBVH 8): the hit count and SORT's four
(prim, t, u, v) slots per ray, as Fbvh::GetIntersect(ray, BSSRDFIntersections&,
rc, matID) leaves them (accel/fast_bvh.hpp:656-819).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from sort_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def main():
    tri = scenes.sphere_field(48, 2, seed=21)  # 320 triangles per sphere, ground quad last
    per = 320
    mat = np.zeros(tri.shape[0], np.int32)
    mat[:48 * per] = (np.arange(48 * per) // per) % 3
    rng = np.random.default_rng(22)
    # long rays through the field: origins on a plane at z = -30, aimed across it
    m = 4096
    o = np.stack([rng.uniform(-10, 10, m), rng.uniform(-10, 10, m), np.full(m, -30.0)])
    tgt = np.stack([rng.uniform(-10, 10, m), rng.uniform(-10, 10, m), np.full(m, 30.0)])
    d = tgt - o
    d /= np.linalg.norm(d, axis=0)
    long_rays = np.concatenate([o, d, np.zeros((1, m)), np.full((1, m), 3.4e38)]).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([long_rays, scenes.camera_rays(48, 48, seed=23),
                                                scenes.random_rays(4096, seed=24)], axis=1))
    ray_mat = rng.integers(0, 3, rays.shape[1]).astype(np.int32)
    ref = Reference()
    out = {"triangles": tri, "mat_of_tri": mat, "rays": rays, "ray_mat": ray_mat}
    for w in (4, 8):
        count, prim, t, u, v = ref.build_materials(tri, mat, 3, w).multi(rays, ray_mat)
        out.update({f"count{w}": count, f"prim{w}": prim, f"t{w}": t, f"u{w}": u, f"v{w}": v})
        print(f"width {w}: hits kept per ray {np.bincount(count)}")
        # one material everywhere: long rays collect more than 4 hits, so
        # SORT's overwrite-the-farthest path and its maxt culling are exercised
        count, prim, t, u, v = ref.build_materials(tri, np.zeros_like(mat), 1, w).multi(rays, np.zeros_like(ray_mat))
        out.update({f"count{w}_one": count, f"prim{w}_one": prim, f"t{w}_one": t, f"u{w}_one": u, f"v{w}_one": v})
        print(f"width {w}, one material: hits kept per ray {np.bincount(count)}")
    np.savez_compressed(os.path.join(OUT, "multi.npz"), **out)


if __name__ == "__main__":
    main()
