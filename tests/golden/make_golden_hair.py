"""Generate tests/golden/hair.npz: SORT's answers on a scene with hair (oracle/_ref).

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden_hair.py

16 level-2 icospheres plus a ground quad, followed by 400 hair strands of 8
segments (SORT's Line shapes, made as HairVisual makes them, entity/visual.cpp:
41-97). Rays: some aimed at random points of the segments (most hit a line),
random rays, camera rays. Stored per width (QBVH 4, OBVH 8): closest hit
(prim, t, u, v) as Fbvh::GetIntersect returns it (line hits from
intersectLine_SIMD, simd/simd_line.h:232-330) and the any-hit answer.
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
    tri = scenes.sphere_field(16, 2, seed=51)
    lines = scenes.hair_strands(400, 8, seed=52)
    rng = np.random.default_rng(53)
    m = 6000
    k = rng.integers(0, lines.shape[0], m)
    f = rng.uniform(0.05, 0.95, m)[:, None]
    tgt = lines[k, 0:3] * (1 - f) + lines[k, 3:6] * f + rng.normal(scale=0.01, size=(m, 3))
    o = tgt + rng.normal(size=(m, 3)) * 6.0
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    aimed = np.concatenate([o.T, d.T, np.zeros((1, m)), np.full((1, m), 3.4e38)]).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([aimed, scenes.random_rays(4000, seed=54),
                                                scenes.camera_rays(48, 48, seed=55)], axis=1))
    ref = Reference()
    out = {"triangles": tri, "lines": lines, "rays": rays}
    for w in (4, 8):
        tree = ref.build_hair(tri, lines, w)
        prim, t, u, v = tree.closest(rays)
        out.update({f"prim{w}": prim, f"t{w}": t, f"u{w}": u, f"v{w}": v, f"occ{w}": tree.any(rays),
                    f"topology{w}": tree.topology()})
        on_line = prim >= tri.shape[0]
        print(f"width {w}: hits {np.mean(prim >= 0):.3f}, on lines {np.mean(on_line):.3f}, "
              f"occluded {np.mean(out[f'occ{w}']):.3f}")
    np.savez_compressed(os.path.join(OUT, "hair.npz"), **out)


if __name__ == "__main__":
    main()
