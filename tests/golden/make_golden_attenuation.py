"""Generate tests/golden/attenuation.npz: SORT's transparent-shadow query (oracle/_ref).

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden_attenuation.py

A 48-sphere field plus a ground quad. Materials 0..5: four transparent ones
(one with a zero channel, one fully black) and two opaque ones. Two material
assignments: by sphere (rays cross whole transparent shells), and per triangle
at random (a leaf's SIMD packs mix transparent and opaque hits, so SORT's rule
of checking only each pack's nearest hit matters). Rays: long rays across the
field, shadow-like random segments, and camera rays. Stored per width (QBVH 4,
OBVH 8) and assignment: the rgb attenuation Scene::GetAttenuation returns
(core/scene.cpp:192-208 over accel/accelerator.cpp:26-69).
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
TRANSPARENT = np.array([1, 1, 1, 1, 0, 0], np.int32)
RGB = np.array([[0.5, 0.75, 0.875], [0.9, 0.6, 0.3], [0.5, 0.0, 1.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0],
                [0.3, 0.3, 0.3]], np.float32)


def main():
    tri = scenes.sphere_field(48, 2, seed=41)  # 320 triangles per sphere, ground quad last
    per = 320
    rng = np.random.default_rng(42)
    by_sphere = np.zeros(tri.shape[0], np.int32)
    sphere_mat = rng.choice(6, 48, p=[0.3, 0.3, 0.1, 0.05, 0.15, 0.1]).astype(np.int32)
    by_sphere[:48 * per] = np.repeat(sphere_mat, per)
    by_sphere[48 * per:] = 4  # opaque ground
    per_tri = rng.choice(6, tri.shape[0], p=[0.35, 0.3, 0.05, 0.05, 0.15, 0.1]).astype(np.int32)
    m = 3072
    o = np.stack([rng.uniform(-10, 10, m), rng.uniform(-10, 10, m), np.full(m, -30.0)])
    tgt = np.stack([rng.uniform(-10, 10, m), rng.uniform(-10, 10, m), np.full(m, 30.0)])
    d = tgt - o
    length = np.linalg.norm(d, axis=0)
    d /= length
    long_rays = np.concatenate([o, d, np.full((1, m), 1e-4), (length - 0.01)[None]]).astype(np.float32)
    shadow = scenes.random_rays(3072, seed=43)
    shadow[7] = rng.uniform(1.0, 25.0, shadow.shape[1]).astype(np.float32)  # finite segments
    rays = np.ascontiguousarray(np.concatenate([long_rays, shadow, scenes.camera_rays(40, 40, seed=44)], axis=1))
    ref = Reference()
    out = {"triangles": tri, "by_sphere": by_sphere, "per_tri": per_tri, "transparent": TRANSPARENT, "rgb": RGB,
           "rays": rays}
    for w in (4, 8):
        for name, mat in (("by_sphere", by_sphere), ("per_tri", per_tri)):
            att = ref.build_transparent(tri, mat, TRANSPARENT, RGB, w).attenuation(rays)
            out[f"att{w}_{name}"] = att
            print(f"width {w}, {name}: unattenuated {np.mean(att[0] == 1):.3f}, black {np.mean(att.sum(0) == 0):.3f}, "
                  f"partial {np.mean((att[0] > 0) & (att[0] < 1)):.3f}")
    np.savez_compressed(os.path.join(OUT, "attenuation.npz"), **out)


if __name__ == "__main__":
    main()
