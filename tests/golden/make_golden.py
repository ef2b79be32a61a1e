"""Generate tests/golden/*.npz from SORT's own code (oracle/_ref/libsortref.so).

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden.py

Each fixture stores its inputs (triangles, rays) next to the reference outputs,
so the tests need neither the reference tree nor the scene generator to be
bit-stable across machines. The outputs are what SORT's compiled Qbvh / Obvh
return through Accelerator::GetIntersect and GetAttenuation.
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


def edge_scene() -> np.ndarray:
    """Ties and degeneracies: duplicated triangles (equal t, different ids), a
    shared-edge fan, zero-area triangles, an axis-aligned wall, coincident
    centroids (forces the zero-width SAH bin case)."""
    tris = []
    # fan of 8 triangles around (0, 0, 0) in the z = 0 plane, sharing edges
    for k in range(8):
        a0, a1 = 2 * np.pi * k / 8, 2 * np.pi * (k + 1) / 8
        tris.append([0, 0, 0, np.cos(a0), np.sin(a0), 0, np.cos(a1), np.sin(a1), 0])
    base = np.array(tris, np.float64)
    dup = base.copy()                    # exact duplicates -> exact t ties
    tris = np.concatenate([base, dup])
    # zero-area triangles (collinear, point)
    degen = np.array([[2, 2, 1, 3, 3, 1, 4, 4, 1], [1, 1, 1, 1, 1, 1, 1, 1, 1]], np.float64)
    # axis-aligned wall at x = 3 (two triangles)
    wall = np.array([[3, -2, -2, 3, 2, -2, 3, 2, 2], [3, -2, -2, 3, 2, 2, 3, -2, 2]], np.float64)
    # 24 copies of one small triangle at the same place (coincident centroids)
    stack = np.tile(np.array([[-3, 0, 0, -3, 0.5, 0, -3, 0, 0.5]], np.float64), (24, 1))
    return np.ascontiguousarray(np.concatenate([tris, degen, wall, stack]).astype(np.float32))


def edge_rays() -> np.ndarray:
    rng = np.random.default_rng(5)
    rows = []
    # straight down the z axis through the fan centre and along shared edges
    for k in range(8):
        a = 2 * np.pi * k / 8
        for s in (0.0, 0.25, 0.5, 0.999):
            rows.append([s * np.cos(a), s * np.sin(a), 5, 0, 0, -1, 0, 3.4e38])
    # axis-aligned rays at the wall and the coincident stack
    rows += [[0, 0, 0, 1, 0, 0, 0, 3.4e38], [-5, 0.1, 0.1, 1, 0, 0, 0, 3.4e38],
             [0, 0.1, 0.1, -1, 0, 0, 0, 3.4e38], [3, 0, 0, 1, 0, 0, 0, 3.4e38],
             [0, 0, 5, 0, 0, -1, 5, 3.4e38],     # tmin equal to the hit distance: t > tmin fails
             [0.1, 0.1, 5, 0, 0, -1, 0, 5],      # tmax equal to the hit distance: t <= tmax passes
             [0.1, 0.1, 5, 0, 0, -1, 0, 4.999]]  # tmax just short
    o = rng.uniform(-4, 4, (200, 3))
    d = rng.normal(size=(200, 3))
    d[::3, 1] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    for i in range(200):
        rows.append([*o[i], *d[i], 0, 3.4e38])
    r = np.array(rows, np.float64).T
    return np.ascontiguousarray(r.astype(np.float32))


def spheres_case() -> tuple[np.ndarray, np.ndarray]:
    tri = scenes.sphere_field(6, 2, seed=21)          # 1,922 triangles
    cam = scenes.camera_rays(48, 48, seed=22)          # 2,304 primary rays
    rnd = scenes.random_rays(1024, seed=23)
    return tri, np.ascontiguousarray(np.concatenate([cam, rnd], axis=1))


def directions() -> np.ndarray:
    rng = np.random.default_rng(9)
    d = rng.normal(size=(256, 3))
    d[:32, 0] = 0
    d[32:64, 1] = 0
    d[64:80, :2] = 0
    d[80:96] = np.round(d[80:96])
    d[80:96][np.all(d[80:96] == 0, axis=1)] = 1.0
    return d.astype(np.float32)


def run_case(ref: Reference, name: str, tri: np.ndarray, rays: np.ndarray, depth: int, leaf: int) -> None:
    out = dict(triangles=tri, rays=rays, max_depth=np.int32(depth), max_leaf=np.int32(leaf))
    for w in (4, 8):
        tree = ref.build(tri, w, depth, leaf)
        prim, t, u, v = tree.closest(rays)
        occ = tree.any(rays)
        out[f"w{w}_topology"] = tree.topology()
        out[f"w{w}_depth"] = np.int32(tree.depth())
        out[f"w{w}_bbox"] = tree.bbox()
        out[f"w{w}_prim"], out[f"w{w}_t"], out[f"w{w}_u"], out[f"w{w}_v"] = prim, t, u, v
        out[f"w{w}_occ"] = occ
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    print(name, tri.shape[0], "triangles", rays.shape[1], "rays")


def main() -> None:
    ref = Reference()
    tri, rays = spheres_case()
    run_case(ref, "spheres_1922", tri, rays, 16, 8)
    run_case(ref, "edges", edge_scene(), edge_rays(), 16, 8)
    run_case(ref, "edges_leaf1_depth4", edge_scene(), edge_rays(), 4, 1)
    d = directions()
    lx = np.zeros((len(d), 3), np.int32)
    sc = np.zeros((len(d), 3), np.float32)
    for i in range(len(d)):
        ref.L.sortref_ray_prepare(d[i].ctypes.data, lx[i].ctypes.data, sc[i].ctypes.data)
    np.savez_compressed(os.path.join(OUT, "ray_prepare.npz"), dirs=d, local=lx, scale=sc)
    print("ray_prepare", len(d), "directions")


if __name__ == "__main__":
    main()
