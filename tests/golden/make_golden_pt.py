"""Generate tests/golden/pt_spheres.npz from SORT's own path tracer.

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden_pt.py

SORT's PathTracing::Li (compiled from its sources into oracle/_ref/libsortref.so)
renders the scene of sort_b200.scenes.pt_scene(16, 2): a converged image at 4096
samples per pixel, an independent second one (their RMSE is the noise floor two
converged renders differ by), and eight 16-sample renders whose RMSE against the
converged image is the noise a 16-sample render shows. The GPU test compares its
own renders against these numbers.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import RefPathTracer  # noqa: E402
from sort_b200 import scenes  # noqa: E402

W, H, DEPTH = 48, 48, 5


def rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)))


def main():
    tri, mat_of_tri, mats, light, _, _ = scenes.pt_scene(16, 2)
    pt = RefPathTracer().build(tri, mat_of_tri, mats, light)
    conv = pt.render(scenes.CAMERA, W, H, 4096, DEPTH, seed=101)
    conv2 = pt.render(scenes.CAMERA, W, H, 4096, DEPTH, seed=202)
    r16 = [rmse(pt.render(scenes.CAMERA, W, H, 16, DEPTH, seed=300 + k), conv) for k in range(8)]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "pt_spheres.npz"), converged=conv,
                        converged_b=conv2, rmse_converged_pair=np.float64(rmse(conv, conv2)),
                        rmse16=np.array(r16), width=np.int32(W), height=np.int32(H), depth=np.int32(DEPTH),
                        spheres=np.int32(16), level=np.int32(2), camera=scenes.CAMERA, light=light)
    print("mean", conv.mean(axis=(0, 1)), "pair rmse", rmse(conv, conv2), "rmse16", np.mean(r16), np.std(r16))


if __name__ == "__main__":
    main()
