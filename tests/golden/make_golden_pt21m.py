"""Generate tests/golden/pt21m.npz: SORT's path-traced renders of the 1080p
path-tracing workload's scene, on a crop of its frame (oracle/_ref).

Run from the repository root after ``make -C oracle ref`` (a few minutes on 8
cores; SORT builds its 21M-triangle tree on one thread):

    python tests/golden/make_golden_pt21m.py

Scene: sort_b200.scenes.pt_scene(1024, 5) -- 1,024 level-5 icospheres and a
ground quad (20,971,522 triangles) with per-sphere materials (half Lambert,
half GGX conductor) and the rectangular area light. Camera: the workload's
(scenes.CAMERA, 1920x1080, 45 degrees vertical) cropped to a 192x108
window centred on full-frame pixel (600, 100): the lit sphere tops below the
light, where the frame has signal (much of it is in shadow). The window is
rendered as the same pinhole aimed through that pixel with the field of view
narrowed to the window (crop_camera). SORT's PathTracing::Li (depth 5, NEE with MIS,
Russian roulette) renders it at 1024 samples per pixel twice (independent
seeds: their RMSE is the floor two converged renders differ by) and eight
times at 16 samples (their RMSE against the converged image is the noise a
16-sample render shows). The GPU test compares its own renders with these.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.oracle import RefPathTracer  # noqa: E402
from sort_b200 import scenes  # noqa: E402

FULL_W, FULL_H, CROP_W, CROP_H, DEPTH = 1920, 1080, 192, 108, 5
CROP_CENTRE = (600.0, 100.0)  # full-frame pixel the window is centred on


def crop_camera(camera=scenes.CAMERA, centre=CROP_CENTRE, full_w=FULL_W, full_h=FULL_H, crop_h=CROP_H):
    """The pinhole aimed through full-frame pixel `centre` of camera's
    full_w x full_h frame, with the vertical field of view of crop_h rows."""
    cam = np.array(camera, np.float64)
    eye, target, up = cam[0:3], cam[3:6], cam[6:9]
    fwd = (target - eye) / np.linalg.norm(target - eye)
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    half_h = np.tan(np.radians(cam[9]) * 0.5)
    half_w = half_h * full_w / full_h
    sx = (centre[0] / full_w * 2.0 - 1.0) * half_w
    sy = (1.0 - centre[1] / full_h * 2.0) * half_h
    d = fwd + right * sx + upv * sy
    out = cam.copy()
    out[3:6] = eye + d / np.linalg.norm(d) * np.linalg.norm(target - eye)
    out[9] = np.degrees(2.0 * np.arctan(half_h * crop_h / full_h))
    return out.astype(np.float32)


def rmse(a, b):
    return float(np.sqrt(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)))


def main():
    t0 = time.time()
    tri, mat_of_tri, mats, light, _, _ = scenes.pt_scene(1024, 5)
    pt = RefPathTracer().build(tri, mat_of_tri, mats, light)
    print(f"SORT scene built in {time.time() - t0:.1f} s")
    cam = crop_camera()
    t0 = time.time()
    conv = pt.render(cam, CROP_W, CROP_H, 1024, DEPTH, seed=4101)
    print(f"converged render in {time.time() - t0:.1f} s")
    conv2 = pt.render(cam, CROP_W, CROP_H, 1024, DEPTH, seed=4202)
    r16 = [rmse(pt.render(cam, CROP_W, CROP_H, 16, DEPTH, seed=4300 + k), conv) for k in range(8)]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "pt21m.npz"), converged=conv,
                        rmse_converged_pair=np.float64(rmse(conv, conv2)), rmse16=np.array(r16),
                        width=np.int32(CROP_W), height=np.int32(CROP_H), depth=np.int32(DEPTH), camera=cam,
                        full_width=np.int32(FULL_W), full_height=np.int32(FULL_H), light=light,
                        crop_centre=np.array(CROP_CENTRE, np.float32),
                        spp_converged=np.int32(1024))
    print("mean", conv.mean(axis=(0, 1)), "pair rmse", rmse(conv, conv2), "rmse16", np.mean(r16), np.std(r16))


if __name__ == "__main__":
    main()
