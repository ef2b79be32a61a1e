"""Path-traced image parity on the 1080p path-tracing workload's own scene.

The scene is the benchmark's (sort_b200.scenes.pt_scene(1024, 5): 20,971,522
triangles, per-sphere Lambert and GGX-conductor materials, the rectangular
area light), the camera the benchmark's 1920x1080 pinhole cropped to its
central 192x108 pixels (tests/golden/make_golden_pt21m.py). SORT's RNG is
seeded from the wall clock, so renders agree in distribution; the bar, at
equal sample counts, against SORT's own renders (tests/golden/pt21m.npz):
  * 1024 spp: RMSE to SORT's converged image at most 1.3x the RMSE between two
    independent SORT 1024-spp renders, each channel's mean within 1%;
  * 16 spp (the benchmark's sample count): mean RMSE over 8 seeds within 25%
    of SORT's own 16-spp RMSE;
for FP32 nodes and for 8-bit child boxes.
"""
import json
import os

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2)))


@pytest.fixture(scope="module")
def scene21m():
    assert torch.cuda.is_available(), "GPU test needs a CUDA device"
    from sort_b200 import scenes
    _, _, mats, light, tri_gpu, mat_gpu = scenes.pt_scene(1024, 5)
    return tri_gpu, mat_gpu, mats, light


@pytest.mark.parametrize("nodes", ["fp32", "q8"])
def test_pt21m_matches_sort(scene21m, nodes):
    from sort_b200 import _lib
    from sort_b200.pathtracer import PathTracer
    z = golden("pt21m")
    tri_gpu, mat_gpu, mats, light = scene21m
    fmt = _lib.SG_NODES_QUANT8 if nodes == "q8" else _lib.SG_NODES_FP32
    pt = PathTracer(tri_gpu, mat_gpu, mats, light, node_format=fmt)
    cam, w, h, d = z["camera"], int(z["width"]), int(z["height"]), int(z["depth"])
    conv = z["converged"]
    img = pt.Render(cam, w, h, int(z["spp_converged"]), d, seed=11).cpu().numpy()
    assert np.isfinite(img).all()
    r_conv = rmse(img, conv)
    pair = float(z["rmse_converged_pair"])
    m_gpu, m_ref = img.mean(axis=(0, 1)), conv.mean(axis=(0, 1))
    r16 = [rmse(pt.Render(cam, w, h, 16, d, seed=600 + k).cpu().numpy(), conv) for k in range(8)]
    ref16 = float(np.mean(z["rmse16"]))
    pt.Release()
    report = {"workload": "pathtrace_21m crop 192x108 of 1920x1080", "nodes": nodes,
              "rmse_1024spp_vs_sort": r_conv, "sort_pair_rmse_1024spp": pair,
              "rmse_16spp_mean": float(np.mean(r16)), "sort_rmse_16spp_mean": ref16,
              "mean_rgb_gpu": m_gpu.tolist(), "mean_rgb_sort": m_ref.tolist()}
    print(json.dumps(report))
    out = os.environ.get("SORTGPU_REPORT_DIR")
    if out and os.path.isdir(out):
        with open(os.path.join(out, f"pt21m_{nodes}.json"), "w") as f:
            json.dump(report, f)
    assert r_conv <= 1.3 * pair, (r_conv, pair)
    assert np.all(np.abs(m_gpu - m_ref) / m_ref < 0.01), (m_gpu, m_ref)
    assert abs(np.mean(r16) - ref16) <= 0.25 * ref16, (np.mean(r16), ref16)
