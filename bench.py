"""Benchmark: incoherent closest-hit Mrays/s on the 21M-triangle OBVH workload.

Workload (one "step" = one batch through the hot path): 1,024 level-5 icospheres
plus a ground quad (20,971,522 triangles), built as SORT's OBVH (width 8,
max depth 16, leaf 8); 4,194,304 cosine-weighted diffuse rays spawned from the
hits of a 2048x2048 pinhole camera, traced closest-hit in one launch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours: every rank holds a replica of the tree and traces its own 4M-ray batch
(weak scaling, no collective on the data path). value = all ranks' rays / the
slowest rank's device time. e2e = the same batch through the host-buffer C-ABI
call (pinned host rays in, hits out, copies inside the timed region).
reference: SORT's own OBVH code (compiled from its sources into oracle/_ref)
on the host cores, on a bounded sample of the same rays each step; rank 0 only.

Other workloads (--workload):
  raycast    81,922-triangle QBVH, 1M jittered primary rays (L2-resident tree);
  pathtrace  the 21M scene with per-sphere materials, 1920x1080, depth 5, one
             sample per pixel per step (wavefront path tracer);
  batched    8 resident scenes (10k..16M triangles), a list of uneven ray
             batches per step: persistent multi-scene kernel under a captured
             CUDA graph (autotuned) vs one plain launch per batch;
  serve      4 resident path-tracing scenes, a Poisson stream of render
             requests: the render server vs FIFO per-request renders;
  build      GPU build of the 21M-triangle OBVH (SORT's tree), one build per
             step; reference arm: SORT's single-threaded Fbvh::Build.
--nodes q8 times 8-bit child boxes (closest, raycast, pathtrace).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s incoherent closest-hit"
UNIT = "Mrays/s"
SPHERES, LEVEL, IMAGE = 1024, 5, 2048
WIDTH, DEPTH, LEAF = 8, 16, 8
NODE_BYTES = {4: 112, 8: 224}   # FP32 canonical wide node: W*24 B boxes + W*4 B refs
TRI_BYTES = 36                  # 9 floats per triangle test
RAY_IN, HIT_OUT = 32, 16
CPU_SAMPLE = 262_144            # rays per CPU-baseline step
NODE_FORMATS = {"fp32": 0, "q8": 1}
BUILDERS = {"host": 0, "gpu": 1, "lbvh": 2, "ploc": 3}  # host / gpu: SORT's tree; lbvh / ploc: built from Morton order
MORTON_TREES = {"lbvh": "LBVH (radix tree over the Morton order, built on the GPU)",
                "ploc": "PLOC (parallel locally-ordered clustering over the Morton order, built on the GPU)"}


def workload_config(extra=None):
    cfg = {
        "workload": "incoherent_21m: 1,024 level-5 icospheres + ground quad = 20,971,522 triangles, "
                    "OBVH (width 8, depth 16, leaf 8), 4,194,304 cosine-diffuse closest-hit rays per GPU "
                    "from 2048x2048 primary hits",
        "scene_seed": 1,
        "nodes": "fp32",
        "l2": "inputs larger than L2: 1.25 GB tree + 128 MB rays per launch (no flush)",
    }
    if extra:
        cfg.update(extra)
    return cfg


def raycast_config(extra=None):
    cfg = {
        "workload": "raycast_82k: 64 level-3 icospheres + ground quad = 81,922 triangles, QBVH (width 4, depth 16, "
                    "leaf 8), 1,048,576 jittered primary rays (1024x1024 pinhole at (0,0,30), 45 deg) per GPU",
        "scene_seed": 1,
        "nodes": "fp32",
        "l2": "tree (5 MB) is L2-resident by design of this workload; rays 32 MB",
    }
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def make_rays(acc, tri, rank: int, device):
    """Primary camera rays traced on the GPU, then the diffuse + shadow batches."""
    import torch

    from sort_b200 import scenes
    cam = scenes.camera_rays(IMAGE, IMAGE, seed=7)
    h = acc.GetIntersect(torch.from_numpy(cam).to(device))
    prim = h.prim.cpu().numpy()
    t = h.t.cpu().numpy()
    diffuse, shadow = scenes.bounce_rays(tri, cam, prim, t, IMAGE * IMAGE, seed=11 + rank)
    return diffuse, shadow


def reference_cpu(tri, rays, steps: int, warmup: int, threads: int, sample: int, width: int = WIDTH):
    """SORT's OBVH on the host cores; returns (Mrays/s, kind, description, the
    last timed block's first ray, SORT's (prim, t) for that block, the tree)."""
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        from oracle.oracle import Port
        impl, kind = Port(), "port"
    else:
        impl, kind = Reference(), "reference"
    tree = impl.build(tri, width, DEPTH, LEAF)
    n = rays.shape[1]
    times = []
    s, prim, t = 0, None, None
    for k in range(warmup + steps):
        s = (k * sample) % max(1, n - sample)
        block = np.ascontiguousarray(rays[:, s:s + sample])
        t0 = time.perf_counter()
        prim, t, _, _ = tree.closest(block, threads)
        dt = time.perf_counter() - t0
        if k >= warmup:
            times.append(dt)
    rate = sample * len(times) / sum(times) / 1e6
    return rate, kind, f"{sample} of the {n} diffuse rays per step, {len(times)} timed steps", s, (prim, t)


def parity_on_sample(tri, rays, first, sort_hits, gpu_prim, gpu_t):
    """The GPU's hits on the CPU baseline's last block against SORT's, and both
    hits' t error against an FP64 re-intersection of the hit triangle."""
    from oracle.oracle import Port
    sp, st = sort_hits
    m = sp.shape[0]
    gp, gt = gpu_prim[first:first + m], gpu_t[first:first + m]
    block = np.ascontiguousarray(rays[:, first:first + m])
    port = Port()
    eg = port.fp64_rel_err(tri, gp, gt, block)
    es = port.fp64_rel_err(tri, sp, st, block)

    def summary(e):
        return {"max": float(e.max()), "p99": float(np.percentile(e, 99)), "mean": float(e.mean())} if e.size else None
    return {"rays": int(m), "prim_differs": int((gp != sp).sum()),
            "t_bits_differ": int((gt.view(np.int32) != st.view(np.int32)).sum()),
            "fp64_rel_err": {"gpu": summary(eg), "sort": summary(es), "hits": int(eg.size)}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from sort_b200 import scenes
    from oracle.oracle import Reference, reference_available
    tri = scenes.sphere_field(SPHERES, LEVEL, seed=1)
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "SORT reference library (oracle/_ref) not built"}))
        return
    ref = Reference()
    threads = ref.hardware_threads()
    tree = ref.build(tri, WIDTH, DEPTH, LEAF)
    cam = scenes.camera_rays(IMAGE, IMAGE, seed=7)
    prim, t, _, _ = tree.closest(cam, threads)
    diffuse, _ = scenes.bounce_rays(tri, cam, prim, t, IMAGE * IMAGE, seed=11)
    n = diffuse.shape[1]
    sample = args.sample
    times = []
    for k in range(args.warmup + args.steps):
        s = (k * sample) % max(1, n - sample)
        block = np.ascontiguousarray(diffuse[:, s:s + sample])
        t0 = time.perf_counter()
        tree.closest(block, threads)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = sample * len(times) / total / 1e6
    out = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * total / len(times), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config({"sample_rays_per_step": sample}),
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{sample} of the {n} diffuse rays per step (SORT Obvh::GetIntersect, AVX)"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(out))


def run_ours(args):
    import torch
    import torch.distributed as dist

    from sort_b200 import Hits, Obvh, scenes
    from sort_b200.replicas import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=device)

    def barrier():
        if world > 1:
            dist.barrier()

    if args.workload == "raycast":
        # raycast_82k: 64 level-3 icospheres + ground (81,922 triangles) as a QBVH,
        # 1024x1024 jittered primary rays (closest-hit); shadow rays from their hits.
        from sort_b200 import Qbvh
        width = 4
        tri = scenes.sphere_field(64, 3, seed=1)
        acc = Qbvh(DEPTH, LEAF, node_format=NODE_FORMATS[args.nodes], device=local,
                   builder=BUILDERS[args.builder or "host"])
        acc.Build(tri)
        diffuse = scenes.camera_rays(1024, 1024, seed=7 + rank)
        h = acc.GetIntersect(torch.from_numpy(diffuse).to(device))
        _, shadow = scenes.bounce_rays(tri, diffuse, h.prim.cpu().numpy(), h.t.cpu().numpy(), diffuse.shape[1],
                                       seed=11 + rank)
    else:
        width = WIDTH
        tri = scenes.sphere_field(SPHERES, LEVEL, seed=1)
        acc = Obvh(DEPTH, LEAF, node_format=NODE_FORMATS[args.nodes], device=local,
                   builder=BUILDERS[args.builder or "host"])
        acc.Build(tri)
        diffuse, shadow = make_rays(acc, tri, rank, device)
    info = acc.info()
    n = diffuse.shape[1]
    d_diff = torch.from_numpy(diffuse).to(device)
    d_shad = torch.from_numpy(shadow).to(device)

    # SORT's traversal counters on these rays -> algorithmic bytes per ray. The
    # counts are SORT's (FP32 boxes), whatever node format is timed.
    parity = None
    if args.nodes == "fp32" and args.builder not in MORTON_TREES:
        node_tests, prim_tests = acc.TraceStats(d_diff, False)
        a_nodes, a_prims = acc.TraceStats(d_shad, True)
    else:
        ref_acc = type(acc)(DEPTH, LEAF, device=local)
        ref_acc.Build(tri)
        node_tests, prim_tests = ref_acc.TraceStats(d_diff, False)
        a_nodes, a_prims = ref_acc.TraceStats(d_shad, True)
        hf, hq = ref_acc.GetIntersect(d_diff), acc.GetIntersect(d_diff)
        diff = hf.prim != hq.prim
        tie = diff & (hf.prim >= 0) & (hq.prim >= 0) & ((hq.t - hf.t).abs() <= 1e-6 * hf.t)
        parity = {"rays": n, "prim_differs": int(diff.sum()), "near_ties": int(tie.sum()),
                  "same_prim_t_bits_equal": bool(torch.equal(hf.t[~diff], hq.t[~diff]))}
        ref_acc.Release()
        torch.cuda.empty_cache()
    bytes_closest = RAY_IN + HIT_OUT + (node_tests * NODE_BYTES[width] + prim_tests * TRI_BYTES) / n
    bytes_any = RAY_IN + 4 + (a_nodes * NODE_BYTES[width] + a_prims * TRI_BYTES) / n

    stream = torch.cuda.current_stream(device)
    for _ in range(args.warmup):
        acc.GetIntersect(d_diff)
    torch.cuda.synchronize(device)
    barrier()
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            acc.GetIntersect(d_diff)
        end.record(stream)
        torch.cuda.synchronize(device)
    barrier()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(end)
    ms_max = max_over_ranks(ms, device)
    value = world * n * args.steps / (ms_max / 1e3) / 1e6
    launch_ms = ms / args.steps

    # any-hit (shadow) launch, timed the same way
    for _ in range(args.warmup):
        acc.GetAttenuation(d_shad)
    torch.cuda.synchronize(device)
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(args.steps):
        acc.GetAttenuation(d_shad)
    e2.record(stream)
    torch.cuda.synchronize(device)
    any_ms = s2.elapsed_time(e2) / args.steps

    # end to end through the host-buffer C-ABI call, pinned host memory
    h_rays = torch.from_numpy(diffuse).pin_memory()
    outs = Hits(torch.empty(n, dtype=torch.int32).pin_memory().numpy(),
                torch.empty(n, dtype=torch.float32).pin_memory().numpy(),
                torch.empty(n, dtype=torch.float32).pin_memory().numpy(),
                torch.empty(n, dtype=torch.float32).pin_memory().numpy())
    h_np = h_rays.numpy()
    for _ in range(max(1, args.warmup)):
        acc.GetIntersect(h_np, out=outs)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        acc.GetIntersect(h_np, out=outs)
    e2e_s = time.perf_counter() - t0
    e2e_value = world * n * args.steps / max_over_ranks(e2e_s, device) / 1e6

    h_all = acc.GetIntersect(d_diff)  # the timed call's answers, for the parity check below (untimed)
    torch.cuda.synchronize(device)
    gpu_prim, gpu_t = h_all.prim.cpu().numpy(), h_all.t.cpu().numpy()

    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if width == 4:
        # The 82k-triangle tree (~5 MB) stays in L2: its roofline is L2 bandwidth,
        # measured here by the library's probe kernel.
        import ctypes

        from sort_b200 import _lib
        g = ctypes.c_double(0.0)
        _lib.check(_lib.load().sg_probe_l2_read_gbs(local, 64 << 20, 50, ctypes.byref(g)))
        bound, peak, peak_src = "l2", round(g.value, 1), "measured L2 read GB/s (sg_probe_l2_read_gbs, 64 MiB x 50)"
    elif os.path.exists(peaks_path):
        bound, peak, peak_src = "hbm", float(json.load(open(peaks_path))["hbm_gbs"]), "measured hbm_gbs (burst)"
    else:
        bound, peak, peak_src = "hbm", 6650.0, "fallback hbm GB/s"
    achieved = bytes_closest * n / (launch_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):  # ncu DRAM bytes of this kernel, one launch of this workload
        for tj in json.load(open(tpath)):
            if (tj.get("workload") == ("raycast_82k" if width == 4 else "incoherent_21m")
                    and tj.get("nodes") == args.nodes and args.builder not in MORTON_TREES):
                traffic = tj.get("dram_bytes_per_launch")

    if rank == 0:
        sorted_schedule = n >= (1 << 21)
        out = {
            "metric": METRIC if width == 8 else "Mrays/s primary closest-hit", "value": round(value, 3),
            "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": (raycast_config if width == 4 else workload_config)(
                ({"nodes": args.nodes} if args.nodes != "fp32" else {}) |
                ({"tree": MORTON_TREES[args.builder] + "; algorithmic bytes counted on SORT's tree"}
                 if args.builder in MORTON_TREES else {})) | (
                {"parallelism": f"replicas x{world}", "build_seconds": round(info["build_seconds"], 2),
                 "tree_device_bytes": info["device_bytes"],
                 "schedule": "rays in the order of a 30-bit coherence key (hand-written stable radix sort, "
                             "3 passes of 10 bits), then one per thread (default for >= 2^21 closest-hit rays; the "
                             "sort is inside the timed step)"
                             if sorted_schedule else "one ray per thread"}),
            "roofline": {"bound": bound, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_ray": round(bytes_closest, 1),
                         "node_tests_per_ray": round(node_tests / n, 3), "prim_tests_per_ray": round(prim_tests / n, 3),
                         "kernel": f"k_trace_walk<{width},false,{64 if width == 4 else 128},"
                                   + ("true>" if args.nodes == "q8" else "false>"),
                         "launch_ms": round(launch_ms, 4)},
            "anyhit": {"mrays_s": round(n / (any_ms / 1e3) / 1e6, 3), "launch_ms": round(any_ms, 4),
                       "algorithmic_bytes_per_ray": round(bytes_any, 1),
                       "achieved_gbs": round(bytes_any * n / (any_ms / 1e3) / 1e9, 1)},
            "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": int(n * 32),
                    "d2h_bytes_per_step": int(n * 16)},
            "clocks": clocks.summary(),
            # the default schedule sorts closest-hit batches of >= 2^21 FP32 rays: the key kernel (which also
            # counts the first digit), then per 10-bit digit a tile scan, a tile-sum scan and a scatter, the
            # next digit's count between passes, then the traversal kernel: 13 launches for 4M rays
            "gpu_launches": args.steps * (13 if sorted_schedule else 1),
            **({"parity_vs_fp32_nodes": parity} if parity else {}),
        }
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            rate, kind, desc, first, sort_hits = reference_cpu(tri, diffuse, steps=3, warmup=1, threads=threads,
                                                               sample=args.sample, width=width)
            out["cpu_baseline"] = {"value": round(rate, 3), "unit": UNIT, "cores": threads, "kind": kind,
                                   "sample": desc}
            if args.nodes == "fp32" and args.builder not in MORTON_TREES:
                out["parity"] = parity_on_sample(tri, diffuse, first, sort_hits, gpu_prim, gpu_t)
        print(json.dumps(out))
    acc.Release()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


PT_W, PT_H, PT_DEPTH = 1920, 1080, 5


def pt_config(extra=None):
    cfg = {
        "workload": "pathtrace_21m: the incoherent_21m scene with per-sphere materials (50% Lambert albedo "
                    "U(0.2,0.8), 50% GGX conductor roughness U(0.05,0.5)), one 8x8 area light, 1920x1080, "
                    "max depth 5, Russian roulette after depth 3, NEE with MIS; one step = one sample per pixel",
        "nodes": "fp32",
    }
    if extra:
        cfg.update(extra)
    return cfg


def run_pathtrace(args):
    """Path-traced samples/s (one step = one sample for every pixel of 1920x1080)."""
    import torch

    from sort_b200 import scenes
    from sort_b200.pathtracer import PathTracer

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle.oracle import RefPathTracer, reference_available
        if not reference_available():
            print(json.dumps({"impl": "reference", "unavailable": "SORT reference library (oracle/_ref) not built"}))
            return
        tri, m, mats, light, _, _ = scenes.pt_scene(SPHERES, LEVEL)
        ref = RefPathTracer().build(tri, m, mats, light)
        w, h = 192, 108  # bounded pixel sample of the same camera
        times = []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            ref.render(scenes.CAMERA, w, h, 1, PT_DEPTH, seed=1000 + k)
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        value = w * h * len(times) / sum(times) / 1e6
        out = {"impl": "reference", "metric": "path-traced Msamples/s", "value": round(value, 4),
               "unit": "Msamples/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": round(1e3 * sum(times) / len(times), 3), "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": pt_config({"pixels": w * h}),
               "cpu_baseline": {"value": round(value, 4), "unit": "Msamples/s", "cores": os.cpu_count(),
                                "kind": "reference", "sample": f"{w}x{h} pixels, 1 sample each per step"},
               "e2e": {"value": round(value, 4), "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                       "d2h_bytes_per_step": 0}, "gpu_launches": 0}
        print(json.dumps(out))
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    _, _, mats, light, tri_gpu, mat_gpu = scenes.pt_scene(SPHERES, LEVEL)
    pt = PathTracer(tri_gpu, mat_gpu, mats, light, device=local, node_format=NODE_FORMATS[args.nodes])
    img = torch.empty((PT_H, PT_W, 3), dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)
    pt.Render(scenes.CAMERA, PT_W, PT_H, args.warmup, PT_DEPTH, seed=1, out=img)
    torch.cuda.synchronize(device)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        pt.Render(scenes.CAMERA, PT_W, PT_H, args.steps, PT_DEPTH, seed=2, out=img)
        end.record(stream)
        torch.cuda.synchronize(device)
    ms = start.elapsed_time(end)
    ext, sh = pt.RayCounts()
    host_img = torch.empty((PT_H, PT_W, 3), dtype=torch.float32).pin_memory()  # the caller's result buffer
    t0 = time.perf_counter()
    pt.Render(scenes.CAMERA, PT_W, PT_H, args.steps, PT_DEPTH, seed=3, out=img)
    host_img.copy_(img)
    e2e_s = time.perf_counter() - t0
    samples = PT_W * PT_H * args.steps
    # Image error against SORT's converged render of a 192x108 window of this
    # frame (tests/golden/pt21m.npz, made by SORT's PathTracing::Li at 1024 spp),
    # at the workload's 16 spp, beside SORT's own 16-spp error (untimed).
    rmse_info = None
    gpath = os.path.join(ROOT, "tests", "golden", "pt21m.npz")
    if os.path.exists(gpath):
        z = np.load(gpath)
        conv = z["converged"].astype(np.float64)
        errs = []
        for k in range(4):
            win = pt.Render(z["camera"], int(z["width"]), int(z["height"]), 16, int(z["depth"]), seed=900 + k)
            errs.append(float(np.sqrt(np.mean((win.cpu().numpy().astype(np.float64) - conv) ** 2))))
        rmse_info = {"window": "192x108 of the 1920x1080 frame centred on pixel (600, 100)", "spp": 16,
                     "rmse_vs_sort_converged": round(float(np.mean(errs)), 5),
                     "sort_16spp_rmse": round(float(np.mean(z["rmse16"])), 5),
                     "sort_converged_pair_rmse": round(float(z["rmse_converged_pair"]), 5)}
    out = {"metric": "path-traced Msamples/s", "value": round(samples / (ms / 1e3) / 1e6, 3), "unit": "Msamples/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded procedural scene)",
           "config": pt_config({"nodes": args.nodes, "frame_spp_per_s": round(args.steps / (ms / 1e3), 3),
                                "rays_per_sample": round((ext + sh) / samples, 3),
                                "extension_rays": ext, "shadow_rays": sh,
                                "mrays_s": round((ext + sh) / (ms / 1e3) / 1e6, 2)}),
           "e2e": {"value": round(samples / e2e_s / 1e6, 3), "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": int(host_img.numel() * 4 / args.steps)},
           "clocks": clocks.summary(), "image_mean": [round(float(v), 5) for v in host_img.mean(dim=(0, 1))],
           **({"image_rmse": rmse_info} if rmse_info else {}),
           # per sample: generate, flush + per bounce (extend, shade, shadow, resolve, accumulate, count)
           "gpu_launches": args.steps * (2 + 6 * PT_DEPTH) + 2}
    if rank == 0:
        print(json.dumps(out))
    pt.Release()


# batched_31m: 8 resident scenes from the ray-cast recipe at ~10k ... 16M
# triangles, as (icosphere count, subdivision level).
BATCH_SCENES = [(8, 3), (40, 3), (40, 4), (50, 5), (100, 5), (200, 5), (400, 5), (800, 5)]
BATCH_MIN, BATCH_MAX = 4096, 4_194_304


def batched_config(extra=None):
    cfg = {
        "workload": "batched_31m: 8 resident scenes (icosphere fields of 10,242 / 51,202 / 204,802 / 1,024,002 / "
                    "2,048,002 / 4,096,002 / 8,192,002 / 16,384,002 triangles); per step a fixed list of ray "
                    "batches, sizes log-uniform in [4,096, 4,194,304], scene uniform, 50% jittered primary / 50% "
                    "cosine-diffuse bounce rays, closest hit; persistent batch kernel under a captured CUDA graph "
                    "(autotuned) vs one plain launch per batch, same trees, FIFO order",
        "l2": "inputs larger than L2: 2.4 GB of trees, ~1.2 GB of rays per step (no flush)",
    }
    if extra:
        cfg.update(extra)
    return cfg


def run_batched(args):
    """Batched uneven launch: Mrays/s and per-batch latency, persistent graph vs plain launches."""
    import ctypes

    import torch

    from sort_b200 import Batch, Batcher, Obvh, Qbvh, _lib, scenes

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    stream = torch.cuda.current_stream(device)
    rng = np.random.default_rng(args.batch_seed)
    accs, alts, pools, tri_counts = [], [], [], []
    for k, (count, level) in enumerate(BATCH_SCENES):
        tri = scenes.sphere_field(count, level, seed=100 + k)
        a8 = Obvh(DEPTH, LEAF, device=local)
        a8.Build(tri)
        a4 = Qbvh(DEPTH, LEAF, device=local)
        a4.Build(tri)
        cam = scenes.camera_rays(IMAGE, IMAGE, seed=200 + k)
        h = a8.GetIntersect(torch.from_numpy(cam).to(device))
        diffuse, _ = scenes.bounce_rays(tri, cam, h.prim.cpu().numpy(), h.t.cpu().numpy(), IMAGE * IMAGE,
                                        seed=300 + k + rank)
        pools.append((torch.from_numpy(cam).to(device), torch.from_numpy(diffuse).to(device)))
        accs.append(a8)
        alts.append(a4)
        tri_counts.append(int(tri.shape[0]))
    sizes = np.exp(rng.uniform(np.log(BATCH_MIN), np.log(BATCH_MAX), args.batches)).astype(np.int64)
    which = rng.integers(0, len(BATCH_SCENES), args.batches)
    kind = rng.integers(0, 2, args.batches)
    rays = []
    for m, s, kd in zip(sizes, which, kind):
        pool = pools[s][kd]
        a = int(rng.integers(0, pool.shape[1] - m + 1))
        rays.append(pool[:, a:a + m].contiguous())
    del pools
    torch.cuda.empty_cache()
    total = int(sizes.sum())

    # Autotune (tree width per scene, block / stack / refill) on this batch list.
    batcher = Batcher(device=local, max_batches=max(args.batches, 16))
    batches = [Batch(accs[s], r) for s, r in zip(which, rays)]
    tuning, use_alt = batcher.autotune(batches, [alts[s] for s in which], reps=2)
    chosen = {}
    for s, u in zip(which, use_alt):
        chosen[int(s)] = alts[s] if u else accs[s]
    batches = [Batch(chosen[int(s)], r, hits=b.hits) for s, r, b in zip(which, rays, batches)]

    # SORT's traversal counts per batch on the chosen trees -> algorithmic bytes.
    alg_bytes = 0.0
    for b in batches:
        nt, pt = b.accel.TraceStats(b.rays, False)
        alg_bytes += b.rays.shape[1] * (RAY_IN + HIT_OUT) + nt * NODE_BYTES[b.accel.WIDTH] + pt * TRI_BYTES

    # Plain arm: one sg_trace_closest per batch, preallocated outputs, FIFO.
    lib = _lib.load()
    plain_calls = []
    for b in batches:
        r = b.rays
        n = r.shape[1]
        rs = _lib.Rays(*[r.data_ptr() + 4 * k * n for k in range(8)])
        hs = _lib.Hits(b.hits.prim.data_ptr(), b.hits.t.data_ptr(), b.hits.u.data_ptr(), b.hits.v.data_ptr())
        plain_calls.append((b.accel._h, ctypes.byref(rs), n, ctypes.byref(hs), rs, hs))
    sptr = stream.cuda_stream

    def plain_step(events=None):
        for k, (h, rs, n, hs, _, _) in enumerate(plain_calls):
            _lib.check(lib.sg_trace_closest(h, rs, n, hs, sptr))
            if events is not None:
                events[k].record(stream)

    def timed(fn, steps):
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(device)
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        plain_step()
        batcher.run(batches)
    torch.cuda.synchronize(device)
    with ClockSampler(local) as clocks:
        ms_plain = timed(plain_step, args.steps)
        ms_pers = timed(lambda: batcher.run(batches), args.steps)

    # Per-batch latency (completion since the step's start), one step at a time.
    lat_plain, lat_pers, lat_sjf = [], [], []
    order_sjf = sorted(range(len(batches)), key=lambda k: int(batches[k].rays.shape[1]))
    for _ in range(args.steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in batches]
        e0 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        plain_step(ev)
        torch.cuda.synchronize(device)
        lat_plain += [e0.elapsed_time(e) for e in ev]
        batcher.run(batches)
        lat_pers += [d / 1e6 for d in batcher.wait()]
        batcher.run([batches[k] for k in order_sjf])
        lat_sjf += [d / 1e6 for d in batcher.wait()]

    def pct(x, q):
        return round(float(np.percentile(np.asarray(x), q)), 3)

    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = ((float(json.load(open(peaks_path))["hbm_gbs"]), "measured") if os.path.exists(peaks_path)
                      else (6650.0, "fallback"))
    achieved = alg_bytes / (ms_pers / args.steps / 1e3) / 1e9
    value = total * args.steps / (ms_pers / 1e3) / 1e6
    plain_value = total * args.steps / (ms_plain / 1e3) / 1e6
    ngroups = len({(b.accel.WIDTH) for b in batches})
    if rank == 0:
        out = {
            "metric": "Mrays/s batched uneven closest-hit", "value": round(value, 3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_pers / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scenes and rays)",
            "config": batched_config({"batches": args.batches, "batch_seed": args.batch_seed, "rays_per_step": total,
                                      "scene_triangles": tri_counts, "tuning": tuning,
                                      "scene_widths": {str(s): chosen[s].WIDTH for s in sorted(chosen)}}),
            "plain": {"value": round(plain_value, 3), "unit": UNIT, "ms_per_step": round(ms_plain / args.steps, 4),
                      "latency_ms": {"p50": pct(lat_plain, 50), "p99": pct(lat_plain, 99)}},
            "persistent": {"latency_ms": {"p50": pct(lat_pers, 50), "p99": pct(lat_pers, 99)},
                           "shortest_first_latency_ms": {"p50": pct(lat_sjf, 50), "p99": pct(lat_sjf, 99)}},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None,
                         "peak_source": f"{peak_src} hbm_gbs (burst)",
                         "algorithmic_bytes_per_ray": round(alg_bytes / total, 1),
                         "kernel": "k_trace_batches"},
            "clocks": clocks.summary(),
            # per step: the graph's begin kernel + one persistent kernel per width group
            "gpu_launches": args.steps * (1 + ngroups),
        }
        print(json.dumps(out))
    batcher.Release()
    for a in accs + alts:
        a.Release()


# serve_27m: 4 resident path-tracing scenes (~100k, 1M, 5M, 20M triangles) as
# (icosphere count, subdivision level) with per-sphere materials.
SERVE_SCENES = [(20, 4), (50, 5), (245, 5), (1000, 5)]


def serve_config(extra=None):
    cfg = {
        "workload": "serve_27m: 4 resident path-tracing scenes (102,404 / 1,024,004 / 5,017,604 / 20,480,004 "
                    "triangles, per-sphere Lambert / GGX-conductor materials, one area light); render requests "
                    "arrive as a Poisson stream; each picks a scene uniformly, a tile from 64x64 to 1920x1080 "
                    "(log-uniform scale), spp from {1, 4, 16, 64}, depth 5; latency = arrival to image in host "
                    "memory; server (shared path pool + wavefront queues, continuous batching) vs FIFO "
                    "per-request sg_pt_render launches",
        "images": "bit-identical between the two arms (same per-pixel arithmetic and sample order), so equal RMSE",
    }
    if extra:
        cfg.update(extra)
    return cfg


def run_serve(args):
    """Serving: p50/p99 request latency and samples/s, server vs FIFO per-request launches."""
    import queue as queue_mod

    import torch

    from sort_b200 import scenes
    from sort_b200.pathtracer import PathTracer
    from sort_b200.server import RenderServer

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    tracers, tri_counts = [], []
    for k, (count, level) in enumerate(SERVE_SCENES):
        _, _, mats, light, tri, mat = scenes.pt_scene(count, level, seed=1 + k)
        tracers.append(PathTracer(tri, mat, mats, light, device=local))
        tri_counts.append(int(tri.shape[0]))
    rng = np.random.default_rng(args.batch_seed)

    def draw(n):
        s = rng.uniform(0.0, 1.0, n)
        w = np.round(64 * (1920 / 64) ** s).astype(int)
        h = np.round(64 * (1080 / 64) ** s).astype(int)
        spp = rng.choice([1, 4, 16, 64], n)
        sc = rng.integers(0, len(tracers), n)
        return [(int(a), int(b), int(c), int(d), 1000 + i) for i, (a, b, c, d) in enumerate(zip(sc, w, h, spp))]

    reqs = draw(args.requests)
    work = float(sum(w * h * spp for _, w, h, spp, _ in reqs))
    out_imgs = [torch.empty((h, w, 3), dtype=torch.float32).pin_memory() for _, w, h, _, _ in reqs]

    # Warm both arms (buffers at the largest size, graphs captured).
    for t in tracers:
        t.Render(scenes.CAMERA, 1920, 1080, 1, PT_DEPTH, seed=1)
    torch.cuda.synchronize(device)
    srv = RenderServer(device=local, path_slots=args.path_slots, pixel_budget=1 << 24, max_requests=1024,
                       steps_per_poll=args.steps_per_poll, samples_per_claim=args.samples_per_claim,
                       solo_pixels=args.solo_pixels)
    for t in tracers:
        srv.add_scene(t)
    srv.wait(srv.submit(0, scenes.CAMERA, 64, 64, 1))

    def fifo_run(arrivals):
        """One worker renders requests in arrival order (sg_pt_render + copy out)."""
        q = queue_mod.Queue()
        lat = [0.0] * len(reqs)
        t0 = time.perf_counter()

        def worker():
            stream = torch.cuda.current_stream(device)
            for _ in range(len(reqs)):
                i = q.get()
                sc, w, h, spp, seed = reqs[i]
                img = tracers[sc].Render(scenes.CAMERA, w, h, spp, PT_DEPTH, seed=seed)
                out_imgs[i].copy_(img, non_blocking=True)
                stream.synchronize()
                lat[i] = time.perf_counter() - (t0 + arrivals[i])

        th = threading.Thread(target=worker)
        th.start()
        for i, a in enumerate(arrivals):
            d = t0 + a - time.perf_counter()
            if d > 0:
                time.sleep(d)
            q.put(i)
        th.join()
        return lat, time.perf_counter() - t0

    def server_run(arrivals):
        tickets = [0] * len(reqs)
        t0 = time.perf_counter()
        for i, a in enumerate(arrivals):
            d = t0 + a - time.perf_counter()
            if d > 0:
                time.sleep(d)
            sc, w, h, spp, seed = reqs[i]
            tickets[i] = srv.submit(sc, scenes.CAMERA, w, h, spp, PT_DEPTH, seed=seed, image=out_imgs[i].numpy())
        lat = []
        first_submit, last_done = None, 0
        for t in tickets:
            _, res = srv.wait(t)
            lat.append(res["latency_s"])
            first_submit = res["submit_ns"] if first_submit is None else min(first_submit, res["submit_ns"])
            last_done = max(last_done, res["done_ns"])
        return lat, (last_done - first_submit) / 1e9

    def pct(x, q):
        return round(1e3 * float(np.percentile(np.asarray(x), q)), 2)

    # Closed loop (everything arrives at once): capacity of each arm.
    zero = [0.0] * len(reqs)
    with ClockSampler(local) as clocks:
        fifo_lat0, fifo_span0 = fifo_run(zero)
        st0 = srv.stats()
        srv_lat0, srv_span0 = server_run(zero)
        st1 = srv.stats()
        # the server's own kernels in the closed-loop run: per graph replay the admission pair, 8 per
        # bounce step and a continuation trace on the side stream for every step but the last; per
        # solo wave a generate and a flush, 6 per bounce
        spp_ = args.steps_per_poll
        launches0 = ((st1["graph_replays"] - st0["graph_replays"]) * (2 + 8 * spp_ + spp_ - 1)
                     + (st1["solo_waves"] - st0["solo_waves"]) * (2 + 6 * PT_DEPTH))
        fifo_rate = len(reqs) / fifo_span0
        rows = []
        for frac in args.loads:
            lam = frac * fifo_rate
            arr = np.cumsum(rng.exponential(1.0 / lam, len(reqs)))
            arr = (arr - arr[0]).tolist()
            fl, fs = fifo_run(arr)
            sl, ss = server_run(arr)
            rows.append({"load_vs_fifo_capacity": frac, "arrival_rate_req_s": round(lam, 3),
                         "fifo": {"p50_ms": pct(fl, 50), "p99_ms": pct(fl, 99),
                                  "msamples_s": round(work / fs / 1e6, 2)},
                         "server": {"p50_ms": pct(sl, 50), "p99_ms": pct(sl, 99),
                                    "msamples_s": round(work / ss / 1e6, 2)}})
    st = srv.stats()
    srv.close()
    value = work / srv_span0 / 1e6
    if rank == 0:
        out = {
            "metric": "served path-traced Msamples/s", "value": round(value, 3), "unit": "Msamples/s", "n_gpus": 1,
            "steps": len(reqs), "warmup": 1, "ms_per_step": round(1e3 * srv_span0 / len(reqs), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scenes and request stream)",
            "config": serve_config({"requests": len(reqs), "seed": args.batch_seed, "scene_triangles": tri_counts,
                                    "path_slots": args.path_slots, "samples_per_claim": args.samples_per_claim,
                                    "steps_per_poll": args.steps_per_poll,
                                    "solo_pixels": (args.solo_pixels or 1) if args.solo_pixels >= 0 else None,
                                    "samples_per_run": int(work)}),
            "closed_loop": {"server": {"msamples_s": round(value, 2), "p50_ms": pct(srv_lat0, 50),
                                       "p99_ms": pct(srv_lat0, 99)},
                            "fifo": {"msamples_s": round(work / fifo_span0 / 1e6, 2), "p50_ms": pct(fifo_lat0, 50),
                                     "p99_ms": pct(fifo_lat0, 99)}},
            "poisson": rows,
            "server_stats": st,
            "gpu_launches": int(launches0),
            "clocks": clocks.summary(),
        }
        print(json.dumps(out))
    for t in tracers:
        t.Release()


BUILD_SAMPLE = (64, LEVEL)  # SORT's single-threaded build, timed on 64 of the 1,024 spheres (1,310,722 triangles)


def build_config(extra=None, builder="gpu"):
    tree = {"gpu": "GPU builder (SG_BUILDER_GPU), the same tree as SORT's Fbvh::Build",
            "host": "this library's host builder, the same tree as SORT's Fbvh::Build",
            "lbvh": "Morton-order wide BVH built on the GPU (SG_BUILDER_LBVH), not SORT's tree",
            "ploc": "clustered wide BVH built on the GPU (SG_BUILDER_PLOC), not SORT's tree"}[builder]
    cfg = {
        "workload": "build_21m: BVH build of 1,024 level-5 icospheres + ground quad = 20,971,522 triangles, "
                    f"width 8, leaf 8, from host triangles; {tree}",
        "scene_seed": 1,
        "timing": "value: the library's clock around the whole build (triangle upload, GPU passes, and for "
                  "SORT's tree the host flattening); e2e: the create call (build + node upload) from host "
                  "triangles",
        "l2": "inputs larger than L2: 755 MB of triangles per build (no flush)",
    }
    if extra:
        cfg.update(extra)
    return cfg


def sort_build_rate(threads_note=True):
    """SORT's own Accelerator::Build (single-threaded, as SORT builds) on the bounded sample."""
    from sort_b200 import scenes
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        return None
    spheres, level = BUILD_SAMPLE
    tri = scenes.sphere_field(spheres, level, seed=1)
    ref = Reference()
    secs = []
    for _ in range(3):
        tree = ref.build(tri, WIDTH, DEPTH, LEAF)
        secs.append(tree.build_seconds())
        del tree
    rate = tri.shape[0] / statistics.median(secs) / 1e6
    return {"value": round(rate, 3), "unit": "Mtriangles/s", "cores": 1, "kind": "reference",
            "sample": f"{tri.shape[0]} triangles ({spheres} level-{level} icospheres + ground), median of 3 "
                      "SORT Obvh::Build calls"}


def run_build(args):
    """build_21m: GPU builds of the 21M-triangle OBVH, one build per step."""
    import torch

    from sort_b200 import Obvh, _lib, scenes
    from sort_b200.replicas import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        base = sort_build_rate()
        if base is None:
            print(json.dumps({"impl": "reference", "unavailable": "SORT reference library (oracle/_ref) not built"}))
            return
        print(json.dumps({
            "impl": "reference", "metric": "Mtriangles/s BVH build", "value": base["value"],
            "unit": "Mtriangles/s", "n_gpus": args.gpus, "steps": 3, "warmup": 0, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": build_config({"sample": base["sample"]}), "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "Mtriangles/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}, "gpu_launches": 0}))
        return
    import torch.distributed as dist
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=device)
    tri = scenes.sphere_field(SPHERES, LEVEL, seed=1)
    n = tri.shape[0]
    build_s, create_s, info = [], [], None
    with ClockSampler(local) as clocks:
        for k in range(args.warmup + args.steps):
            if world > 1:
                dist.barrier()
            acc = Obvh(max_node_depth=DEPTH, max_pri_in_leaf=LEAF, builder=BUILDERS[args.builder or "gpu"],
                       device=local)
            t0 = time.perf_counter()
            acc.Build(tri)
            t1 = time.perf_counter()
            info = acc.info()
            acc.Release()
            if k >= args.warmup:
                build_s.append(info["build_seconds"])
                create_s.append(t1 - t0)
    mean_build = max_over_ranks(statistics.mean(build_s), device)
    mean_create = max_over_ranks(statistics.mean(create_s), device)
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    tris_bytes = (n + 8) * 48
    node_bytes = info["device_bytes"] - tris_bytes
    lbvh = args.builder in MORTON_TREES
    shapes = info["interior_nodes"] + info["leaves"]
    out = {
        "metric": "Mtriangles/s BVH build", "value": round(world * n / mean_build / 1e6, 3), "unit": "Mtriangles/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * mean_build, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": build_config({"depth": info["depth"], "interior_nodes": info["interior_nodes"],
                                "leaves": info["leaves"], "rounds": info["build_rounds"]}, args.builder or "gpu"),
        "e2e": {"value": round(world * n / mean_create / 1e6, 3), "unit": "Mtriangles/s",
                # the triangles; the host builder's nodes, or the GPU builder's node map (8 B per node)
                "h2d_bytes_per_step": int(n * 36 + (0 if lbvh else node_bytes if (args.builder or "gpu") == "host"
                                                    else 8 * info["interior_nodes"])),
                "d2h_bytes_per_step": int(16 * info["build_rounds"] if lbvh else n * 4 + shapes * 40)},
        "gpu_launches": info["build_launches"] * args.steps,
        "roofline": None,
        **({"tree": MORTON_TREES[args.builder] + ", not SORT's tree (same hits except near-ties "
                    "and box-grazing rays)"} if lbvh else {}),
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = sort_build_rate()
        host = Obvh(max_node_depth=DEPTH, max_pri_in_leaf=LEAF, builder=_lib.SG_BUILDER_HOST, device=local)
        host.Build(tri)
        out["host_builder"] = {"value": round(n / host.info()["build_seconds"] / 1e6, 3), "unit": "Mtriangles/s",
                               "cores": os.cpu_count(), "note": "this library's multithreaded C++ builder"}
        host.Release()
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["closest", "raycast", "pathtrace", "batched", "serve", "build"],
                   default="closest")
    p.add_argument("--requests", type=int, default=120, help="serve workload: requests per run")
    p.add_argument("--path-slots", type=int, default=1 << 21, help="serve workload: server path pool")
    p.add_argument("--samples-per-claim", type=int, default=64,
                   help="serve workload: samples a pool slot renders of one pixel before handing it back")
    p.add_argument("--steps-per-poll", type=int, default=2,
                   help="serve workload: bounce steps per graph replay (even)")
    p.add_argument("--solo-pixels", type=int, default=0,
                   help="serve workload: multi-sample requests this large render in the solo lanes as "
                        "whole-frame waves (0: every one, -1: never)")
    p.add_argument("--loads", type=float, nargs="*", default=[0.5, 0.8, 1.0],
                   help="serve workload: Poisson arrival rates as fractions of the FIFO arm's capacity")
    p.add_argument("--batches", type=int, default=64, help="batched workload: ray batches per step")
    p.add_argument("--batch-seed", type=int, default=7, help="batched workload: seed of the batch list")
    p.add_argument("--sample", type=int, default=CPU_SAMPLE)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--builder", choices=sorted(BUILDERS), default=None,
                   help="tree builder: host/gpu build SORT's tree (closest default host), lbvh / ploc the trees built "
                        "from the Morton order (build workload default gpu)")
    p.add_argument("--nodes", choices=sorted(NODE_FORMATS), default="fp32",
                   help="child-box format of the timed tree (q8: 8-bit, outward-rounded)")
    args = p.parse_args()
    if args.workload == "pathtrace":
        run_pathtrace(args)
    elif args.workload == "build":
        run_build(args)
    elif args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "serve workload: SORT renders one image per "
                              "process; its per-sample CPU rate is the pathtrace workload's reference arm"}))
        else:
            run_serve(args)
    elif args.workload == "batched":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "batched workload: SORT has no batch API; "
                              "its per-ray CPU rate is the closest workload's reference arm"}))
        else:
            run_batched(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
