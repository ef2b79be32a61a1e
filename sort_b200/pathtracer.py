"""Python mirror of SORT's PathTracing integrator over libsortgpu.

Mirrors integrator/pathtracing.h (``max_recursive_depth``, ``Li``) for whole
images: ``PathTracer.Render`` runs the wavefront path tracer (sg_pt_render)
over an ``Obvh``/``Qbvh`` built from the same triangles.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .accel import Obvh, Qbvh


class PathTracer:
    def __init__(self, triangles, mat_of_tri, materials, light, width: int = 8, max_node_depth: int = 16,
                 max_pri_in_leaf: int = 8, device: int = 0, node_format: int = _lib.SG_NODES_FP32):
        self.tri = np.ascontiguousarray(np.asarray(triangles, np.float32).reshape(-1, 9))
        self.mat_of_tri = np.ascontiguousarray(np.asarray(mat_of_tri, np.int32))
        self.materials = np.ascontiguousarray(np.asarray(materials, np.float32).reshape(-1, 10))
        self.light = np.ascontiguousarray(np.asarray(light, np.float32))
        if self.mat_of_tri.shape[0] != self.tri.shape[0]:
            raise ValueError("one material index per triangle")
        self.accel = (Qbvh if width == 4 else Obvh)(max_node_depth, max_pri_in_leaf, node_format=node_format,
                                                    device=device)
        self.accel.Build(self.tri)
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.sg_pt_create(self.accel._h, self.tri.ctypes.data, self.tri.shape[0],
                                    self.mat_of_tri.ctypes.data, self.materials.ctypes.data, self.materials.shape[0],
                                    self.light.ctypes.data, ctypes.byref(h)))
        self._h = h
        self.device = device

    def Render(self, camera, width: int, height: int, spp: int, max_recursive_depth: int = 5, seed: int = 1,
               out=None, stream=None, rows=None):
        """Mean radiance per pixel, a float32 CUDA tensor (height, width, 3).
        rows=(begin, end): only those rows of the frame, (end - begin, width, 3),
        each pixel with its random numbers in the whole frame (sg_pt_render_rows)."""
        import torch
        cam = np.ascontiguousarray(np.asarray(camera, np.float32))
        dev = torch.device("cuda", self.device)
        r0, r1 = (0, height) if rows is None else (int(rows[0]), int(rows[1]))
        img = out if out is not None else torch.empty((r1 - r0, width, 3), dtype=torch.float32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        lib = _lib.load()
        if rows is None:
            _lib.check(lib.sg_pt_render(self._h, cam.ctypes.data, width, height, spp, max_recursive_depth, seed,
                                        img.data_ptr(), s))
        else:
            _lib.check(lib.sg_pt_render_rows(self._h, cam.ctypes.data, width, height, r0, r1, spp,
                                             max_recursive_depth, seed, img.data_ptr(), s))
        return img

    def RayCounts(self, stream=None):
        """(extension rays, shadow rays) traced by the last Render (synchronises)."""
        import torch
        a, b = ctypes.c_int64(0), ctypes.c_int64(0)
        s = stream if stream is not None else torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream
        _lib.check(_lib.load().sg_pt_ray_counts(self._h, ctypes.byref(a), ctypes.byref(b), s))
        return a.value, b.value

    def Release(self):
        if getattr(self, "_h", None) is not None:
            _lib.load().sg_pt_destroy(self._h)
            self._h = None
        if getattr(self, "accel", None) is not None:
            self.accel.Release()

    def __del__(self):
        try:
            self.Release()
        except Exception:
            pass
