"""SORT's binary scene stream, read through libsortgpu (sg_stream_* in include/sortgpu.h).

    s = SortStream("scene.sort")
    s.info["integrator"] == sid("PathTracing"); s.triangles; s.lines; s.camera
    acc = s.accelerator()          # the stream's Qbvh/Obvh (its depth and leaf size), built
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def sid(name: str) -> int:
    """SORT's StringID of a class name (core/strid.h:40-65)."""
    crc = 0
    for ch in name.encode("ascii"):
        crc ^= ch
        for _ in range(8):
            crc = (crc >> 1) ^ (-(crc & 1) & 0xEDB88320)
    return (~crc) & 0xFFFFFFFF


class SortStream:
    def __init__(self, path: str):
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.sg_stream_open(str(path).encode(), ctypes.byref(h)))
        self._h = h
        info = _lib.StreamInfo()
        _lib.check(lib.sg_stream_info_get(h, ctypes.byref(info)))
        self.info = {name: getattr(info, name) for name, _ in _lib.StreamInfo._fields_}
        nt, nl = info.triangles, info.lines
        self.triangles = np.empty((nt, 9), np.float32)
        self.tri_material = np.empty(nt, np.int32)
        _lib.check(lib.sg_stream_triangles(h, self.triangles.ctypes.data, self.tri_material.ctypes.data))
        self.lines = np.empty((nl, 10), np.float32)
        self.line_material = np.empty(nl, np.int32)
        _lib.check(lib.sg_stream_lines(h, self.lines.ctypes.data, self.line_material.ctypes.data))
        self.camera = None
        if info.has_camera:
            c = _lib.StreamCamera()
            _lib.check(lib.sg_stream_camera_get(h, ctypes.byref(c)))
            self.camera = {name: (list(getattr(c, name)) if name in ("eye", "up", "target") else getattr(c, name))
                           for name, _ in _lib.StreamCamera._fields_}
        self.area_lights = []
        for k in range(info.area_lights):
            a = _lib.StreamAreaLight()
            _lib.check(lib.sg_stream_area_light_get(h, k, ctypes.byref(a)))
            self.area_lights.append({"light2world": np.array(a.light2world, np.float32).reshape(4, 4),
                                     "energy": a.energy, "intensity": list(a.intensity), "shape": a.shape,
                                     "size_x": a.size_x, "size_y": a.size_y})
        from .accel import SHAPE_DTYPE
        self.area_shapes = np.zeros(info.area_lights, SHAPE_DTYPE)
        if info.area_lights:
            _lib.check(lib.sg_stream_area_shapes(h, self.area_shapes.ctypes.data))
        # primitive indices (triangles, segments, shapes) in the order SORT's scene visits them
        self.order = np.empty(nt + nl + info.area_lights, np.int32)
        if self.order.size:
            _lib.check(lib.sg_stream_primitive_order(h, self.order.ctypes.data))
        self.materials = []
        for k in range(info.materials):
            buf = ctypes.create_string_buffer(4096)
            flags = ctypes.c_int32(0)
            _lib.check(lib.sg_stream_material(h, k, buf, len(buf), ctypes.byref(flags)))
            self.materials.append((buf.value.decode(), flags.value))

    def scene(self):
        """The geometry as an accel.Scene: triangles, hair segments in world space,
        area lights' shapes (in that order; accelerator() builds in the order the
        stream's entities present them)."""
        from .accel import Scene
        return Scene(self.triangles, self.lines if len(self.lines) else None,
                     self.area_shapes if len(self.area_shapes) else None)

    def accelerator(self, builder: int = _lib.SG_BUILDER_HOST, device: int = 0, node_format: int = 0,
                    width: int | None = None):
        """The stream's accelerator built over its scene (sg_stream_scene_create): Obvh/Qbvh with the
        stream's depth and leaf size; any other class becomes SORT's fallback, a QBVH (width overrides
        the class). Hair segments keep their entity's transform exactly as SORT's Line::SetTransform
        applies it."""
        from .accel import Obvh, Qbvh
        obvh = self.info["accelerator"] == sid("Obvh") if width is None else width == 8
        if self.info["accelerator"] in (sid("Obvh"), sid("Qbvh")):
            depth, leaf = self.info["accel_max_depth"], self.info["accel_max_leaf"]
        else:
            depth, leaf = 16, 8
        acc = (Obvh if obvh else Qbvh)(depth, leaf, node_format=node_format, device=device, builder=builder)
        acc.Release()
        h = ctypes.c_void_p()
        _lib.check(_lib.load().sg_stream_scene_create(self._h, ctypes.byref(acc._opts()), ctypes.byref(h)))
        acc._h = h
        info = _lib.SceneInfo()
        _lib.check(_lib.load().sg_scene_info_get(h, ctypes.byref(info)))
        acc._info = info
        return acc

    def close(self):
        if self._h is not None:
            _lib.load().sg_stream_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
