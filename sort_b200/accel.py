"""Python mirror of SORT's ``Accelerator`` API over libsortgpu.

Mirrors accel/accelerator.h:55-156 and the Qbvh/Obvh classes of
accel/qbvh.h / accel/obvh.h (both ``Fbvh``, accel/fast_bvh.h:101-213):

=====================  ==================================================
SORT                    here
=====================  ==================================================
``Fbvh::Serialize``     ``Serialize(max_node_depth, max_pri_in_leaf)``
``Accelerator::Build``  ``Build(scene)`` (scene = Scene or (n, 9) triangles)
``GetIntersect``        ``GetIntersect(rays)`` -> ``Hits`` (batched)
``GetAttenuation``      ``GetAttenuation(rays)`` -> occluded flags (opaque scenes)
``IsOccluded``          ``IsOccluded(rays)`` (same query)
``GetBBox``             ``GetBBox()``
``GetIsValid``          ``GetIsValid()``
``Clone``               ``Clone()`` (configuration only, like SORT's)
=====================  ==================================================

Rays are a float32 (8, n) structure-of-arrays block (ox, oy, oz, dx, dy, dz,
tmin, tmax): a CUDA tensor runs the device-pointer entry points on the current
stream; a numpy array runs the host-buffer entry points (copies inside the call).
A miss reports prim = -1 and t = FLT_MAX, as SORT leaves SurfaceInteraction::t.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

FLT_MAX = 3.4028234663852886e38


@dataclass
class Hits:
    prim: object  # int32 per ray, -1 on a miss
    t: object     # float32 per ray
    u: object     # barycentric weight of vertex 1
    v: object     # barycentric weight of vertex 2


# sg_area_shape: SORT's Quad (size = sizeX, sizeY) or Disk (size[0] = radius)
# in the x-z plane of its frame, and its Transform (local-to-world matrix and
# its inverse, row-major).
SHAPE_DTYPE = np.dtype([("kind", "<i4"), ("size", "<f4", (2,)), ("matrix", "<f4", (16,)),
                        ("inverse", "<f4", (16,))])


def area_shapes(kind, size, matrix, inverse) -> np.ndarray:
    """An array of area shapes: kind (n,) of SG_SHAPE_QUAD / SG_SHAPE_DISK,
    size (n, 2), matrix and inverse (n, 16) or (n, 4, 4)."""
    kind = np.atleast_1d(np.asarray(kind, np.int32))
    out = np.zeros(kind.shape[0], SHAPE_DTYPE)
    out["kind"] = kind
    out["size"] = np.asarray(size, np.float32).reshape(-1, 2)
    out["matrix"] = np.asarray(matrix, np.float32).reshape(-1, 16)
    out["inverse"] = np.asarray(inverse, np.float32).reshape(-1, 16)
    return out


class Scene:
    """Primitives in SORT's order: a triangle soup, optionally hair line segments
    ((m, 10) float32 rows of p0 xyz, p1 xyz, v0, v1, w0, w1 half widths, world
    space) and area-light shapes (an array of SHAPE_DTYPE). Primitive indices:
    the triangles, then the lines, then the shapes. `order` (optional): every
    primitive index in the order SORT's ScenePrimitiveIterator visits them,
    which decides the tree SORT builds (default: indices in increasing order)."""

    def __init__(self, triangles, lines=None, shapes=None, order=None):
        tri = np.ascontiguousarray(np.asarray(triangles, dtype=np.float32).reshape(-1, 9))
        self.triangles = tri
        self.lines = None if lines is None else np.ascontiguousarray(
            np.asarray(lines, dtype=np.float32).reshape(-1, 10))
        self.shapes = None if shapes is None else np.ascontiguousarray(np.asarray(shapes, SHAPE_DTYPE).reshape(-1))
        self.order = None if order is None else np.ascontiguousarray(np.asarray(order, np.int32).reshape(-1))

    def GetPrimitiveCount(self) -> int:
        return (int(self.triangles.shape[0]) + (0 if self.lines is None else int(self.lines.shape[0])) +
                (0 if self.shapes is None else int(self.shapes.shape[0])))

    def _shapes_struct(self) -> _lib.Shapes:
        s = _lib.Shapes()
        s.triangles, s.ntri = self.triangles.ctypes.data, self.triangles.shape[0]
        if self.lines is not None:
            s.lines, s.nlines = self.lines.ctypes.data, self.lines.shape[0]
        if self.shapes is not None:
            s.shapes, s.nshapes = self.shapes.ctypes.data, self.shapes.shape[0]
        if self.order is not None:
            s.order = self.order.ctypes.data
        return s


def _torch():
    import torch
    return torch


class Accelerator:
    """Wide BVH over one scene, resident on one GPU."""

    WIDTH = 8

    def __init__(self, max_node_depth: int = 16, max_pri_in_leaf: int = 8, node_format: int = _lib.SG_NODES_FP32,
                 device: int = 0, build_threads: int = 0, builder: int = _lib.SG_BUILDER_HOST):
        self.max_node_depth = int(max_node_depth)
        self.max_pri_in_leaf = int(max_pri_in_leaf)
        self.node_format = int(node_format)
        self.device = int(device)
        self.build_threads = int(build_threads)
        self.builder = int(builder)  # SG_BUILDER_HOST or SG_BUILDER_GPU: the same tree either way
        self._h = None
        self._info = None

    # -- configuration ------------------------------------------------------------
    def Serialize(self, max_node_depth: int, max_pri_in_leaf: int) -> None:
        """Fbvh::Serialize reads m_maxNodeDepth then m_maxPriInLeaf."""
        self.max_node_depth = int(max_node_depth)
        self.max_pri_in_leaf = int(max_pri_in_leaf)

    def Clone(self) -> "Accelerator":
        return type(self)(self.max_node_depth, self.max_pri_in_leaf, self.node_format, self.device,
                          self.build_threads)

    def _opts(self) -> _lib.BuildOpts:
        o = _lib.BuildOpts()
        o.width = self.WIDTH
        o.max_depth = self.max_node_depth
        o.max_leaf = self.max_pri_in_leaf
        o.node_format = self.node_format
        o.device = self.device
        o.build_threads = self.build_threads
        o.builder = self.builder
        return o

    # -- build ----------------------------------------------------------------------
    def Build(self, scene) -> None:
        sc = scene if isinstance(scene, Scene) else Scene(scene)
        tri = sc.triangles
        self.Release()
        lib = _lib.load()
        h = ctypes.c_void_p()
        if sc.shapes is not None or sc.order is not None:
            _lib.check(lib.sg_scene_create_shapes(ctypes.byref(sc._shapes_struct()), ctypes.byref(self._opts()),
                                                  ctypes.byref(h)))
        elif sc.lines is None:
            _lib.check(lib.sg_scene_create(tri.ctypes.data, tri.shape[0], ctypes.byref(self._opts()),
                                           ctypes.byref(h)))
        else:
            _lib.check(lib.sg_scene_create_hair(tri.ctypes.data, tri.shape[0], sc.lines.ctypes.data,
                                                sc.lines.shape[0], ctypes.byref(self._opts()), ctypes.byref(h)))
        self._h = h
        info = _lib.SceneInfo()
        _lib.check(lib.sg_scene_info_get(h, ctypes.byref(info)))
        self._info = info

    def Release(self) -> None:
        if self._h is not None:
            _lib.load().sg_scene_destroy(self._h)
            self._h = None
            self._info = None

    def __del__(self):
        try:
            self.Release()
        except Exception:
            pass

    # -- queries --------------------------------------------------------------------
    def _require(self):
        if self._h is None:
            raise RuntimeError("Build() has not been called")

    @staticmethod
    def _ray_struct(rays):
        base = rays.data_ptr()
        n = rays.shape[1]
        r = _lib.Rays()
        for k, name in enumerate(("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")):
            setattr(r, name, base + 4 * k * n)
        return r

    def GetIntersect(self, rays, stream=None, out: Hits | None = None) -> Hits:
        """Closest hit per ray. With host (numpy) rays, ``out`` may supply the four
        result arrays (e.g. views of pinned memory) to fill in place."""
        self._require()
        lib = _lib.load()
        if isinstance(rays, np.ndarray):
            r = np.ascontiguousarray(rays, dtype=np.float32)
            n = r.shape[1]
            if out is not None:
                prim, t, u, v = out.prim, out.t, out.u, out.v
                for a, dt in ((prim, np.int32), (t, np.float32), (u, np.float32), (v, np.float32)):
                    if a.dtype != dt or a.shape != (n,) or not a.flags.c_contiguous:
                        raise ValueError("out arrays must be contiguous, length n, int32/float32")
            else:
                prim = np.empty(n, np.int32)
                t = np.empty(n, np.float32)
                u = np.empty(n, np.float32)
                v = np.empty(n, np.float32)
            _lib.check(lib.sg_trace_closest_host(self._h, r.ctypes.data, n, prim.ctypes.data, t.ctypes.data,
                                                 u.ctypes.data, v.ctypes.data))
            return Hits(prim, t, u, v)
        torch = _torch()
        rays = rays.contiguous()
        if rays.dtype != torch.float32 or rays.dim() != 2 or rays.shape[0] != 8 or not rays.is_cuda:
            raise ValueError("rays must be a float32 CUDA tensor of shape (8, n)")
        n = rays.shape[1]
        dev = rays.device
        prim = torch.empty(n, dtype=torch.int32, device=dev)
        t = torch.empty(n, dtype=torch.float32, device=dev)
        u = torch.empty(n, dtype=torch.float32, device=dev)
        v = torch.empty(n, dtype=torch.float32, device=dev)
        h = _lib.Hits(prim.data_ptr(), t.data_ptr(), u.data_ptr(), v.data_ptr())
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.sg_trace_closest(self._h, ctypes.byref(self._ray_struct(rays)), n, ctypes.byref(h), s))
        return Hits(prim, t, u, v)

    def GetAttenuation(self, rays, stream=None):
        """Occlusion flags (1 = an opaque primitive lies in (tmin, tmax])."""
        self._require()
        lib = _lib.load()
        if isinstance(rays, np.ndarray):
            r = np.ascontiguousarray(rays, dtype=np.float32)
            n = r.shape[1]
            occ = np.empty(n, np.uint8)
            _lib.check(lib.sg_trace_any_host(self._h, r.ctypes.data, n, occ.ctypes.data))
            return occ
        torch = _torch()
        rays = rays.contiguous()
        if rays.dtype != torch.float32 or rays.dim() != 2 or rays.shape[0] != 8 or not rays.is_cuda:
            raise ValueError("rays must be a float32 CUDA tensor of shape (8, n)")
        n = rays.shape[1]
        occ = torch.empty(n, dtype=torch.uint8, device=rays.device)
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        _lib.check(lib.sg_trace_any(self._h, ctypes.byref(self._ray_struct(rays)), n, occ.data_ptr(), s))
        return occ

    IsOccluded = GetAttenuation

    def GetIntersectBSSRDF(self, rays, prim_material, ray_material, stream=None):
        """SORT's BSSRDF probe query, GetIntersect(ray, BSSRDFIntersections&, rc,
        matID) (accel/fast_bvh.hpp:656-819), for a CUDA ray batch: up to 4 hits
        per ray on primitives whose material (prim_material, int32 per
        primitive) equals the ray's (ray_material, int32 per ray). Returns
        (count, prim, t, u, v); the last four have shape (n, 4), in SORT's slots."""
        self._require()
        torch = _torch()
        rays = rays.contiguous()
        n = rays.shape[1]
        dev = rays.device
        pm = torch.as_tensor(prim_material, dtype=torch.int32, device=dev).contiguous()
        rm = torch.as_tensor(ray_material, dtype=torch.int32, device=dev).contiguous()
        if pm.numel() != self._info.triangles or rm.numel() != n:
            raise ValueError("one material per primitive and one per ray")
        count = torch.empty(n, dtype=torch.int32, device=dev)
        prim = torch.empty((n, 4), dtype=torch.int32, device=dev)
        t, u, v = (torch.empty((n, 4), dtype=torch.float32, device=dev) for _ in range(3))
        h = _lib.MultiHits(count.data_ptr(), prim.data_ptr(), t.data_ptr(), u.data_ptr(), v.data_ptr())
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.load().sg_trace_multi(self._h, ctypes.byref(self._ray_struct(rays)), n, pm.data_ptr(),
                                              rm.data_ptr(), ctypes.byref(h), s))
        return count, prim, t, u, v

    def SetMaterials(self, prim_material) -> None:
        """The material id of every primitive (int32, input order), kept on the
        device for the queries that depend on materials."""
        self._require()
        m = np.ascontiguousarray(np.asarray(prim_material, dtype=np.int32).reshape(-1))
        _lib.check(_lib.load().sg_scene_set_materials(self._h, m.ctypes.data, m.size))

    @staticmethod
    def transparency_table(transparent, rgb) -> np.ndarray:
        """The sg_transparency array for per-material flags and rgb triples."""
        flags = np.asarray(transparent, dtype=np.int32).reshape(-1)
        col = np.asarray(rgb, dtype=np.float32).reshape(-1, 3)
        if col.shape[0] != flags.size:
            raise ValueError("one transparency flag and one rgb triple per material")
        table = np.zeros(flags.size, dtype=[("transparent", np.int32), ("rgb", np.float32, 3)])
        table["transparent"] = flags
        table["rgb"] = col
        return table

    def GetAttenuationTransparent(self, rays, transparent, rgb, stream=None):
        """SORT's Scene::GetAttenuation (core/scene.cpp:192-208) with transparent
        materials, for a CUDA ray batch: per material a HasTransparency flag and a
        constant EvaluateTransparency rgb; primitive materials from SetMaterials.
        Returns a (3, n) float32 tensor (r, g, b rows)."""
        self._require()
        torch = _torch()
        rays = rays.contiguous()
        n = rays.shape[1]
        dev = rays.device
        table = self.transparency_table(transparent, rgb)
        d_table = torch.from_numpy(table.view(np.uint8).copy()).to(dev)
        out = torch.empty((3, n), dtype=torch.float32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.load().sg_trace_attenuation(self._h, ctypes.byref(self._ray_struct(rays)), n,
                                                    d_table.data_ptr(), table.size, out.data_ptr(), s))
        return out

    def TraceStats(self, rays, any_hit: bool = False, stream=None):
        """(interior nodes tested, primitives tested) summed over a CUDA ray batch,
        counted as SORT's traversal statistics count them."""
        self._require()
        torch = _torch()
        rays = rays.contiguous()
        a, b = ctypes.c_int64(0), ctypes.c_int64(0)
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        _lib.check(_lib.load().sg_trace_stats(self._h, ctypes.byref(self._ray_struct(rays)), rays.shape[1],
                                              1 if any_hit else 0, ctypes.byref(a), ctypes.byref(b), s))
        return a.value, b.value

    # -- launch schedule (results never depend on it) ------------------------------
    def SetTuning(self, schedule: int | None = None, refill_threshold: int | None = None) -> None:
        self._require()
        lib = _lib.load()
        t = _lib.Tuning()
        _lib.check(lib.sg_scene_get_tuning(self._h, ctypes.byref(t)))
        if schedule is not None:
            t.schedule = int(schedule)
        if refill_threshold is not None:
            t.refill_threshold = int(refill_threshold)
        _lib.check(lib.sg_scene_set_tuning(self._h, ctypes.byref(t)))

    def GetTuning(self) -> dict:
        self._require()
        t = _lib.Tuning()
        _lib.check(_lib.load().sg_scene_get_tuning(self._h, ctypes.byref(t)))
        return {"schedule": t.schedule, "refill_threshold": t.refill_threshold}

    # -- introspection ------------------------------------------------------------
    def GetBBox(self):
        self._require()
        return tuple(self._info.bbox)

    def GetIsValid(self) -> bool:
        return self._h is not None and bool(self._info.valid)

    def info(self) -> dict:
        self._require()
        i = self._info
        return dict(triangles=i.triangles, interior_nodes=i.interior_nodes, leaves=i.leaves, depth=i.depth,
                    width=i.width, node_format=i.node_format, valid=bool(i.valid), bbox=tuple(i.bbox),
                    device_bytes=i.device_bytes, build_seconds=i.build_seconds,
                    build_rounds=i.build_rounds, build_launches=i.build_launches)

    def topology(self) -> np.ndarray:
        self._require()
        lib = _lib.load()
        need = ctypes.c_int64(0)
        lib.sg_scene_topology(self._h, None, 0, ctypes.byref(need))
        out = np.empty(max(need.value, 1), np.int32)
        _lib.check(lib.sg_scene_topology(self._h, out.ctypes.data, out.size, ctypes.byref(need)))
        return out[:need.value]


class Qbvh(Accelerator):
    """SORT's QBVH: 4-wide."""
    WIDTH = 4


class Obvh(Accelerator):
    """SORT's OBVH: 8-wide."""
    WIDTH = 8


def build_topology_host(triangles, width: int, max_depth: int = 16, max_leaf: int = 8, threads: int = 0,
                        lines=None, shapes=None, order=None):
    """Build on the host only and return (topology stream, depth); needs no GPU.
    With hair segments (lines, (m, 10)) and area shapes, they follow the
    triangles, as in Scene; `order` as in Scene."""
    lib = _lib.load()
    sc = Scene(triangles, lines, shapes, order) if (shapes is not None or order is not None) else None
    tri = np.ascontiguousarray(np.asarray(triangles, np.float32).reshape(-1, 9))
    ln = None if lines is None else np.ascontiguousarray(np.asarray(lines, np.float32).reshape(-1, 10))
    o = _lib.BuildOpts()
    lib.sg_default_build_opts(ctypes.byref(o))
    o.width, o.max_depth, o.max_leaf, o.build_threads = width, max_depth, max_leaf, threads
    need = ctypes.c_int64(0)
    depth = ctypes.c_int32(0)

    def call(out, cap):
        if sc is not None:
            return lib.sg_build_topology_host_shapes(ctypes.byref(sc._shapes_struct()), ctypes.byref(o), out, cap,
                                                     ctypes.byref(need), ctypes.byref(depth))
        if ln is None:
            return lib.sg_build_topology_host(tri.ctypes.data, tri.shape[0], ctypes.byref(o), out, cap,
                                              ctypes.byref(need), ctypes.byref(depth))
        return lib.sg_build_topology_host_hair(tri.ctypes.data, tri.shape[0], ln.ctypes.data, ln.shape[0],
                                               ctypes.byref(o), out, cap, ctypes.byref(need), ctypes.byref(depth))

    st = call(None, 0)
    if st not in (_lib.SG_OK, 5):
        _lib.check(st)
    out = np.empty(max(need.value, 1), np.int32)
    _lib.check(call(out.ctypes.data, out.size))
    return out[:need.value], depth.value
