"""ctypes loaders for the two CPU oracles (TEST INFRASTRUCTURE ONLY).

* ``Port``      -- the C restatement in oracle/port (built into oracle/_build).
* ``Reference`` -- SORT's own sources compiled with the harness in oracle/ref
                   (built into oracle/_ref; needs the reference tree to build).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use these.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libsortref.so")
# The same harness with SORT's scenes built by the Gbvh adapter over the GPU engine.
REF_GBVH_LIB = os.path.join(HERE, "_ref", "libsortref_gbvh.so")
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64


def build_port() -> str:
    """Compile the restated oracle if needed (gcc only; no reference tree needed)."""
    src = [os.path.join(HERE, "port", f) for f in ("oracle.c", "oracle.h")]
    if not os.path.exists(PORT_LIB) or any(os.path.getmtime(s) > os.path.getmtime(PORT_LIB) for s in src):
        subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
    return PORT_LIB


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


class _Tree:
    def __init__(self, api, handle, width, ntri):
        self.api, self.h, self.width, self.ntri = api, handle, width, ntri

    def __del__(self):
        try:
            self.api._free(self.h)
        except Exception:
            pass

    def topology(self) -> np.ndarray:
        need = self.api._topo(self.h, None, 0)
        need = -need if need < 0 else need
        out = np.empty(max(need, 1), np.int32)
        k = self.api._topo(self.h, out.ctypes.data, out.size)
        return out[:k]

    def depth(self) -> int:
        return int(self.api._depth(self.h))

    def attenuation(self, rays: np.ndarray, threads: int = 0) -> np.ndarray:
        """Scene::GetAttenuation per ray (reference library only): (3, n) rgb."""
        r = np.ascontiguousarray(rays, np.float32)
        n = r.shape[1]
        out = np.empty((3, n), np.float32)
        self.api.L.sortref_trace_attenuation(self.h, r.ctypes.data, n, out.ctypes.data, threads or os.cpu_count())
        return out

    def build_seconds(self) -> float:
        """Duration of SORT's Accelerator::Build for this tree (reference library only)."""
        return float(self.api.L.sortref_build_seconds(self.h))

    def bbox(self) -> np.ndarray:
        b = np.empty(6, np.float32)
        self.api._bbox(self.h, b.ctypes.data)
        return b

    def closest(self, rays: np.ndarray, threads: int = 0):
        r = np.ascontiguousarray(rays, np.float32)
        n = r.shape[1]
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        u = np.empty(n, np.float32)
        v = np.empty(n, np.float32)
        self.api._closest(self.h, r.ctypes.data, n, prim.ctypes.data, t.ctypes.data, u.ctypes.data, v.ctypes.data,
                          threads or os.cpu_count())
        return prim, t, u, v

    def any(self, rays: np.ndarray, threads: int = 0) -> np.ndarray:
        r = np.ascontiguousarray(rays, np.float32)
        n = r.shape[1]
        occ = np.empty(n, np.uint8)
        self.api._any(self.h, r.ctypes.data, n, occ.ctypes.data, threads or os.cpu_count())
        return occ

    def multi(self, rays: np.ndarray, ray_mat: np.ndarray, threads: int = 0):
        """BSSRDF probe query: (count, prim, t, u, v), the last four (n, 4)."""
        r = np.ascontiguousarray(rays, np.float32)
        n = r.shape[1]
        rm = np.ascontiguousarray(ray_mat, np.int32)
        count = np.empty(n, np.int32)
        prim = np.empty((n, 4), np.int32)
        t, u, v = (np.empty((n, 4), np.float32) for _ in range(3))
        self.api._multi(self.h, r.ctypes.data, n, rm.ctypes.data, count.ctypes.data, prim.ctypes.data, t.ctypes.data,
                        u.ctypes.data, v.ctypes.data, threads or os.cpu_count())
        return count, prim, t, u, v


class Port:
    """The C restatement (oracle/port/oracle.c)."""

    def __init__(self):
        L = ctypes.CDLL(build_port())
        L.orc_build.restype = _vp
        L.orc_build.argtypes = [ctypes.c_int, _vp, _i64, ctypes.c_int, ctypes.c_int]
        L.orc_free.argtypes = [_vp]
        L.orc_topology.restype = _i64
        L.orc_topology.argtypes = [_vp, _vp, _i64]
        L.orc_depth.argtypes = [_vp]
        L.orc_scene_bbox.argtypes = [_vp, _vp]
        L.orc_trace_closest.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _vp, ctypes.c_int]
        L.orc_trace_any.argtypes = [_vp, _vp, _i64, _vp, ctypes.c_int]
        L.orc_count.argtypes = [_vp, _vp, _i64, ctypes.c_int, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                ctypes.c_int]
        L.orc_ray_prepare.argtypes = [_vp, _vp, _vp]
        L.orc_tri_test.restype = ctypes.c_int
        L.orc_tri_test.argtypes = [_vp, _i64, _vp, _i64, _i64, ctypes.POINTER(ctypes.c_float)]
        L.orc_fp64_intersect.restype = ctypes.c_double
        L.orc_fp64_intersect.argtypes = [_vp, _i64, _vp, _i64, _i64]
        L.orc_fp64_t_batch.argtypes = [_vp, _vp, _vp, _i64, _vp]
        self.L = L
        self._free, self._topo, self._depth, self._bbox = L.orc_free, L.orc_topology, L.orc_depth, L.orc_scene_bbox
        self._closest, self._any = L.orc_trace_closest, L.orc_trace_any

    def build(self, tri: np.ndarray, width: int, max_depth: int = 16, max_leaf: int = 8) -> _Tree:
        tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        h = self.L.orc_build(width, tri.ctypes.data, tri.shape[0], max_depth, max_leaf)
        if not h:
            raise ValueError("oracle build failed")
        return _Tree(self, h, width, tri.shape[0])

    def count(self, tree: _Tree, rays: np.ndarray, any_hit: bool = False, threads: int = 0):
        r = np.ascontiguousarray(rays, np.float32)
        a, b = _i64(0), _i64(0)
        self.L.orc_count(tree.h, r.ctypes.data, r.shape[1], 1 if any_hit else 0, ctypes.byref(a), ctypes.byref(b),
                         threads or os.cpu_count())
        return a.value, b.value

    def tri_t(self, tri: np.ndarray, prim: int, rays: np.ndarray, i: int):
        """SORT's FP32 watertight test of ray i against one triangle: t or None."""
        tri = np.ascontiguousarray(tri, np.float32)
        r = np.ascontiguousarray(rays, np.float32)
        t = ctypes.c_float(0.0)
        ok = self.L.orc_tri_test(tri.ctypes.data, prim, r.ctypes.data, r.shape[1], i, ctypes.byref(t))
        return t.value if ok else None

    def fp64_t(self, tri: np.ndarray, prim: int, rays: np.ndarray, i: int) -> float:
        tri = np.ascontiguousarray(tri, np.float32)
        r = np.ascontiguousarray(rays, np.float32)
        return float(self.L.orc_fp64_intersect(tri.ctypes.data, prim, r.ctypes.data, r.shape[1], i))

    def fp64_t_batch(self, tri: np.ndarray, prim: np.ndarray, rays: np.ndarray) -> np.ndarray:
        """FP64 re-intersection of every ray with its hit triangle (-1 where prim < 0)."""
        tri = np.ascontiguousarray(tri, np.float32)
        r = np.ascontiguousarray(rays, np.float32)
        p = np.ascontiguousarray(prim, np.int32)
        out = np.empty(r.shape[1], np.float64)
        self.L.orc_fp64_t_batch(tri.ctypes.data, p.ctypes.data, r.ctypes.data, r.shape[1], out.ctypes.data)
        return out

    def fp64_rel_err(self, tri: np.ndarray, prim: np.ndarray, t: np.ndarray, rays: np.ndarray) -> np.ndarray:
        """|t - t_fp64| / t_fp64 per hit ray (hits whose FP64 test misses are left out)."""
        t64 = self.fp64_t_batch(tri, prim, rays)
        ok = (np.asarray(prim) >= 0) & (t64 > 0)
        return np.abs(np.asarray(t, np.float64)[ok] - t64[ok]) / t64[ok]


def _load_reference(adapter: bool):
    path = REF_GBVH_LIB if adapter else REF_LIB
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    L = ctypes.CDLL(path)
    if adapter:
        L.sortref_use_gbvh.argtypes = [ctypes.c_int]
        L.sortref_use_gbvh(1)
    return L


class Reference:
    """SORT's own QBVH/OBVH compiled from its sources (oracle/_ref/libsortref.so).
    adapter=True: the same SORT code with its scenes' accelerator being the
    Gbvh adapter over the GPU engine (oracle/_ref/libsortref_gbvh.so)."""

    def __init__(self, adapter: bool = False):
        L = _load_reference(adapter)
        L.sortref_scene_create.restype = _vp
        L.sortref_scene_create.argtypes = [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.sortref_scene_destroy.argtypes = [_vp]
        L.sortref_topology.restype = _i64
        L.sortref_topology.argtypes = [_vp, _vp, _i64]
        L.sortref_depth.argtypes = [_vp]
        L.sortref_scene_bbox.argtypes = [_vp, _vp]
        L.sortref_trace_closest.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _vp, ctypes.c_int]
        L.sortref_trace_any.argtypes = [_vp, _vp, _i64, _vp, ctypes.c_int]
        L.sortref_ray_prepare.argtypes = [_vp, _vp, _vp]
        L.sortref_scene_create_mat.restype = _vp
        L.sortref_scene_create_mat.argtypes = [ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int]
        L.sortref_trace_multi.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int]
        L.sortref_build_seconds.restype = ctypes.c_double
        L.sortref_build_seconds.argtypes = [_vp]
        L.sortref_scene_create_transparent.restype = _vp
        L.sortref_scene_create_transparent.argtypes = [ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp,
                                                       ctypes.c_int, ctypes.c_int]
        L.sortref_trace_attenuation.argtypes = [_vp, _vp, _i64, _vp, ctypes.c_int]
        L.sortref_scene_from_stream.restype = _vp
        L.sortref_scene_from_stream.argtypes = [ctypes.c_char_p, _i64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.sortref_light_shape.argtypes = [_vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, _vp]
        L.sortref_scene_create_shapes.restype = _vp
        L.sortref_scene_create_shapes.argtypes = [ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                                  ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int]
        L.sortref_scene_create_hair.restype = _vp
        L.sortref_scene_create_hair.argtypes = [ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int]
        self.L = L
        self._free, self._topo, self._depth = L.sortref_scene_destroy, L.sortref_topology, L.sortref_depth
        self._bbox, self._closest, self._any = L.sortref_scene_bbox, L.sortref_trace_closest, L.sortref_trace_any
        self._multi = L.sortref_trace_multi

    def build_materials(self, tri: np.ndarray, mat_of_tri: np.ndarray, nmat: int, width: int, max_depth: int = 16,
                        max_leaf: int = 8) -> _Tree:
        """A tree whose triangles carry materials 0..nmat-1 (for the multi-hit query)."""
        tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        m = np.ascontiguousarray(mat_of_tri, np.int32)
        h = self.L.sortref_scene_create_mat(width, tri.ctypes.data, tri.shape[0], m.ctypes.data, int(nmat),
                                            max_depth, max_leaf)
        if not h:
            raise ValueError("reference build failed")
        return _Tree(self, h, width, tri.shape[0])

    def build_transparent(self, tri: np.ndarray, mat_of_tri: np.ndarray, transparent, rgb, width: int,
                          max_depth: int = 16, max_leaf: int = 8) -> _Tree:
        """A tree whose materials 0..nmat-1 carry a HasTransparency flag and a
        constant transparency (for the transparent-shadow query)."""
        tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        m = np.ascontiguousarray(mat_of_tri, np.int32)
        flags = np.ascontiguousarray(transparent, np.int32).reshape(-1)
        col = np.ascontiguousarray(rgb, np.float32).reshape(-1, 3)
        if col.shape[0] != flags.size:
            raise ValueError("one flag and one rgb triple per material")
        h = self.L.sortref_scene_create_transparent(width, tri.ctypes.data, tri.shape[0], m.ctypes.data, flags.size,
                                                    flags.ctypes.data, col.ctypes.data, max_depth, max_leaf)
        if not h:
            raise ValueError("reference build failed")
        return _Tree(self, h, width, tri.shape[0])

    def build_from_stream(self, path: str, entity_offset: int, ntri: int, width: int, max_depth: int = 16,
                          max_leaf: int = 8) -> _Tree:
        """SORT's own visuals deserialized from a scene stream's entity section, then its tree."""
        h = self.L.sortref_scene_from_stream(str(path).encode(), entity_offset, width, max_depth, max_leaf)
        if not h:
            raise ValueError("reference could not read the stream")
        return _Tree(self, h, width, ntri)

    def build_hair(self, tri: np.ndarray, lines: np.ndarray, width: int, max_depth: int = 16,
                   max_leaf: int = 8) -> _Tree:
        """Triangles followed by hair segments (m, 10): p0, p1, v0, v1, w0, w1."""
        tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        ln = np.ascontiguousarray(lines, np.float32).reshape(-1, 10)
        h = self.L.sortref_scene_create_hair(width, tri.ctypes.data, tri.shape[0], ln.ctypes.data, ln.shape[0],
                                             max_depth, max_leaf)
        if not h:
            raise ValueError("reference build failed")
        return _Tree(self, h, width, tri.shape[0] + ln.shape[0])

    def light_shape(self, light2world, shape: int, a: float, b: float = 0.0) -> np.ndarray:
        """The 35-word shape record SORT makes for an area light (0 SQUARE,
        1 RECTANGLE, 2 DISK) whose streamed transform is light2world (4x4)."""
        m = np.ascontiguousarray(light2world, np.float32).reshape(16)
        out = np.zeros(35, np.float32)
        self.L.sortref_light_shape(m.ctypes.data, int(shape), float(a), float(b), out.ctypes.data)
        return out

    def build_shapes(self, tri: np.ndarray, lines, shapes, order, width: int, max_depth: int = 16,
                     max_leaf: int = 8) -> _Tree:
        """Triangles, hair segments (m, 10) and area shapes (records of 35 words:
        kind, size x, size y, matrix[16], inverse[16]; the layout of
        sort_b200.SHAPE_DTYPE), ids in that order; `order` lists the ids in the
        order SORT's scene presents them (None: increasing)."""
        tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        ln = np.zeros((0, 10), np.float32) if lines is None else np.ascontiguousarray(lines, np.float32).reshape(-1, 10)
        sh = np.zeros(0, np.dtype((np.void, 140))) if shapes is None else np.ascontiguousarray(shapes)
        if sh.dtype.itemsize != 140:
            raise ValueError("area shape records are 140 bytes")
        od = None if order is None else np.ascontiguousarray(order, np.int32)
        h = self.L.sortref_scene_create_shapes(width, tri.ctypes.data, tri.shape[0], ln.ctypes.data, ln.shape[0],
                                               sh.ctypes.data, sh.shape[0], None if od is None else od.ctypes.data,
                                               max_depth, max_leaf)
        if not h:
            raise ValueError("reference build failed")
        return _Tree(self, h, width, tri.shape[0] + ln.shape[0] + sh.shape[0])

    def build(self, tri: np.ndarray, width: int, max_depth: int = 16, max_leaf: int = 8) -> _Tree:
        tri = np.ascontiguousarray(tri, np.float32).reshape(-1, 9)
        h = self.L.sortref_scene_create(width, tri.ctypes.data, tri.shape[0], max_depth, max_leaf)
        if not h:
            raise ValueError("reference build failed")
        return _Tree(self, h, width, tri.shape[0])

    def hardware_threads(self) -> int:
        return int(self.L.sortref_hardware_threads())


class RefPathTracer:
    """SORT's PathTracing::Li over a harness-built scene (oracle/ref/harness_pt.cpp);
    adapter=True: its accelerator is the Gbvh adapter over the GPU engine."""

    def __init__(self, adapter: bool = False):
        L = _load_reference(adapter)
        L.sortref_pt_scene_create.restype = _vp
        L.sortref_pt_scene_create.argtypes = [ctypes.c_int, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp, _vp,
                                              ctypes.c_int, ctypes.c_int]
        L.sortref_pt_scene_destroy.argtypes = [_vp]
        L.sortref_pt_render.argtypes = [_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_uint32, _vp, ctypes.c_int]
        self.L = L
        self.h = None

    def build(self, tri, mat_of_tri, materials, light, width=8, max_depth=16, max_leaf=8):
        self._keep = [np.ascontiguousarray(tri, np.float32).reshape(-1, 9),
                      np.ascontiguousarray(mat_of_tri, np.int32), np.ascontiguousarray(materials, np.float32),
                      np.ascontiguousarray(light, np.float32)]
        t, m, mats, lt = self._keep
        self.h = self.L.sortref_pt_scene_create(width, t.ctypes.data, t.shape[0], m.ctypes.data, mats.shape[0],
                                                mats.ctypes.data, lt.ctypes.data, max_depth, max_leaf)
        if not self.h:
            raise ValueError("reference path-tracing scene build failed")
        return self

    def render(self, camera, width, height, spp, max_depth=5, seed=1, threads=0) -> np.ndarray:
        cam = np.ascontiguousarray(camera, np.float32)
        out = np.zeros((height, width, 3), np.float32)
        self.L.sortref_pt_render(self.h, max_depth, cam.ctypes.data, width, height, spp, seed, out.ctypes.data,
                                 threads or os.cpu_count())
        return out

    def __del__(self):
        if self.h:
            self.L.sortref_pt_scene_destroy(self.h)
