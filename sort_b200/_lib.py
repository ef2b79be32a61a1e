"""ctypes binding of libsortgpu.so (the C ABI declared in include/sortgpu.h).

The library is built in-tree by ``make -C sort_b200/csrc`` (``__graft_entry__.build``).
Loading fails loudly when it is missing: there is no CPU fallback for any query.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsortgpu.so")

SG_OK = 0
SG_NODES_FP32 = 0
SG_NODES_QUANT8 = 1

SG_ERR_LIMIT = 5
SG_ERR_CANCELLED = 7
STATUS_NAMES = {0: "SG_OK", 1: "SG_ERR_INVALID_ARGUMENT", 2: "SG_ERR_CUDA", 3: "SG_ERR_OUT_OF_MEMORY",
                4: "SG_ERR_UNSUPPORTED", 5: "SG_ERR_LIMIT", 6: "SG_ERR_INTERNAL", 7: "SG_ERR_CANCELLED"}


class SortGpuError(RuntimeError):
    """A libsortgpu call returned a status other than SG_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class BuildOpts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("max_depth", ctypes.c_int32), ("max_leaf", ctypes.c_int32),
                ("node_format", ctypes.c_int32), ("device", ctypes.c_int32), ("build_threads", ctypes.c_int32),
                ("builder", ctypes.c_int32)]


SG_BUILDER_HOST = 0
SG_BUILDER_GPU = 1
SG_BUILDER_LBVH = 2
SG_BUILDER_PLOC = 3


class Rays(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")]


class Hits(ctypes.Structure):
    _fields_ = [("prim", ctypes.c_void_p), ("t", ctypes.c_void_p), ("u", ctypes.c_void_p), ("v", ctypes.c_void_p)]


class Tuning(ctypes.Structure):
    _fields_ = [("schedule", ctypes.c_int32), ("refill_threshold", ctypes.c_int32)]


class SceneInfo(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_int64), ("interior_nodes", ctypes.c_int64), ("leaves", ctypes.c_int64),
                ("depth", ctypes.c_int32), ("width", ctypes.c_int32), ("node_format", ctypes.c_int32),
                ("valid", ctypes.c_int32), ("bbox", ctypes.c_float * 6), ("device_bytes", ctypes.c_int64),
                ("build_seconds", ctypes.c_double), ("build_rounds", ctypes.c_int32),
                ("build_launches", ctypes.c_int32)]


class MultiHits(ctypes.Structure):
    _fields_ = [("count", ctypes.c_void_p), ("prim", ctypes.c_void_p), ("t", ctypes.c_void_p), ("u", ctypes.c_void_p),
                ("v", ctypes.c_void_p)]


class Transparency(ctypes.Structure):
    _fields_ = [("transparent", ctypes.c_int32), ("rgb", ctypes.c_float * 3)]


class StreamInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("version", "threads", "spp", "image_width", "image_height")] + [
        ("clamp", ctypes.c_float), ("integrator", ctypes.c_uint32), ("max_depth", ctypes.c_int32),
        ("bssrdf_bounces", ctypes.c_int32), ("ao_max_distance", ctypes.c_float), ("mis", ctypes.c_int32),
        ("ir_path_sets", ctypes.c_int32), ("ir_paths", ctypes.c_int32), ("ir_min_distance", ctypes.c_float),
        ("triangles", ctypes.c_int64), ("lines", ctypes.c_int64)] + [
        (n, ctypes.c_int32) for n in ("materials", "area_lights", "other_lights", "has_camera", "volumes")] + [
        ("accelerator", ctypes.c_uint32), ("accel_max_depth", ctypes.c_int32), ("accel_max_leaf", ctypes.c_int32),
        ("entity_offset", ctypes.c_int64)]


class StreamCamera(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("up", ctypes.c_float * 3), ("target", ctypes.c_float * 3),
                ("image_width", ctypes.c_int32), ("image_height", ctypes.c_int32), ("lens_radius", ctypes.c_float),
                ("sensor_w", ctypes.c_float), ("sensor_h", ctypes.c_float), ("aspect_fit", ctypes.c_int32),
                ("aspect_ratio_w", ctypes.c_float), ("aspect_ratio_h", ctypes.c_float), ("fov", ctypes.c_float)]


class StreamAreaLight(ctypes.Structure):
    _fields_ = [("light2world", ctypes.c_float * 16), ("energy", ctypes.c_float), ("intensity", ctypes.c_float * 3),
                ("shape", ctypes.c_uint32), ("size_x", ctypes.c_float), ("size_y", ctypes.c_float)]


class Batch(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("rays", ctypes.c_void_p), ("stride", ctypes.c_int64),
                ("n", ctypes.c_int64), ("any", ctypes.c_int32), ("reserved", ctypes.c_int32), ("hits", Hits),
                ("occluded", ctypes.c_void_p)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("block_threads", ctypes.c_int32), ("stack", ctypes.c_int32), ("refill_threshold", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("max_requests", ctypes.c_int32), ("path_slots", ctypes.c_int64),
                ("pixel_budget", ctypes.c_int64), ("steps_per_poll", ctypes.c_int32),
                ("samples_per_claim", ctypes.c_int32), ("solo_pixels", ctypes.c_int64)]


class Request(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_int32), ("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("spp", ctypes.c_int32), ("max_depth", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("seed", ctypes.c_uint64), ("camera", ctypes.c_float * 10), ("image", ctypes.c_void_p)]


class RequestResult(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_int64), ("status", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("submit_ns", ctypes.c_int64), ("admit_ns", ctypes.c_int64), ("done_ns", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int64) for name in ("requests_done", "samples_done", "extension_rays", "shadow_rays",
                                                    "graph_replays", "queued", "admitted", "solo_waves")]


SG_SHAPE_QUAD = 0
SG_SHAPE_DISK = 1


class AreaShape(ctypes.Structure):
    """sg_area_shape: SORT's Quad (size = sizeX, sizeY) or Disk (size[0] = radius)
    with its Transform (matrix and inverse, row-major)."""
    _fields_ = [("kind", ctypes.c_int32), ("size", ctypes.c_float * 2), ("matrix", ctypes.c_float * 16),
                ("inverse", ctypes.c_float * 16)]


class Shapes(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_void_p), ("ntri", ctypes.c_int64), ("lines", ctypes.c_void_p),
                ("nlines", ctypes.c_int64), ("shapes", ctypes.c_void_p), ("nshapes", ctypes.c_int64),
                ("order", ctypes.c_void_p)]


_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_SIGNATURES = {
    "sg_default_server_opts": (None, [ctypes.POINTER(ServerOpts)]),
    "sg_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOpts), ctypes.POINTER(_vp)]),
    "sg_server_add_scene": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_int32)]),
    "sg_server_submit": (ctypes.c_int, [_vp, ctypes.POINTER(Request), ctypes.POINTER(_i64)]),
    "sg_server_wait": (ctypes.c_int, [_vp, _i64, _i64, ctypes.POINTER(RequestResult)]),
    "sg_server_cancel": (ctypes.c_int, [_vp, _i64]),
    "sg_server_stats_get": (ctypes.c_int, [_vp, ctypes.POINTER(ServerStats)]),
    "sg_server_destroy": (ctypes.c_int, [_vp]),
    "sg_batcher_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(_vp)]),
    "sg_batcher_destroy": (ctypes.c_int, [_vp]),
    "sg_batcher_set_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(BatchTuning)]),
    "sg_batcher_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(BatchTuning)]),
    "sg_batcher_run": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _i64, _vp]),
    "sg_batcher_wait": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
    "sg_batcher_autotune": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, _vp,
                                           ctypes.POINTER(BatchTuning), _vp]),
    "sg_default_build_opts": (None, [ctypes.POINTER(BuildOpts)]),
    "sg_scene_create": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(BuildOpts), ctypes.POINTER(_vp)]),
    "sg_scene_create_hair": (ctypes.c_int, [_vp, _i64, _vp, _i64, ctypes.POINTER(BuildOpts), ctypes.POINTER(_vp)]),
    "sg_stream_area_shapes": (ctypes.c_int, [_vp, _vp]),
    "sg_stream_primitive_order": (ctypes.c_int, [_vp, _vp]),
    "sg_scene_create_shapes": (ctypes.c_int, [ctypes.POINTER(Shapes), ctypes.POINTER(BuildOpts), ctypes.POINTER(_vp)]),
    "sg_build_topology_host_shapes": (ctypes.c_int, [ctypes.POINTER(Shapes), ctypes.POINTER(BuildOpts), _vp, _i64,
                                                     ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_int32)]),
    "sg_scene_destroy": (ctypes.c_int, [_vp]),
    "sg_scene_info_get": (ctypes.c_int, [_vp, ctypes.POINTER(SceneInfo)]),
    "sg_scene_topology": (ctypes.c_int, [_vp, _vp, _i64, ctypes.POINTER(_i64)]),
    "sg_build_topology_host": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(BuildOpts), _vp, _i64,
                                              ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_int32)]),
    "sg_stream_open": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_vp)]),
    "sg_stream_info_get": (ctypes.c_int, [_vp, ctypes.POINTER(StreamInfo)]),
    "sg_stream_triangles": (ctypes.c_int, [_vp, _vp, _vp]),
    "sg_stream_lines": (ctypes.c_int, [_vp, _vp, _vp]),
    "sg_stream_camera_get": (ctypes.c_int, [_vp, ctypes.POINTER(StreamCamera)]),
    "sg_stream_area_light_get": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.POINTER(StreamAreaLight)]),
    "sg_stream_material": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_char_p, _i64, ctypes.POINTER(ctypes.c_int32)]),
    "sg_stream_scene_create": (ctypes.c_int, [_vp, ctypes.POINTER(BuildOpts), ctypes.POINTER(_vp)]),
    "sg_stream_close": (ctypes.c_int, [_vp]),
    "sg_build_topology_host_hair": (ctypes.c_int, [_vp, _i64, _vp, _i64, ctypes.POINTER(BuildOpts), _vp, _i64,
                                                   ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_int32)]),
    "sg_scene_set_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(Tuning)]),
    "sg_scene_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(Tuning)]),
    "sg_trace_closest": (ctypes.c_int, [_vp, ctypes.POINTER(Rays), _i64, ctypes.POINTER(Hits), _vp]),
    "sg_trace_any": (ctypes.c_int, [_vp, ctypes.POINTER(Rays), _i64, _vp, _vp]),
    "sg_trace_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Rays), _i64, ctypes.c_int32, ctypes.POINTER(_i64),
                                      ctypes.POINTER(_i64), _vp]),
    "sg_trace_closest_host": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, _vp, _vp]),
    "sg_trace_any_host": (ctypes.c_int, [_vp, _vp, _i64, _vp]),
    "sg_trace_closest_host_static": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "sg_pt_create": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, ctypes.c_int32, _vp, ctypes.POINTER(_vp)]),
    "sg_pt_render": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_uint64, _vp, _vp]),
    "sg_pt_render_rows": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, _vp, _vp]),
    "sg_pt_destroy": (ctypes.c_int, [_vp]),
    "sg_pt_ray_counts": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), _vp]),
    "sg_trace_multi": (ctypes.c_int, [_vp, ctypes.POINTER(Rays), _i64, _vp, _vp, ctypes.POINTER(MultiHits), _vp]),
    "sg_scene_set_materials": (ctypes.c_int, [_vp, _vp, _i64]),
    "sg_trace_multi_host": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sg_trace_attenuation": (ctypes.c_int, [_vp, ctypes.POINTER(Rays), _i64, _vp, ctypes.c_int32, _vp, _vp]),
    "sg_trace_attenuation_host": (ctypes.c_int, [_vp, _vp, _i64, _vp, ctypes.c_int32, _vp]),
    "sg_probe_l2_read_gbs": (ctypes.c_int, [ctypes.c_int32, _i64, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]),
    "sg_last_error": (ctypes.c_char_p, []),
    "sg_version": (ctypes.c_char_p, []),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libsortgpu.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C sort_b200/csrc` "
                           "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != SG_OK:
        msg = load().sg_last_error().decode("utf-8", "replace")
        raise SortGpuError(status, msg)


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)
