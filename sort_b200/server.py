"""Render server over libsortgpu's sg_server: resident path-tracing scenes,
requests of uneven sizes admitted by pixel budget and rendered concurrently in
shared wavefront queues (continuous batching).

Each request's image is bit-identical to ``PathTracer.Render`` of the same
request (same scene, camera, size, samples, depth and seed), alone or in any
mix of other requests. SORT has no counterpart: it renders one image per
process (work/image_evaluation/image_evaluation.cpp:120-305).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _pinned(shape):
    """A page-locked float32 host array (falls back to pageable memory without torch)."""
    try:
        import torch
        return torch.empty(shape, dtype=torch.float32).pin_memory().numpy()
    except Exception:
        return np.empty(shape, np.float32)


class RenderServer:
    def __init__(self, device: int = 0, path_slots: int = 1 << 20, pixel_budget: int = 1 << 24,
                 max_requests: int = 1024, steps_per_poll: int = 4, samples_per_claim: int = 1,
                 solo_pixels: int = 0):
        """solo_pixels: multi-sample requests of at least this many pixels
        render in the solo lanes as whole-frame waves (0: every one, < 0:
        never); the pool renders the rest."""
        o = _lib.ServerOpts()
        _lib.load().sg_default_server_opts(ctypes.byref(o))
        o.device, o.path_slots, o.pixel_budget = int(device), int(path_slots), int(pixel_budget)
        o.max_requests, o.steps_per_poll = int(max_requests), int(steps_per_poll)
        o.samples_per_claim = int(samples_per_claim)
        o.solo_pixels = int(solo_pixels)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().sg_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._scenes = []   # keep the PathTracer objects alive
        self._images = {}   # ticket -> host image

    def add_scene(self, pathtracer) -> int:
        """Makes a PathTracer's scene resident in the server; returns its id."""
        sid = ctypes.c_int32(0)
        _lib.check(_lib.load().sg_server_add_scene(self._h, pathtracer._h, ctypes.byref(sid)))
        self._scenes.append(pathtracer)
        return sid.value

    def submit(self, scene: int, camera, width: int, height: int, spp: int, max_depth: int = 5,
               seed: int = 1, image: np.ndarray | None = None) -> int:
        """Queues a render; returns its ticket."""
        img = image if image is not None else _pinned((height, width, 3))
        if img.dtype != np.float32 or img.shape != (height, width, 3) or not img.flags.c_contiguous:
            raise ValueError("image must be a contiguous float32 (height, width, 3) array")
        q = _lib.Request()
        q.scene, q.width, q.height, q.spp, q.max_depth = int(scene), int(width), int(height), int(spp), int(max_depth)
        q.seed = int(seed)
        for k, v in enumerate(np.asarray(camera, np.float32).reshape(10)):
            q.camera[k] = float(v)
        q.image = img.ctypes.data
        t = ctypes.c_int64(0)
        _lib.check(_lib.load().sg_server_submit(self._h, ctypes.byref(q), ctypes.byref(t)))
        self._images[t.value] = img
        return t.value

    def wait(self, ticket: int, timeout: float | None = None):
        """Blocks until the ticket completes; returns (image, result dict). A
        cancelled request returns (None, result) with status SG_ERR_CANCELLED."""
        r = _lib.RequestResult()
        ns = -1 if timeout is None else int(timeout * 1e9)
        _lib.check(_lib.load().sg_server_wait(self._h, int(ticket), ns, ctypes.byref(r)))
        img = self._images.pop(int(ticket), None)
        res = {"ticket": r.ticket, "status": r.status, "submit_ns": r.submit_ns, "admit_ns": r.admit_ns,
               "done_ns": r.done_ns, "latency_s": (r.done_ns - r.submit_ns) / 1e9}
        return (img if r.status == _lib.SG_OK else None), res

    def cancel(self, ticket: int) -> None:
        _lib.check(_lib.load().sg_server_cancel(self._h, int(ticket)))

    def stats(self) -> dict:
        s = _lib.ServerStats()
        _lib.check(_lib.load().sg_server_stats_get(self._h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in _lib.ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            _lib.check(_lib.load().sg_server_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
