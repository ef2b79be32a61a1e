"""Batched multi-scene traversal over libsortgpu's sg_batcher.

Many ray batches, over many resident scenes (``Accelerator`` objects on one
GPU) and of uneven sizes, are traced by one replay of a captured CUDA graph:
one persistent kernel per group of batches that share a tree width, node
format and query drains all of them. Each batch's results are exactly what
``GetIntersect`` / ``GetAttenuation`` return for it alone.

SORT has no such API; it stands in for SORT's render workers, each calling
``Accelerator::GetIntersect`` on its own rays
(work/image_evaluation/image_evaluation.cpp:70-75, 153-279).

Rays: a float32 CUDA tensor of shape (8, n) whose rows are ox, oy, oz, dx, dy,
dz, tmin, tmax; a column slice ``pool[:, a:b]`` of a larger block is accepted
as is (the row stride is passed to the kernel).
"""
from __future__ import annotations

import ctypes
import json
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .accel import Hits


@dataclass
class Batch:
    accel: object            # a built Accelerator (Qbvh / Obvh) on the batcher's device
    rays: object             # float32 CUDA tensor (8, n), unit stride along n
    any: bool = False        # False: closest hit into ``hits``; True: occlusion into ``occluded``
    hits: Hits | None = None
    occluded: object = None
    _keep: list = field(default_factory=list, repr=False)


def _torch():
    import torch
    return torch


class Batcher:
    """Runs lists of ``Batch`` on one GPU through sg_batcher."""

    def __init__(self, device: int = 0, max_batches: int = 4096):
        self.device = int(device)
        self.max_batches = int(max_batches)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().sg_batcher_create(self.device, self.max_batches, ctypes.byref(h)))
        self._h = h
        self._last = None
        self.budget_cut = False

    def Release(self) -> None:
        if self._h:
            _lib.check(_lib.load().sg_batcher_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.Release()
        except Exception:
            pass

    # -- tuning ---------------------------------------------------------------------
    @property
    def tuning(self) -> dict:
        t = _lib.BatchTuning()
        _lib.check(_lib.load().sg_batcher_get_tuning(self._h, ctypes.byref(t)))
        return {"block_threads": t.block_threads, "stack": t.stack, "refill_threshold": t.refill_threshold,
                "blocks_per_sm": t.blocks_per_sm}

    @tuning.setter
    def tuning(self, value: dict) -> None:
        cur = self.tuning
        cur.update(value)
        t = _lib.BatchTuning(cur["block_threads"], cur["stack"], cur["refill_threshold"], cur["blocks_per_sm"])
        _lib.check(_lib.load().sg_batcher_set_tuning(self._h, ctypes.byref(t)))

    # -- runs -----------------------------------------------------------------------
    def _table(self, batches: list[Batch]):
        torch = _torch()
        n = len(batches)
        arr = (_lib.Batch * max(n, 1))()
        for k, b in enumerate(batches):
            r = b.rays
            if r.dtype != torch.float32 or r.dim() != 2 or r.shape[0] != 8 or not r.is_cuda:
                raise ValueError(f"batch {k}: rays must be a float32 CUDA tensor of shape (8, n)")
            if r.shape[1] > 1 and r.stride(1) != 1:
                raise ValueError(f"batch {k}: rays must have unit stride along n")
            m = int(r.shape[1])
            dev = r.device
            if b.any:
                if b.occluded is None:
                    b.occluded = torch.empty(m, dtype=torch.uint8, device=dev)
                hits = _lib.Hits()
                occ = b.occluded.data_ptr()
            else:
                if b.hits is None:
                    b.hits = Hits(torch.empty(m, dtype=torch.int32, device=dev),
                                  torch.empty(m, dtype=torch.float32, device=dev),
                                  torch.empty(m, dtype=torch.float32, device=dev),
                                  torch.empty(m, dtype=torch.float32, device=dev))
                hits = _lib.Hits(b.hits.prim.data_ptr(), b.hits.t.data_ptr(), b.hits.u.data_ptr(),
                                 b.hits.v.data_ptr())
                occ = None
            b.accel._require()
            arr[k] = _lib.Batch(b.accel._h.value, r.data_ptr() if m else None, int(r.stride(0)) if m else 0, m,
                                1 if b.any else 0, 0, hits, occ)
        return arr

    def _stream(self, stream):
        if stream is not None:
            return stream
        torch = _torch()
        return torch.cuda.current_stream(torch.device("cuda", self.device)).cuda_stream

    def run(self, batches: list[Batch], budget_ns: int = 0, stream=None) -> list[Batch]:
        """Enqueues one run of every batch (no synchronisation); fills each
        batch's ``hits`` / ``occluded`` (allocated here when absent)."""
        arr = self._table(batches)
        _lib.check(_lib.load().sg_batcher_run(self._h, ctypes.cast(arr, ctypes.c_void_p), len(batches),
                                              int(budget_ns), self._stream(stream)))
        self._last = (arr, list(batches))
        return batches

    def wait(self, stream=None) -> np.ndarray:
        """Synchronises; per batch of the last run, ns from the run's start to its
        last ray, -1 where a time budget left it incomplete (``budget_cut``)."""
        if self._last is None:
            raise RuntimeError("no run to wait for")
        n = len(self._last[1])
        done = np.empty(max(n, 1), np.int64)
        st = _lib.load().sg_batcher_wait(self._h, done.ctypes.data, n, self._stream(stream))
        self.budget_cut = st == 5
        if st not in (_lib.SG_OK, 5):
            _lib.check(st)
        return done[:n]

    def autotune(self, batches: list[Batch], alternatives: list | None = None, reps: int = 3, stream=None,
                 cache: str | None = None):
        """Times runs of ``batches`` to pick the tree width per scene (from
        ``alternatives``: per batch the same scene built at the other width, or
        None) and the kernel tuning, which is installed. Returns (tuning,
        use_alternative per batch). With ``cache`` (a JSON file), a result for
        the same device, scenes and batch sizes is reused without timing."""
        key = None
        if cache:
            torch = _torch()
            sig = [(b.accel.info()["triangles"], b.accel.WIDTH, int(b.rays.shape[1]), bool(b.any),
                    None if not alternatives or alternatives[k] is None else alternatives[k].WIDTH)
                   for k, b in enumerate(batches)]
            key = json.dumps([torch.cuda.get_device_name(self.device), sig])
            if os.path.exists(cache):
                with open(cache) as f:
                    db = json.load(f)
                if key in db:
                    self.tuning = db[key]["tuning"]
                    return self.tuning, list(db[key]["use_alternative"])
        arr = self._table(batches)
        n = len(batches)
        alt_arr = None
        use = np.zeros(max(n, 1), np.int32)
        if alternatives is not None:
            if len(alternatives) != n:
                raise ValueError("one alternative (or None) per batch")
            alt_arr = (ctypes.c_void_p * n)(*[a._h.value if a is not None else None for a in alternatives])
        best = _lib.BatchTuning()
        _lib.check(_lib.load().sg_batcher_autotune(self._h, ctypes.cast(arr, ctypes.c_void_p),
                                                   ctypes.cast(alt_arr, ctypes.c_void_p) if alt_arr else None, n,
                                                   int(reps), use.ctypes.data, ctypes.byref(best),
                                                   self._stream(stream)))
        tuning = self.tuning
        use_alt = [int(x) for x in use[:n]]
        if cache:
            db = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    db = json.load(f)
            db[key] = {"tuning": tuning, "use_alternative": use_alt}
            with open(cache, "w") as f:
                json.dump(db, f, indent=1)
        return tuning, use_alt
