"""sort_b200: B200-native ray-query engine behind SORT's Accelerator API.

The compute path is libsortgpu.so (C ABI: include/sortgpu.h), built in-tree from
sort_b200/csrc. This package is a thin host-side mirror of SORT's Accelerator
interface over that library (accel.py), plus the seeded synthetic workloads
(scenes.py).
"""
from .accel import SHAPE_DTYPE, Accelerator, Hits, Obvh, Qbvh, Scene, area_shapes, build_topology_host  # noqa: F401
from ._lib import SortGpuError  # noqa: F401
from .batcher import Batch, Batcher  # noqa: F401

__all__ = ["Accelerator", "Qbvh", "Obvh", "Scene", "Hits", "SortGpuError", "build_topology_host", "Batch", "Batcher",
           "SHAPE_DTYPE", "area_shapes"]
