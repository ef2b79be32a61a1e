"""Writes SORT binary scene streams for the ingest tests (test infrastructure).

Follows the byte layout SORT's loader reads and its Blender exporter writes
(blender-plugin/addons/sortblend/exporter.py: export_global_config 416-445,
export_materials 726-930, export_scene 227-410, mesh 560-586, hair 590-647):
4-byte scalars, 1-byte bools, NUL-terminated strings, StringIDs as SORT's
32-bit class-name hashes. No SORT scene file ships with the reference, so the
tests make their own.
"""
from __future__ import annotations

import struct

import numpy as np

from sort_b200.stream import sid


class Writer:
    def __init__(self):
        self.b = bytearray()

    def u32(self, v):
        self.b += struct.pack("<I", int(v) & 0xFFFFFFFF)

    def i32(self, v):
        self.b += struct.pack("<i", int(v))

    def f32(self, v):
        self.b += struct.pack("<f", float(v))

    def flag(self, v):
        self.b += struct.pack("<?", bool(v))

    def string(self, s):
        self.b += s.encode("ascii") + b"\0"

    def sid(self, name):
        self.u32(sid(name))

    def matrix(self, m):
        for x in np.asarray(m, np.float32).reshape(16):
            self.f32(x)


def _graph(w, units, connections):
    w.u32(len(units))
    for name, typ, params in units:
        w.string(name)
        w.string(typ)
        w.u32(len(params))
        for pname, value in params:
            w.string(pname)
            if isinstance(value, str):
                w.i32(4)
                w.string(value)
            elif np.ndim(value) == 0:
                w.i32(1)
                w.f32(value)
            else:
                w.i32(3)
                for x in value:
                    w.f32(x)
    w.u32(len(connections))
    for c in connections:
        for s in c:
            w.string(s)


def write_stream(path, *, integrator="PathTracing", max_depth=5, spp=16, size=(64, 48), clamp=0.0,
                 materials=(), entities=(), accelerator=("Obvh", 16, 8)):
    """materials: (name, transparent, sss) tuples; entities: tuples of
    ("camera", eye, up, target), ("mesh", xf16, [(verts (n,3), tris (m,3), mats (m,))...]),
    ("hair", xf16, strands [(k,3) points...], width_tip, width_bottom, mat),
    ("area", xf16, energy, rgb, shape, sizes), ("point"|"dir"|"spot"|"sky", xf16)."""
    w = Writer()
    # global configuration (loadConfig)
    w.i32(0)
    w.string("")
    w.i32(0)
    w.i32(spp)
    w.i32(size[0])
    w.i32(size[1])
    w.f32(clamp)
    w.sid(integrator)
    w.i32(max_depth)
    if integrator == "PathTracing":
        w.i32(2)
    elif integrator == "AmbientOcclusion":
        w.f32(3.5)
    elif integrator in ("BidirPathTracing", "LightTracing"):
        w.flag(True)
    elif integrator == "InstantRadiosity":
        w.i32(4)
        w.i32(64)
        w.f32(0.25)
    # material section: one resource, a shader unit and group template, then the materials
    w.u32(1)
    w.string("textures/wood.png")
    w.sid("Texture2D")
    w.sid("ShaderUnitTemplate")
    w.string("SORTNode_Material_Diffuse")
    w.string("shader diffuse(color base = color(1.0), out closure bxdf){ bxdf = lambert(base); }")
    w.u32(1)
    w.string("tex")
    w.string("textures/wood.png")
    w.sid("ShaderGroupTemplate")
    w.string("Group_0")
    _graph(w, [("a", "SORTNode_Material_Diffuse", [("base", (0.5, 0.25, 1.0)), ("rough", 0.3)])],
           [("a", "bxdf", "out", "bxdf")])
    w.string("a")
    w.u32(1)
    w.string("bxdf")
    w.string("group_input")
    w.u32(2)
    w.string("x")
    w.string("y")
    for name, transparent, sss in materials:
        w.sid("Material")
        w.string(name)
        w.sid("Surface Shader")
        _graph(w, [("n0", "SORTNode_Material_Diffuse", [("base", (0.8, 0.8, 0.8)), ("map", "tex")]),
                   ("n1", "SORTNode_Output", [])], [("n0", "bxdf", "n1", "Surface")])
        w.sid("Invalid Volume Shader")
        w.flag(transparent)
        w.flag(sss)
        w.f32(0.1)
        w.u32(32)
    w.sid("End of Material")
    # entities
    w.sid("verification bits")
    for e in entities:
        kind = e[0]
        if kind == "camera":
            w.sid("PerspectiveCameraEntity")
            for v in (e[1], e[2], e[3]):
                for x in v:
                    w.f32(x)
            w.u32(size[0])
            w.u32(size[1])
            w.f32(0.0)
            w.f32(36.0)
            w.f32(24.0)
            w.i32(0)
            w.f32(1.0)
            w.f32(1.0)
            w.f32(0.69)
        elif kind == "mesh":
            w.sid("VisualEntity")
            w.matrix(e[1])
            w.u32(len(e[2]))
            for verts, tris, mats in e[2]:
                w.sid("MeshVisual")
                w.flag(True)
                w.i32(len(verts))
                for v in np.asarray(verts, np.float32):
                    for x in (*v, 0.0, 1.0, 0.0, 0.5, 0.5):
                        w.f32(x)
                w.i32(len(tris))
                for t, m in zip(np.asarray(tris), np.asarray(mats)):
                    for x in (*t, m):
                        w.i32(x)
                w.sid("no_volume")
                w.sid("end of mesh")
        elif kind == "hair":
            _, xf, strands, tip, bottom, mat = e
            w.sid("VisualEntity")
            w.matrix(xf)
            w.u32(1)
            w.sid("HairVisual")
            w.u32(len(strands))
            w.f32(tip)
            w.f32(bottom)
            w.i32(mat)
            for pts in strands:
                w.u32(len(pts) - 1)
                for p in np.asarray(pts, np.float32):
                    for x in p:
                        w.f32(x)
        elif kind == "area":
            _, xf, energy, rgb, shape, sizes = e
            w.sid("AreaLightEntity")
            w.matrix(xf)
            w.f32(energy)
            for x in rgb:
                w.f32(x)
            w.sid(shape)
            for x in sizes:
                w.f32(x)
        elif kind in ("point", "dir", "spot"):
            w.sid({"point": "PointLightEntity", "dir": "DirLightEntity", "spot": "SpotLightEntity"}[kind])
            w.matrix(e[1])
            w.f32(10.0)
            for x in (1.0, 0.9, 0.8):
                w.f32(x)
            if kind == "spot":
                w.f32(0.9)
                w.f32(0.1)
        elif kind == "sky":
            w.sid("SkyLightEntity")
            w.matrix(e[1])
            w.f32(1.0)
            for x in (0.2, 0.3, 0.4):
                w.f32(x)
            w.string("")
        else:
            raise ValueError(kind)
    w.sid("End of Entities")
    name, depth, leaf = accelerator
    w.sid(name)
    if name in ("Qbvh", "Obvh", "Bvh", "KDTree", "OcTree"):
        w.i32(depth)
        w.i32(leaf)
    with open(path, "wb") as f:
        f.write(bytes(w.b))
    return len(w.b)
