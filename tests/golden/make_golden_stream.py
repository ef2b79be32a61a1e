"""Generate tests/golden/scene.sort and tests/golden/stream.npz (oracle/_ref).

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden_stream.py

scene.sort is a SORT scene stream written by tests/sortstream_writer.py: a
PathTracing configuration, a material section with a resource, a shader unit
template, a shader group template and three materials, then a camera, two
mesh entities (two transformed icospheres in one, a ground quad in the
other) with a scaled, rotated RECTANGLE area light between them, a hair
entity with its own transform, a DISK area light, a point light, a SQUARE
area light and a sky light, and an Obvh accelerator. stream.npz holds what
SORT does with the entity section: its own MeshVisual / HairVisual Serialize
and ApplyTransform, each area light's shape as AreaLightEntity::Serialize
makes it (entity/light_entity.cpp:97-154), its tree (width 4 and 8) over the
primitives in entity order, and its closest hits and any-hit answers for a
ray set, plus the tree topologies.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle.oracle import Reference  # noqa: E402
from sort_b200 import scenes  # noqa: E402
from sort_b200.stream import SortStream  # noqa: E402
from sortstream_writer import write_stream  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def transform(angle, axis, scale, offset):
    axis = np.asarray(axis, np.float64) / np.linalg.norm(axis)
    c, s = np.cos(angle), np.sin(angle)
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    r = np.eye(3) * c + s * k + (1 - c) * np.outer(axis, axis)
    m = np.eye(4)
    m[:3, :3] = r * scale
    m[:3, 3] = offset
    return m.astype(np.float32)


def scene_entities():
    verts, faces = scenes.icosphere(3)
    rng = np.random.default_rng(61)
    mesh_a = (verts, faces, rng.integers(0, 3, len(faces)))
    mesh_b = (verts * 0.5, faces, rng.integers(-1, 3, len(faces)))
    ground = (np.array([[-20, -3, -20], [20, -3, -20], [20, -3, 20], [-20, -3, 20]], np.float32),
              np.array([[0, 1, 2], [0, 2, 3]]), np.array([1, 1]))
    strands = []
    for _ in range(60):
        root = rng.uniform(-1, 1, 3)
        root /= np.linalg.norm(root)
        pts = [root]
        d = root.copy()
        for _ in range(int(rng.integers(2, 8))):
            d = d + rng.normal(scale=0.3, size=3)
            d /= np.linalg.norm(d)
            pts.append(pts[-1] + 0.25 * d)
        strands.append(np.array(pts, np.float32))
    return [
        ("camera", (0.0, 1.0, 12.0), (0.0, 1.0, 0.0), (0.0, 0.0, 0.0)),
        ("mesh", transform(0.4, (1, 2, 3), 2.0, (-3, 0, 0)), [mesh_a, mesh_b]),
        ("area", transform(2.6, (1, 0.3, 0.2), 1.5, (0, 4, 1)), 20.0, (1.0, 0.95, 0.9), "RECTANGLE", (2.0, 1.5)),
        ("mesh", np.eye(4, dtype=np.float32), [ground]),
        ("hair", transform(-0.7, (0, 1, 1), 2.0, (3, 0.5, 0)), strands, 0.01, 0.04, 2),
        ("area", transform(0.9, (0, 0.2, 1), 1.0, (4, -1, 2)), 10.0, (0.9, 0.9, 1.0), "DISK", (1.2,)),
        ("point", transform(0.0, (1, 0, 0), 1.0, (5, 5, 5))),
        ("area", transform(3.1, (1, 0, 0.1), 0.8, (-4, 5, -2)), 5.0, (1.0, 1.0, 1.0), "SQUARE", (2.5,)),
        ("sky", np.eye(4, dtype=np.float32)),
    ]


def main():
    path = os.path.join(OUT, "scene.sort")
    write_stream(path, materials=[("Wood", False, False), ("Glass", True, False), ("Skin", False, True)],
                 entities=scene_entities(), accelerator=("Obvh", 16, 8))
    s = SortStream(path)
    ntri, nlines, nshapes = s.info["triangles"], s.info["lines"], s.info["area_lights"]
    rng = np.random.default_rng(62)
    m = 3000  # rays aimed at the geometry: hair segment points and triangle centres
    pick = rng.integers(0, nlines, m // 2)
    f = rng.uniform(0.1, 0.9, (m // 2, 1))
    tgt = np.concatenate([s.lines[pick, 0:3] * (1 - f) + s.lines[pick, 3:6] * f,
                          s.triangles[rng.integers(0, ntri, m - m // 2)].reshape(-1, 3, 3).mean(1)])
    o = tgt + rng.normal(size=(m, 3)) * 8.0
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    aimed = np.concatenate([o.T, d.T, np.zeros((1, m)), np.full((1, m), 3.4e38)]).astype(np.float32)
    # rays aimed at points of the area lights' shapes (in their local frames)
    ml = 1500
    k = rng.integers(0, nshapes, ml)
    sh = s.area_shapes
    loc = np.stack([rng.uniform(-0.6, 0.6, ml) * sh["size"][k, 0], np.zeros(ml),
                    rng.uniform(-0.6, 0.6, ml) * np.where(sh["kind"][k] == 1, sh["size"][k, 0], sh["size"][k, 1]),
                    np.ones(ml)], 1)
    tgt = np.einsum("nij,nj->ni", sh["matrix"][k].astype(np.float64).reshape(-1, 4, 4), loc)[:, :3]
    o = tgt + rng.normal(size=(ml, 3)) * 8.0
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    at_lights = np.concatenate([o.T, d.T, np.zeros((1, ml)), np.full((1, ml), 3.4e38)]).astype(np.float32)
    rays = np.ascontiguousarray(np.concatenate([aimed, at_lights, scenes.random_rays(2000, seed=63, box=6.0)],
                                               axis=1))
    ref = Reference()
    from sort_b200.stream import sid
    kinds = {sid("SQUARE"): 0, sid("RECTANGLE"): 1, sid("DISK"): 2}
    light_shapes = np.stack([ref.light_shape(a["light2world"], kinds[a["shape"]], a["size_x"], a["size_y"])
                             for a in s.area_lights])
    out = {"rays": rays, "entity_offset": s.info["entity_offset"], "triangles": ntri, "lines": nlines,
           "shapes": nshapes, "light_shapes": light_shapes}
    for w in (4, 8):
        tree = ref.build_from_stream(path, s.info["entity_offset"], ntri + nlines + nshapes, w)
        prim, t, u, v = tree.closest(rays)
        out.update({f"prim{w}": prim, f"t{w}": t, f"u{w}": u, f"v{w}": v, f"occ{w}": tree.any(rays),
                    f"topology{w}": tree.topology(), f"depth{w}": tree.depth()})
        print(f"width {w}: hits {np.mean(prim >= 0):.3f}, on hair {np.mean((prim >= ntri) & (prim < ntri + nlines)):.3f}"
              f", on lights {np.mean(prim >= ntri + nlines):.3f}")
    np.savez_compressed(os.path.join(OUT, "stream.npz"), **out)
    print(f"{ntri} triangles, {nlines} hair segments, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
