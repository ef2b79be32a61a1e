"""SORT scene streams (sg_stream_*), read on the host; no GPU needed.

tests/golden/scene.sort was written in the layout SORT loads (see
tests/sortstream_writer.py) and tests/golden/stream.npz holds what SORT's own
MeshVisual / HairVisual readers and its Obvh / Qbvh make of the entity
section. The reader must report the configuration, materials, camera and
lights as written, the world-space triangles as Mesh::ApplyTransform computes
them, hair segments as HairVisual derives them, and build SORT's tree over them.
"""
import os

import numpy as np
import pytest

from conftest import renumber_topology, ROOT, golden, same_bits

GOLDEN = os.path.join(ROOT, "tests", "golden", "scene.sort")


def _f32_point(m, p):
    """Matrix::TransformPoint in float32, SORT's order."""
    f = np.float32
    m = m.astype(f)
    out = []
    for r in range(3):
        out.append(((p[:, 0] * m[r, 0] + p[:, 1] * m[r, 1]).astype(f) + (p[:, 2] * m[r, 2]).astype(f) + m[r, 3])
                   .astype(f))
    return np.stack(out, 1)


def test_stream_fields_as_written():
    from sort_b200.stream import SortStream, sid
    s = SortStream(GOLDEN)
    i = s.info
    assert i["integrator"] == sid("PathTracing") and i["max_depth"] == 5 and i["bssrdf_bounces"] == 2
    assert (i["spp"], i["image_width"], i["image_height"]) == (16, 64, 48)
    assert i["accelerator"] == sid("Obvh") and (i["accel_max_depth"], i["accel_max_leaf"]) == (16, 8)
    assert i["triangles"] == 2 * 1280 + 2 and i["lines"] > 0 and i["materials"] == 3
    assert i["area_lights"] == 3 and i["other_lights"] == 2 and i["has_camera"] == 1 and i["volumes"] == 0
    assert s.materials == [("Wood", 0), ("Glass", 1), ("Skin", 2)]
    assert s.camera["eye"] == [0.0, 1.0, 12.0] and s.camera["image_width"] == 64
    a = s.area_lights[0]
    assert a["shape"] == sid("RECTANGLE") and (a["size_x"], a["size_y"]) == (2.0, 1.5) and a["energy"] == 20.0
    assert i["entity_offset"] == int(golden("stream")["entity_offset"])


def test_stream_geometry_is_sorts():
    """World-space triangles as Mesh::ApplyTransform computes them, in SORT's
    primitive order, and SORT's tree over triangles and hair."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden_stream import scene_entities
    from sort_b200 import build_topology_host
    from sort_b200.stream import SortStream
    s = SortStream(GOLDEN)
    ents = scene_entities()
    expect = []
    for e in ents:
        if e[0] == "mesh":
            for verts, tris, _ in e[2]:
                w = _f32_point(e[1], np.asarray(verts, np.float32))
                expect.append(w[np.asarray(tris)].reshape(-1, 9))
    assert same_bits(s.triangles, np.concatenate(expect))
    z = golden("stream")
    n = s.triangles.shape[0] + s.lines.shape[0]
    assert s.order.size == n + 3 and np.array_equal(np.sort(s.order), np.arange(n + 3))
    assert list(s.order[1280 * 2: 1280 * 2 + 1]) == [n]  # the light between the two mesh entities
    sort_index = np.argsort(s.order)  # primitive id -> its place in SORT's primitive order
    for w in (4, 8):
        topo, depth = build_topology_host(s.triangles, w, lines=s.lines, shapes=s.area_shapes, order=s.order)
        assert np.array_equal(renumber_topology(topo, sort_index), z[f"topology{w}"]) and depth == int(z[f"depth{w}"])


def test_stream_light_shapes_are_sorts():
    """Each area light's shape as AreaLightEntity::Serialize leaves it: the
    streamed matrix's inverse (Matrix::Inverse), the scale taken out of both
    (entity/light_entity.cpp:97-106), the shape's sizes; bit for bit against
    the records SORT's own code made for the golden stream."""
    from sort_b200.stream import SortStream
    s = SortStream(GOLDEN)
    assert np.array_equal(s.area_shapes.view(np.uint32).reshape(-1, 35), golden("stream")["light_shapes"].view(np.uint32))


def test_stream_light_shapes_random_transforms(reference, tmp_path):
    """Rotated, scaled and sheared light transforms, every shape kind: our
    stream reader's shapes equal SORT's, computed by SORT's own matrix code."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from sortstream_writer import write_stream
    from sort_b200.stream import SortStream
    rng = np.random.default_rng(81)
    names = ["SQUARE", "RECTANGLE", "DISK"]
    ents = []
    for k in range(24):
        m = np.eye(4, dtype=np.float32)
        m[:3, :3] = rng.normal(size=(3, 3)).astype(np.float32) * np.float32(rng.uniform(0.3, 3.0))
        m[:3, 3] = rng.uniform(-10, 10, 3)
        kind = names[k % 3]
        sizes = (float(rng.uniform(0.00001, 3.0)),) if kind != "RECTANGLE" else tuple(rng.uniform(0.5, 3.0, 2))
        ents.append(("area", m, 1.0, (1.0, 1.0, 1.0), kind, sizes))
    path = tmp_path / "lights.sort"
    write_stream(str(path), materials=[("M", False, False)], entities=ents, accelerator=("Obvh", 16, 8))
    s = SortStream(path)
    for k, a in enumerate(s.area_lights):
        ref = reference.light_shape(a["light2world"], k % 3, a["size_x"], a["size_y"])
        assert np.array_equal(s.area_shapes[k:k + 1].view(np.uint32), ref.view(np.uint32)), k


def test_stream_hair_as_hairvisual_makes_it():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden_stream import scene_entities
    from sort_b200.stream import SortStream
    s = SortStream(GOLDEN)
    hair = [e for e in scene_entities() if e[0] == "hair"][0]
    _, xf, strands, tip, bottom, mat = hair
    f = np.float32
    rows = []
    for pts in strands:
        p = np.asarray(pts, f)
        seg = [np.sqrt(((p[j] - p[j + 1]).astype(f) ** 2).sum(dtype=f)) for j in range(len(p) - 1)]
        total = f(0)
        for x in seg:
            total = f(total + x)
        cur, pv, pw = f(0), f(0), f(bottom)
        for j in range(1, len(p)):
            cur = f(cur + seg[j - 1])
            t = f(cur / total)
            cw = f(f(f(bottom) * f(f(1) - t)) + f(f(tip) * t))
            cv = f(f(f(0) * f(f(1) - t)) + f(f(1) * t))
            rows.append(np.concatenate([p[j - 1], p[j], [pv, cv, pw, cw]]).astype(f))
            pv, pw = cv, cw
    rows = np.array(rows, f)
    world = rows.copy()
    world[:, 0:3] = _f32_point(xf, rows[:, 0:3])
    world[:, 3:6] = _f32_point(xf, rows[:, 3:6])
    assert same_bits(s.lines, world) and (s.line_material == mat).all()


def test_stream_variants_and_errors(tmp_path):
    from sortstream_writer import write_stream
    from sort_b200 import _lib
    from sort_b200.stream import SortStream, sid
    tri = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]]), np.array([0]))
    ent = [("mesh", np.eye(4, dtype=np.float32), [tri]), ("spot", np.eye(4, dtype=np.float32)),
           ("dir", np.eye(4, dtype=np.float32))]
    for integ, key, val in (("AmbientOcclusion", "ao_max_distance", 3.5), ("BidirPathTracing", "mis", 1),
                            ("LightTracing", "mis", 1), ("InstantRadiosity", "ir_paths", 64),
                            ("DirectLight", "max_depth", 5), ("WhittedRT", "max_depth", 5)):
        p = tmp_path / f"{integ}.sort"
        write_stream(p, integrator=integ, materials=[("M", False, False)], entities=ent,
                     accelerator=("KDTree", 20, 4))
        s = SortStream(p)
        assert s.info["integrator"] == sid(integ) and s.info[key] == val
        assert s.info["accelerator"] == sid("KDTree") and s.info["triangles"] == 1 and s.info["other_lights"] == 2
    full = (tmp_path / "WhittedRT.sort").read_bytes()
    (tmp_path / "cut.sort").write_bytes(full[:len(full) // 2])
    with pytest.raises(_lib.SortGpuError) as ex:
        SortStream(tmp_path / "cut.sort")
    assert ex.value.status == 4 and b"stream ends" in _lib.load().sg_last_error()
    with pytest.raises(_lib.SortGpuError) as ex:
        SortStream(tmp_path / "missing.sort")
    assert ex.value.status == 1
    bad = bytearray(full)
    bad[0:4] = (7).to_bytes(4, "little")
    (tmp_path / "version.sort").write_bytes(bytes(bad))
    with pytest.raises(_lib.SortGpuError):
        SortStream(tmp_path / "version.sort")


def test_reference_reads_the_golden_stream(reference):
    """SORT's own readers make the committed answers from scene.sort (pins them)."""
    from sort_b200.stream import SortStream
    z = golden("stream")
    s = SortStream(GOLDEN)
    for w in (4, 8):
        tree = reference.build_from_stream(GOLDEN, s.info["entity_offset"], s.info["triangles"] + s.info["lines"], w)
        prim, t, _, _ = tree.closest(z["rays"])
        assert np.array_equal(prim, z[f"prim{w}"]) and same_bits(t, z[f"t{w}"])
