"""Seeded synthetic scenes and ray batches for the ray-query workloads.

SORT ships no scene files or benchmark inputs, so the workloads are procedural:

* ``sphere_field``: unit icospheres (icosahedron, midpoint-subdivided, projected
  to the sphere) with centres U([-10, 10]^3), a uniform random rotation (a
  normalised Gaussian quaternion) and scale U(0.5, 2), the transform baked into
  world-space vertices as SORT's MeshVisual does (entity/visual.cpp:36-38), plus a
  two-triangle ground quad at y = -11.
* ``camera_rays``: a pinhole camera, one jittered ray per pixel.
* ``bounce_rays``: from each primary hit, one cosine-weighted diffuse ray about
  the facing geometric normal (tmin = 1e-4, the secondary-ray offset of
  integrator/pathtracing.cpp:203) and one shadow ray to a uniform point on a
  2 x 2 area light at y = +15 (tmin = 0.01, tmax = length - 0.01 as
  light/area.cpp:49-50 sets them).

Rays are float32 structure-of-arrays blocks of shape (8, n): ox, oy, oz, dx, dy,
dz, tmin, tmax. Triangles are float32 arrays of shape (n, 9): v0, v1, v2.
"""
from __future__ import annotations

import numpy as np

FLT_MAX = np.float32(3.4028234663852886e38)

# Named workload sizes (triangles = spheres * 20 * 4**level + 2).
WORKLOADS = {
    # 64 spheres at level 3: 81,922 triangles; 1024x1024 primary rays; QBVH.
    "raycast_82k": dict(spheres=64, level=3, width=4, image=(1024, 1024)),
    # 1,024 spheres at level 5: 20,971,522 triangles; 2048x2048 primaries feed
    # 4,194,304 diffuse + 4,194,304 shadow rays; OBVH.
    "incoherent_21m": dict(spheres=1024, level=5, width=8, image=(2048, 2048)),
}


def icosphere(level: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: (vertices float64 (V, 3), faces int64 (20 * 4**level, 3))."""
    p = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0),
         (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
         (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
         (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    # wound so that cross(v2 - v0, v1 - v0) (SORT's geometric normal) points outward
    faces = np.array(f, dtype=np.int64)[:, [0, 2, 1]]
    for _ in range(level):
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        edges = np.concatenate([np.stack([a, b], 1), np.stack([b, c], 1), np.stack([c, a], 1)])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mids = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(verts)
        verts = np.concatenate([verts, mids])
        nf = len(faces)
        ab, bc, ca = inv[:nf] + base, inv[nf:2 * nf] + base, inv[2 * nf:] + base
        faces = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1),
                                np.stack([c, ca, bc], 1), np.stack([ab, bc, ca], 1)])
    return verts, faces


def _rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], 1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], 1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], 1),
    ], 1)


def sphere_field(spheres: int, level: int, seed: int = 1, ground_y: float = -11.0,
                 ground_half: float = 60.0, centre_range: float = 10.0) -> np.ndarray:
    """Triangles (spheres * 20 * 4**level + 2, 9) float32; the ground quad is last."""
    rng = np.random.default_rng(seed)
    verts, faces = icosphere(level)
    centres = rng.uniform(-centre_range, centre_range, size=(spheres, 3))
    rots = _rotations(rng, spheres)
    scales = rng.uniform(0.5, 2.0, size=spheres)
    local = verts[faces].reshape(-1, 3)                    # (F * 3, 3)
    tri = np.empty((spheres, local.shape[0], 3), np.float64)
    for s in range(spheres):                               # rotate, scale, translate
        np.matmul(local, rots[s].T * scales[s], out=tri[s])
        tri[s] += centres[s]
    tri = tri.reshape(-1, 9)
    g = ground_half
    # wound so that cross(v2 - v0, v1 - v0) points up (+y)
    ground = np.array([[-g, ground_y, -g, g, ground_y, g, -g, ground_y, g],
                       [-g, ground_y, -g, g, ground_y, -g, g, ground_y, g]], dtype=np.float64)
    return np.ascontiguousarray(np.concatenate([tri, ground]).astype(np.float32))


def camera_rays(width: int, height: int, seed: int = 7, eye=(0.0, 0.0, 30.0), target=(0.0, 0.0, 0.0),
                up=(0.0, 1.0, 0.0), fov_deg: float = 45.0) -> np.ndarray:
    """Pinhole camera, one jittered ray per pixel, row-major from the top row."""
    rng = np.random.default_rng(seed)
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(up, np.float64))
    right /= np.linalg.norm(right)
    upv = np.cross(right, fwd)
    half_h = np.tan(np.radians(fov_deg) * 0.5)
    half_w = half_h * width / height
    jy, jx = rng.random((2, height, width))
    py, px = np.mgrid[0:height, 0:width]
    sx = ((px + jx) / width * 2.0 - 1.0) * half_w
    sy = (1.0 - (py + jy) / height * 2.0) * half_h
    d = fwd[None, None, :] + sx[..., None] * right + sy[..., None] * upv
    d = d.reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    n = width * height
    rays = np.empty((8, n), np.float32)
    rays[0:3] = eye[:, None]
    rays[3:6] = d.T
    rays[6] = 0.0
    rays[7] = FLT_MAX
    return rays


def geometric_normals(tri: np.ndarray, prim: np.ndarray) -> np.ndarray:
    """Unit normal of cross(v2 - v0, v1 - v0) (SORT's gnormal, simd_triangle.h:331)."""
    v = tri[prim].astype(np.float64).reshape(-1, 3, 3)
    n = np.cross(v[:, 2] - v[:, 0], v[:, 1] - v[:, 0])
    return n / np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)


def bounce_rays(tri: np.ndarray, primary: np.ndarray, prim: np.ndarray, t: np.ndarray, count: int,
                seed: int = 11, light_y: float = 15.0, light_half: float = 1.0):
    """Diffuse + shadow ray batches (each (8, count)) spawned from primary hits.

    Primary ray i maps to output i; a primary that missed takes the next hit in
    a seeded shuffled list of hits instead.
    """
    rng = np.random.default_rng(seed)
    hits = np.nonzero(prim >= 0)[0]
    if len(hits) == 0:
        raise ValueError("no primary hits to bounce from")
    src = np.arange(count) % len(prim)
    missed = prim[src] < 0
    pool = rng.permutation(hits)
    src[missed] = pool[np.arange(missed.sum()) % len(pool)]
    o = primary[0:3, src].T.astype(np.float64)
    d = primary[3:6, src].T.astype(np.float64)
    p = o + d * t[src, None].astype(np.float64)
    n = geometric_normals(tri, prim[src])
    flip = np.sum(n * d, axis=1) > 0
    n[flip] = -n[flip]
    # cosine-weighted direction about n
    u1, u2 = rng.random((2, count))
    r = np.sqrt(u1)
    phi = 2.0 * np.pi * u2
    lx, lz, ly = r * np.cos(phi), r * np.sin(phi), np.sqrt(np.maximum(0.0, 1.0 - u1))
    a = np.where(np.abs(n[:, 0:1]) > 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    tx = np.cross(a, n)
    tx /= np.linalg.norm(tx, axis=1, keepdims=True)
    tz = np.cross(n, tx)
    wd = tx * lx[:, None] + n * ly[:, None] + tz * lz[:, None]
    wd /= np.linalg.norm(wd, axis=1, keepdims=True)
    diffuse = np.empty((8, count), np.float32)
    diffuse[0:3] = p.T
    diffuse[3:6] = wd.T
    diffuse[6] = 1e-4
    diffuse[7] = FLT_MAX
    lp = np.stack([rng.uniform(-light_half, light_half, count), np.full(count, light_y),
                   rng.uniform(-light_half, light_half, count)], 1)
    to_l = lp - p
    dist = np.linalg.norm(to_l, axis=1)
    shadow = np.empty((8, count), np.float32)
    shadow[0:3] = p.T
    shadow[3:6] = (to_l / dist[:, None]).T
    shadow[6] = 0.01
    shadow[7] = dist - 0.01
    return diffuse, shadow


def random_rays(n: int, seed: int = 3, box: float = 12.0, axis_fraction: float = 0.1) -> np.ndarray:
    """Rays from random origins in random directions; a fraction have one or two
    exactly-zero direction components (the |d| < 1e-5 clamp of
    simd/simd_ray_utils.h:61-64), some have finite tmax."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(-box, box, (n, 3))
    d = rng.normal(size=(n, 3))
    k = int(n * axis_fraction)
    if k:
        d[:k, 0] = 0.0
        d[k // 2:k, 2] = 0.0
    d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-30)
    rays = np.empty((8, n), np.float32)
    rays[0:3] = o.T
    rays[3:6] = d.T
    rays[6] = 0.0
    rays[7] = np.where(rng.random(n) < 0.3, rng.uniform(0.5, 30.0, n), FLT_MAX)
    return rays


# Conductor Fresnel parameters (eta, k) per RGB channel for the GGX instances.
CONDUCTORS = {
    "gold": ((0.143, 0.374, 1.442), (3.983, 2.385, 1.603)),
    "copper": ((0.200, 0.924, 1.102), (3.912, 2.452, 2.142)),
    "silver": ((0.155, 0.117, 0.138), (4.828, 3.122, 2.147)),
    "aluminium": ((1.657, 0.880, 0.521), (9.224, 6.270, 4.837)),
}

# Material record: 10 floats — type (0 Lambert, 1 GGX conductor reflection),
# Lambert: albedo r g b; GGX: eta r g b, k r g b, roughness.
MAT_FLOATS = 10


def instance_materials(spheres: int, level: int, seed: int = 5):
    """Per-instance materials for a sphere_field scene (same sphere count/level):
    50% Lambert with albedo U(0.2, 0.8) per channel, 50% GGX conductor reflection
    with roughness U(0.05, 0.5) and (eta, k) from CONDUCTORS; the ground is Lambert
    0.5. Returns (mat_of_tri int32 (ntri,), materials float32 (nmat, 10))."""
    rng = np.random.default_rng(seed)
    names = list(CONDUCTORS)
    mats = np.zeros((spheres + 1, MAT_FLOATS), np.float32)
    for s in range(spheres):
        if rng.random() < 0.5:
            mats[s, 0] = 0.0
            mats[s, 1:4] = rng.uniform(0.2, 0.8, 3)
        else:
            eta, k = CONDUCTORS[names[rng.integers(len(names))]]
            mats[s, 0] = 1.0
            mats[s, 1:4] = eta
            mats[s, 4:7] = k
            mats[s, 7] = rng.uniform(0.05, 0.5)
    mats[spheres, 0] = 0.0
    mats[spheres, 1:4] = 0.5
    per_sphere = 20 * 4 ** level
    mat_of_tri = np.concatenate([np.repeat(np.arange(spheres, dtype=np.int32), per_sphere),
                                 np.full(2, spheres, np.int32)])
    return mat_of_tri, mats


# The rectangular area light of the path-traced workloads: centre, size x,
# size z, RGB intensity; it faces -y (SORT's Quad with its +y normal turned down).
AREA_LIGHT = np.array([0.0, 18.0, 0.0, 8.0, 8.0, 40.0, 40.0, 40.0], np.float32)

# Pinhole camera: eye, target, up, vertical field of view (degrees).
CAMERA = np.array([0.0, 0.0, 30.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 45.0], np.float32)


def light_triangles(light: np.ndarray) -> np.ndarray:
    """The area light's rectangle as two triangles whose geometric normal
    cross(v2 - v0, v1 - v0) points down (-y), as its Quad's normal does."""
    cx, cy, cz, sx, sz = (float(v) for v in light[:5])
    hx, hz = sx * 0.5, sz * 0.5
    a = (cx - hx, cy, cz - hz)
    b = (cx + hx, cy, cz - hz)
    c = (cx + hx, cy, cz + hz)
    d = (cx - hx, cy, cz + hz)
    return np.array([[*a, *c, *b], [*a, *d, *c]], np.float32)


def pt_scene(spheres: int, level: int, seed: int = 1, mat_seed: int = 5, light: np.ndarray | None = None):
    """Path-tracing workload: (triangles without the light, materials per triangle,
    material table, light, triangles with the light quad appended, materials per
    triangle with -1 on the light quad). SORT keeps the light's quad as its own
    primitive; the GPU engine traces it as its two triangles."""
    light = AREA_LIGHT if light is None else light
    tri = sphere_field(spheres, level, seed=seed)
    mat_of_tri, mats = instance_materials(spheres, level, seed=mat_seed)
    tri_gpu = np.ascontiguousarray(np.concatenate([tri, light_triangles(light)]))
    mat_gpu = np.concatenate([mat_of_tri, np.array([-1, -1], np.int32)])
    return tri, mat_of_tri, mats, light, tri_gpu, mat_gpu


def hair_strands(strands: int, steps: int = 8, seed: int = 13, box: float = 10.0, length: float = 3.0,
                 width_bottom: float = 0.05, width_tip: float = 0.01) -> np.ndarray:
    """Hair segments (strands * steps, 10) float32: p0 xyz, p1 xyz, v0, v1, w0, w1.

    Each strand grows from a random root in the box with a random bend; its
    segments get widths and v as SORT's HairVisual derives them from the
    cumulative length (entity/visual.cpp:58-94: width from bottom to tip, v
    from 0 to 1, both interpolated by the length fraction)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((strands * steps, 10), np.float32)
    for s in range(strands):
        p = [rng.uniform(-box, box, 3).astype(np.float32)]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        for _ in range(steps):
            d = d + rng.normal(scale=0.35, size=3)
            d /= np.linalg.norm(d)
            p.append((p[-1] + d * (length / steps) * rng.uniform(0.5, 1.5)).astype(np.float32))
        seg = np.array([np.linalg.norm(p[j + 1].astype(np.float64) - p[j]) for j in range(steps)])
        frac = np.concatenate([[0.0], np.cumsum(seg) / seg.sum()])
        w = width_bottom * (1.0 - frac) + width_tip * frac
        for j in range(steps):
            out[s * steps + j] = (*p[j], *p[j + 1], frac[j], frac[j + 1], w[j], w[j + 1])
    return out


def quad_light_shape(light: np.ndarray) -> np.ndarray:
    """The area light (centre xyz, size x, size z, ...) as SORT's Quad: sizeX x
    sizeY in its frame, turned to face -y (the frame's +y axis maps to world
    -y, its z axis to world -z), as the path-tracing harness places it."""
    from .accel import area_shapes
    cx, cy, cz, sx, sz = (float(v) for v in light[:5])
    m = [1.0, 0.0, 0.0, cx, 0.0, -1.0, 0.0, cy, 0.0, 0.0, -1.0, cz, 0.0, 0.0, 0.0, 1.0]
    inv = [1.0, 0.0, 0.0, -cx, 0.0, -1.0, 0.0, cy, 0.0, 0.0, -1.0, cz, 0.0, 0.0, 0.0, 1.0]
    return area_shapes([0], [[sx, sz]], [m], [inv])


def random_area_shapes(n: int, seed: int = 17, box: float = 10.0, size=(0.5, 4.0), disk_fraction: float = 0.4):
    """n area-light shapes (SORT's Quad / Disk) with random sizes, orientations
    (uniform random rotation, no scale, as SORT's light entity removes scale)
    and positions in the box. Matrices are computed in double precision and
    stored as float32; the inverse is the transposed rotation with the
    translation taken back."""
    from .accel import area_shapes
    rng = np.random.default_rng(seed)
    kinds = (rng.uniform(size=n) < disk_fraction).astype(np.int32)
    sizes = rng.uniform(size[0], size[1], (n, 2))
    mats, invs = [], []
    for k in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        t = rng.uniform(-box, box, 3)
        m = np.eye(4)
        m[:3, :3], m[:3, 3] = r, t
        inv = np.eye(4)
        inv[:3, :3], inv[:3, 3] = r.T, -r.T @ t
        mats.append(m)
        invs.append(inv)
    return area_shapes(kinds, sizes, np.array(mats), np.array(invs))
