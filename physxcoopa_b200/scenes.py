"""Seeded synthetic workloads for the cloth benchmark configurations.

No public dataset exists for this path; every scene is generated from a seed with the sizes and
value distributions of the benchmark configurations:

  single_drape   one 32x32 sheet, 0.05 m spacing, +-1 mm jitter, two top corners pinned (with
                 geodesic tethers), sphere r = 0.3 m 0.5 m below the centre; compliance 0
                 (structural) / 1e-6 (shear) / 1e-4 (bending); 4 substeps x 10 iterations.
  uniform_batch  N sheets of side 64 (default 1024), same constraint types and compliances;
                 per sheet from the seed: pin pattern (2 corners, 4 corners or the full top
                 edge) and one sphere, radius U(0.2, 0.5) m, centre 0.5 m below the sheet
                 centre offset by U(-0.3, 0.3) m per axis.
  uneven_batch   N sheets (default 4096), side U{16..128}, 1-3 colliders each drawn from sphere
                 / capsule (r U(0.1, 0.3), half-length U(0.2, 0.6)) / oriented box (half-extents
                 U(0.1, 0.5)); half the sheets get one point gravity source (9.81, radius 1 m,
                 range 10 m).

Parameters the configurations leave open keep the reference's ClothParams defaults
(physxcoopa/cloth/cloth.h:171-255): damping 0.05, aero drag / lift 0.02, thickness 0.03,
friction 0.5, tether_scale 1.02, max_velocity 100. Sleep plays no part (the solver is stepped
unconditionally). Sheets are horizontal (identity orientation), 1 kg each, rest lengths captured
after the jitter so a sheet starts unstrained.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _abi as A
from .arrays import (ClothArrays, HeightGrid, Hull, Mesh, box, capsule, collider_array, gravity_sources, hull_collider,
                     mesh_collider, sphere)

SPACING = 0.05
STRUCTURAL, SHEAR, BEND = 0.0, 1e-6, 1e-4


@dataclass
class ClothScene:
    name: str
    cloths: List[ClothArrays]
    colliders: List[np.ndarray]
    sources: Optional[List[np.ndarray]] = None
    gravity: tuple = (0.0, 0.0, -9.81)
    substeps: int = 4
    iterations: int = 10
    h: float = 1.0 / 60.0
    meta: dict = field(default_factory=dict)
    # Collider geometry (arrays.Hull / arrays.Mesh); colliders name geometry k by id k + 1, the
    # ids a fresh context hands out when they are registered in this order.
    geometries: list = field(default_factory=list)

    @property
    def vertices(self):
        return sum(len(c.particles) for c in self.cloths)


def cloth_params(**kw):
    p = A.ClothParams.defaults()
    p.stretch_compliance = STRUCTURAL
    p.bend_compliance = BEND
    p.has_shear_compliance = 1
    p.shear_compliance = SHEAR
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def reference_params():
    """The configurations' compliances as the reference's ClothParams can hold them: one stretch
    compliance for the structural and the shear constraints (0), bend 1e-4. The per-batch shear
    compliance of cloth_params() has no counterpart in the reference solver."""
    return cloth_params(has_shear_compliance=0, shear_compliance=0.0)


def grid_desc(side, center, seed, params=None):
    """The pxb_grid_cloth_desc of a benchmark sheet: side x side particles at SPACING, +-1 mm
    jitter from `seed`, 1 kg, shear on."""
    width = (side - 1) * SPACING
    d = A.GridClothDesc()
    d.columns, d.rows, d.width, d.height = side, side, width, width
    d.center = (A.C.c_float * 3)(*[float(v) for v in center])
    d.orientation = (A.C.c_float * 4)(0.0, 0.0, 0.0, 1.0)
    d.total_mass = 1.0
    d.shear = 1
    d.params = params if params is not None else cloth_params()
    d.jitter = 1e-3
    d.jitter_seed = seed
    return d


def _sheet(side, center, seed, pins, params=None, tethers=True):
    from .runtime import HostCloth
    width = (side - 1) * SPACING
    h = HostCloth(side, side, width, width, center=center, params=params or cloth_params(),
                  jitter=1e-3, seed=seed)
    for point, radius in pins:
        h.pin_static(point, radius)
    if tethers and pins:
        h.build_tethers()
    return h.arrays()


def _corner_pins(side, center, pattern):
    half = (side - 1) * SPACING * 0.5
    cx, cy, cz = center
    r = 0.3 * SPACING  # smaller than the spacing: exactly the chosen particle despite the jitter
    top = [((cx - half, cy + half, cz), r), ((cx + half, cy + half, cz), r)]
    if pattern == 0:
        return top
    if pattern == 1:
        return top + [((cx - half, cy - half, cz), r), ((cx + half, cy - half, cz), r)]
    return [((cx - half + k * SPACING, cy + half, cz), r) for k in range(side)]


@dataclass
class SheetSpec:
    """One sheet of a batch as drawn from the batch's seed, before any builder runs."""
    side: int
    center: tuple
    seed: int
    pins: list
    colliders: np.ndarray
    source: Optional[np.ndarray]


def build_sheet(spec, params=None):
    """A planned sheet built by the library's builders (jitter, pins, tethers when pinned)."""
    return _sheet(spec.side, spec.center, spec.seed, spec.pins, params)


def single_drape_name():
    return "single_drape 32x32"


def single_drape_plan(seed=0):
    """The one sheet of the single drape: 32 x 32, two top corners pinned, a sphere of r 0.3 m
    0.5 m below its centre."""
    center = (0.0, 0.0, 1.0)
    return [SheetSpec(32, center, seed, _corner_pins(32, center, 0),
                      collider_array([sphere(0.3, (0.0, 0.0, 0.5))]), None)]


def single_drape(seed=0, params=None):
    s = single_drape_plan(seed)[0]
    return ClothScene(single_drape_name(), [build_sheet(s, params)], [s.colliders], meta={"side": 32})


def uniform_name(n, side):
    return f"uniform_batch {n}x{side}^2"


def uniform_plan(n=1024, side=64, seed=1):
    """The draws of the uniform batch, sheet by sheet: pin pattern, then one sphere."""
    rng = np.random.default_rng(seed)
    center = (0.0, 0.0, 1.0)
    specs = []
    for k in range(n):
        pattern = int(rng.integers(0, 3))
        r = float(rng.uniform(0.2, 0.5))
        off = rng.uniform(-0.3, 0.3, 3)
        col = collider_array([sphere(r, (center[0] + off[0], center[1] + off[1], center[2] - 0.5 + off[2]))])
        specs.append(SheetSpec(side, center, seed * 100003 + k, _corner_pins(side, center, pattern), col, None))
    return specs


def uniform_batch(n=1024, side=64, seed=1, params=None):
    specs = uniform_plan(n, side, seed)
    return ClothScene(uniform_name(n, side), [build_sheet(s, params) for s in specs], [s.colliders for s in specs],
                      meta={"side": side, "n": n})


def _random_quat(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    return tuple(float(v) for v in q.astype(np.float32))


def uneven_plan(n=4096, lo=16, hi=128, seed=2, max_side=None):
    """The draws of the uneven batch, sheet by sheet (side, pins, colliders, gravity source), in
    the order uneven_batch consumes them: the first k specs of a batch of n are the batch of k."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n):
        side = int(rng.integers(lo, hi + 1))
        if max_side is not None:
            side = min(side, max_side)
        center = (0.0, 0.0, 1.0)
        pattern = int(rng.integers(0, 3))
        pins = _corner_pins(side, center, pattern)
        recs = []
        for _ in range(int(rng.integers(1, 4))):
            kind = int(rng.integers(0, 3))
            off = rng.uniform(-0.3, 0.3, 3)
            pos = (float(off[0]), float(off[1]), 0.5 + float(off[2]))
            if kind == 0:
                recs.append(sphere(float(rng.uniform(0.2, 0.5)), pos))
            elif kind == 1:
                recs.append(capsule(float(rng.uniform(0.1, 0.3)), float(rng.uniform(0.2, 0.6)), pos,
                                    _random_quat(rng)))
            else:
                recs.append(box(tuple(float(v) for v in rng.uniform(0.1, 0.5, 3)), pos,
                                _random_quat(rng)))
        src = None
        if k % 2 == 0:
            src = gravity_sources([((float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2)), -3.0),
                                    9.81, 1.0, 10.0)])
        specs.append(SheetSpec(side, center, seed * 100003 + k, pins, collider_array(recs), src))
    return specs


def uneven_name(n, lo=16, hi=128):
    return f"uneven_batch {n} sides U{{{lo}..{hi}}}"


def uneven_batch(n=4096, lo=16, hi=128, seed=2, max_side=None, params=None, first=None):
    """The uneven batch built by the library's builders. `first` builds only the first sheets of
    the batch (a sample with the batch's own draws); `params` replaces cloth_params()."""
    specs = uneven_plan(n, lo, hi, seed, max_side)
    if first is not None:
        specs = specs[:first]
    cloths = [build_sheet(s, params) for s in specs]
    return ClothScene(uneven_name(n, lo, hi), cloths, [s.colliders for s in specs],
                      sources=[s.source for s in specs], meta={"n": n, "lo": lo, "hi": hi})


@dataclass
class StrandScene:
    name: str
    sets: list
    colliders: List[np.ndarray]
    root_path: object = None  # callable(frame) -> (positions (n, 3), orientations or None)
    gravity: tuple = (0.0, 0.0, -9.81)
    substeps: int = 4
    iterations: int = 20
    h: float = 1.0 / 60.0
    meta: dict = field(default_factory=dict)
    # Collider geometry (arrays.Hull / arrays.Mesh); colliders name geometry k by id k + 1, the
    # ids a fresh context hands out when they are registered in this order.
    geometries: list = field(default_factory=list)

    @property
    def particles(self):
        return sum(len(s.particles) for s in self.sets)


def hair_groom(n_strands=65536, count=32, segment=0.01, seed=3, iterations=20):
    """65,536 strands of 32 particles, 1 cm segments, rooted on a sphere of radius 0.1 m (seeded
    directions) and growing outward; one sphere collider (the head) rides with the roots, whose
    centre follows a seeded 0.2 m, 1 Hz sinusoid. Stretch plus the reference's global and local
    shape constraints (its strand "bending"), reference StrandParams defaults otherwise."""
    from .runtime import make_strands
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n_strands, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d[:, 2] = np.abs(d[:, 2])  # upper hemisphere
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    head_r = 0.1
    roots = (d * head_r).astype(np.float32)
    k = np.arange(count, dtype=np.float32)[None, :, None]
    pts = (roots[:, None, :] + d[:, None, :] * (segment * k)).astype(np.float32)
    s = make_strands(list(pts))
    phase = float(rng.uniform(0, 2 * np.pi))
    amp_dir = rng.normal(size=3).astype(np.float32)
    amp_dir /= np.linalg.norm(amp_dir)

    def centre(frame, h=1.0 / 60.0):
        return (0.2 * np.sin(2 * np.pi * 1.0 * frame * h + phase) * amp_dir).astype(np.float32)

    def root_path(frame):
        return (roots + centre(frame)[None, :]).astype(np.float32), None

    def colliders(frame):
        return collider_array([sphere(head_r * 0.95, tuple(centre(frame)))])

    return StrandScene(f"hair_groom {n_strands}x{count}", [s], [colliders(0)], root_path=root_path,
                       iterations=iterations,
                       meta={"n_strands": n_strands, "count": count, "colliders_at": colliders})


def hanging_strands(n_strands=256, count=32, segment=0.01, tilt=0.3, seed=7, iterations=20):
    """Strands hanging from a square grid of roots (2 cm pitch) at z = 1 m, each tilted from
    straight down by a seeded U(-tilt, tilt) in x and y: they swing to rest under gravity, a
    stable equilibrium (unlike a groom growing upward, whose strands buckle). Static roots, no
    colliders, reference StrandParams defaults."""
    from .runtime import make_strands
    rng = np.random.default_rng(seed)
    g = int(np.ceil(np.sqrt(n_strands)))
    xs, ys = np.meshgrid(np.arange(g) * 0.02, np.arange(g) * 0.02)
    roots = np.stack([xs.ravel(), ys.ravel(), np.ones(g * g)], 1)[:n_strands].astype(np.float32)
    d = np.concatenate([rng.uniform(-tilt, tilt, (n_strands, 2)), -np.ones((n_strands, 1))], 1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = np.arange(count)[None, :, None]
    pts = (roots[:, None, :] + d[:, None, :] * segment * k).astype(np.float32)
    s = make_strands(list(pts))
    return StrandScene(f"hanging_strands {n_strands}x{count}", [s], [None], iterations=iterations,
                       meta={"n_strands": n_strands, "count": count})


# ------------------------------------------------------------------------------------------
# Collider geometry: convex hulls and triangle meshes
# ------------------------------------------------------------------------------------------

def _hull_from_faces(vertices, faces):
    """Hull from vertex positions and faces given as vertex-index lists CCW about their outward
    normals; the plane is (unit normal of the first three vertices, dot(normal, first vertex))."""
    v = np.asarray(vertices, np.float32)
    planes, starts, fv = [], [0], []
    for f in faces:
        a, b, c = v[f[0]], v[f[1]], v[f[2]]
        n = np.cross(b - a, c - a).astype(np.float32)
        n = (n / np.float32(np.sqrt(np.dot(n, n)))).astype(np.float32)
        planes.append([n[0], n[1], n[2], np.dot(n, a)])
        fv.extend(f)
        starts.append(len(fv))
    return Hull(v, np.array(planes, np.float32), starts, fv)


def prism_hull(sides=6, radius=0.3, half_height=0.2):
    """A right prism over a regular polygon: two polygon faces and `sides` quads."""
    ang = 2.0 * np.pi * np.arange(sides) / sides
    ring = np.stack([radius * np.cos(ang), radius * np.sin(ang)], 1)
    verts = [(x, y, -half_height) for x, y in ring] + [(x, y, half_height) for x, y in ring]
    faces = [list(range(sides, 2 * sides)), list(range(sides - 1, -1, -1))]
    for i in range(sides):
        j = (i + 1) % sides
        faces.append([i, j, sides + j, sides + i])
    return _hull_from_faces(verts, faces)


def random_hull(n_points=24, radius=0.3, seed=0):
    """Convex hull of points drawn on a jittered sphere: triangular faces (scipy's facets)."""
    from scipy.spatial import ConvexHull
    rng = np.random.default_rng(seed)
    pts = rng.normal(size=(n_points, 3))
    pts = (radius * pts / np.linalg.norm(pts, axis=1, keepdims=True) * rng.uniform(0.8, 1.0, (n_points, 1)))
    pts = pts.astype(np.float32)
    ch = ConvexHull(pts)
    faces = []
    for simplex, eq in zip(ch.simplices, ch.equations):
        a, b, c = pts[simplex]
        if np.dot(np.cross(b - a, c - a), eq[:3]) < 0:
            simplex = simplex[[0, 2, 1]]
        faces.append([int(k) for k in simplex])
    return _hull_from_faces(pts, faces)


def floor_mesh(half=2.0):
    """Two coplanar triangles forming a square floor in the z = 0 plane, normals +Z (the
    reference tests' two-triangle floor)."""
    v = [(-half, -half, 0.0), (half, -half, 0.0), (half, half, 0.0), (-half, half, 0.0)]
    return Mesh(v, [0, 1, 2, 0, 2, 3], [(0, 0, 1), (0, 0, 1)])


def corner_mesh():
    """A right-angled inside corner: floor z = 0 (normal +Z) and wall x = 0 (normal +X)."""
    v = [(0, -1, 0), (1, -1, 0), (1, 1, 0), (0, 1, 0), (0, -1, 1), (0, 1, 1)]
    return Mesh(v, [0, 1, 2, 0, 2, 3, 0, 3, 5, 0, 5, 4], [(0, 0, 1), (0, 0, 1), (1, 0, 0), (1, 0, 0)])


def terrain_mesh(n=32, size=3.0, amp=0.15, seed=0):
    """A height-field terrain: (n + 1)^2 vertices over a size x size square, 2 n^2 triangles
    wound to face +Z, heights a sum of three seeded sine waves of amplitude amp. Normals are left
    to the registration (TriangleMesh::from_triangles' formula)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-size / 2, size / 2, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    Z = np.zeros_like(X)
    for _ in range(3):
        k = rng.uniform(1.0, 4.0, 2)
        ph = rng.uniform(0, 2 * np.pi, 2)
        Z += amp / 3 * np.sin(k[0] * X + ph[0]) * np.cos(k[1] * Y + ph[1])
    verts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.float32)
    idx = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            b, c, d = a + 1, a + n + 2, a + n + 1
            idx += [a, b, c, a, c, d]
    return Mesh(verts, np.array(idx, np.uint32))


def height_grid_terrain(nx=40, ny=40, cell=0.08, amp=0.12, seed=0):
    """A seeded height grid (geometry::HeightGrid): two sine ridges plus uniform noise of
    amplitude amp / 4, centred on the origin by the collider's local centre."""
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny))
    h = amp * (np.sin(0.35 * i + 0.2) * np.cos(0.27 * j)) + rng.uniform(-0.25, 0.25, (ny, nx)) * amp
    return HeightGrid(nx, ny, (cell, cell), h.astype(np.float32).reshape(-1))


def height_grid_drape(side=20, seed=14, params=None):
    """One sheet dropped onto a height-grid terrain (geometry id 1) beside a sphere."""
    grid = height_grid_terrain(40, 36, 0.06, 0.1, seed)
    centre = (-0.5 * 39 * 0.06, -0.5 * 35 * 0.06, 0.0)
    c = _sheet(side, (0.0, 0.0, 0.3), seed, [], params=params, tethers=False)
    cols = collider_array([mesh_collider(1, grid, local_center=centre), sphere(0.12, (0.3, -0.2, 0.15))])
    return ClothScene(f"height_grid_drape {side}x{side}", [c], [cols], meta={"side": side}, geometries=[grid])


def terrain_drape(side=32, seed=11, params=None):
    """One sheet dropped onto a seeded terrain mesh with a rotated convex-hull rock on it and a
    sphere: the mesh, hull and analytic branches in one collider list. Geometry ids 1 (terrain)
    and 2 (rock)."""
    rng = np.random.default_rng(seed)
    terrain = terrain_mesh(24, 3.0, 0.15, seed)
    rock = prism_hull(7, 0.25, 0.15)
    center = (0.0, 0.0, 0.45)
    c = _sheet(side, center, seed, [], params=params, tethers=False)
    cols = collider_array([
        mesh_collider(1, terrain),
        hull_collider(2, rock, (float(rng.uniform(-0.2, 0.2)), float(rng.uniform(-0.2, 0.2)), 0.12),
                      _random_quat(rng), scale=1.1),
        sphere(0.15, (0.4, -0.3, 0.2)),
    ])
    return ClothScene(f"terrain_drape {side}x{side}", [c], [cols], meta={"side": side},
                      geometries=[terrain, rock])


def mesh_floor_batch(n=4096, side=25, seed=12, height_grid=False, params=None):
    """N sheets of side x side (default 4096 x 25^2) resting on one 2048-triangle mesh floor: the
    reference's own costing case for mesh colliders (a 25x25 sheet on a 2048-triangle floor,
    cloth/README.md:98-102), batched. The floor is a 4 x 4 m height field of 32 x 32 cells with
    3 cm seeded bumps; each sheet is placed 6 cm above it at a seeded position, unpinned, with the
    floor as its one collider (geometry id 1). height_grid: the floor's 33 x 33 samples as a
    HeightGrid instead (TriangleMesh::from_height_grid), the same surface samples."""
    rng = np.random.default_rng(seed)
    floor = terrain_mesh(32, 4.0, 0.03, seed)
    if height_grid:
        floor = HeightGrid(33, 33, (0.125, 0.125), np.ascontiguousarray(floor.vertices[:, 2], np.float32))
        col = collider_array([mesh_collider(1, floor, local_center=(-2.0, -2.0, 0.0))])
    else:
        col = collider_array([mesh_collider(1, floor)])
    half = (side - 1) * SPACING * 0.5
    cloths, cols = [], []
    for k in range(n):
        cx, cy = (float(v) for v in rng.uniform(-2.0 + half, 2.0 - half, 2))
        cloths.append(_sheet(side, (cx, cy, 0.06), seed * 100003 + k, [], params=params, tethers=False))
        cols.append(col.copy())
    name = f"mesh_floor_batch {n}x{side}^2" + (" (height-grid floor)" if height_grid else "")
    return ClothScene(name, cloths, cols, meta={"side": side, "n": n},
                      geometries=[floor])


def disc_mesh(radius=0.5, rings=12, center=(0.0, 0.0, 1.0), jitter=0.0, seed=0):
    """A triangulated disc with no grid structure: a centre vertex and `rings` rings of 6k
    vertices (1 + 3 rings (rings + 1) in all), each ring stitched to the one inside it by an
    angle-ordered walk, so vertex valences vary from 5 to 7 and edges run in every direction.
    Vertices get a seeded in-plane jitter of `jitter` x the ring spacing. Faces wind
    counter-clockwise seen from +z. Returns (vertices [n, 3] float32, indices [3 t] uint32)."""
    rng = np.random.default_rng(seed)
    pts = [(0.0, 0.0)]
    start = [0, 1]
    for k in range(1, rings + 1):
        m = 6 * k
        r = radius * k / rings
        for j in range(m):
            a = 2.0 * np.pi * j / m
            pts.append((r * np.cos(a), r * np.sin(a)))
        start.append(len(pts))
    tris = [(0, 1 + j, 1 + (j + 1) % 6) for j in range(6)]
    for k in range(2, rings + 1):
        ni, no = 6 * (k - 1), 6 * k
        si, so = start[k - 1], start[k]
        i = o = 0
        while i < ni or o < no:
            # advance on the ring whose next vertex comes first in angle (exact integer compare)
            if o < no and (i >= ni or (o + 1) * ni <= (i + 1) * no):
                tris.append((si + i % ni, so + o, so + (o + 1) % no))
                o += 1
            else:
                tris.append((si + i, so + o % no, si + (i + 1) % ni))
                i += 1
    v = np.zeros((len(pts), 3), np.float32)
    v[:, :2] = np.array(pts, np.float64)
    if jitter > 0.0:
        v[1:, :2] += rng.uniform(-1.0, 1.0, (len(pts) - 1, 2)) * (jitter * radius / rings)
    v += np.asarray(center, np.float32)
    return v.astype(np.float32), np.array(tris, np.uint32).reshape(-1)


def mesh_cloth(rings=12, radius=0.5, center=(0.0, 0.0, 1.0), seed=0, pins=(), params=None, tethers=True,
               bend=True):
    """A disc-mesh cloth built by pxb_host_cloth_make_mesh, with static pins ((point, radius)
    pairs) and, when pinned, tethers."""
    v, ix = disc_mesh(radius, rings, center, jitter=0.25, seed=seed)
    from .runtime import HostCloth
    h = HostCloth.from_mesh(v, ix, total_mass=1.0, bend=bend, params=params or cloth_params())
    for point, r in pins:
        h.pin_static(point, r)
    if tethers and pins:
        h.build_tethers()
    return h.arrays()


def mesh_drape(rings=12, seed=0):
    """One disc-mesh cloth (1 + 3 rings (rings + 1) particles) pinned at two rim points, falling
    onto a sphere."""
    center = (0.0, 0.0, 1.0)
    radius = 0.5
    pins = [((center[0] - radius, center[1], center[2]), 0.3 * radius / rings),
            ((center[0] + radius, center[1], center[2]), 0.3 * radius / rings)]
    c = mesh_cloth(rings, radius, center, seed, pins)
    col = collider_array([sphere(0.2, (0.0, 0.1, 0.6))])
    return ClothScene(f"mesh_drape disc r{rings}", [c], [col], meta={"rings": rings})


def mesh_cloth_batch(n=1024, rings=20, seed=13):
    """N disc-mesh cloths (default 1024 x 1261 particles, 3660 stretch and 3540 bend
    constraints each), every one pinned at two rim points and draped over its own sphere: the
    general-topology path at batch scale."""
    rng = np.random.default_rng(seed)
    radius = 0.5
    cloths, cols = [], []
    for k in range(n):
        center = (float(rng.uniform(-4, 4)), float(rng.uniform(-4, 4)), 1.0)
        pins = [((center[0] - radius, center[1], center[2]), 0.3 * radius / rings),
                ((center[0] + radius, center[1], center[2]), 0.3 * radius / rings)]
        cloths.append(mesh_cloth(rings, radius, center, seed * 100003 + k, pins))
        cols.append(collider_array([sphere(0.2, (center[0], center[1] + 0.1, 0.6))]))
    return ClothScene(f"mesh_cloth_batch {n}x disc r{rings}", cloths, cols, meta={"rings": rings, "n": n})


def register_geometries(ctx, scene):
    """Registers scene.geometries with a runtime.Context and rewrites the colliders' geometry ids
    from the scene's numbering (geometry k is id k + 1) to the ids the context returned. Returns
    those ids."""
    ids = [ctx.create_geometry(g) for g in scene.geometries]
    remap = {k + 1: gid for k, gid in enumerate(ids)}
    for cols in scene.colliders:
        if cols is None:
            continue
        for c in cols:
            if c["type"] in (A.SHAPE_TRIANGLE_MESH, A.SHAPE_CONVEX_HULL) and int(c["geometry"]) in remap:
                c["geometry"] = remap[int(c["geometry"])]
    scene.geometries_ids = ids
    return ids
