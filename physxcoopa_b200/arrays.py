"""Host-side containers for cloths and strand sets in the reference's memory layout.

`ClothArrays` holds the fields of cloth::Cloth (physxcoopa/cloth/cloth.h:284-315) as numpy
arrays of the reference's own record layouts; `StrandArrays` does the same for hair::StrandSet
(physxcoopa/hair/strand.h:157-191). Both can describe themselves to the C-ABI as a plain
pointer struct (pxb_cloth_desc / pxb_strand_set_desc) without copying.

The collider helpers build pxb_collider snapshots the way the reference does: a
collision::Shape made by Shape::make_sphere/make_box/make_capsule (shape.h:109-136) posed at a
body transform, with ClothCollider::bounds = collision::world_bounds (shape.h:198-228).
"""
from dataclasses import dataclass, field
from typing import Optional
import copy

import numpy as np

from . import _abi as A


@dataclass
class ClothArrays:
    particles: np.ndarray
    stretch: np.ndarray
    stretch_batches: np.ndarray
    bend: np.ndarray
    bend_batches: np.ndarray
    tethers: np.ndarray
    anchors: np.ndarray
    triangles: np.ndarray
    columns: int = 0
    rows: int = 0
    params: A.ClothParams = field(default_factory=A.ClothParams.defaults)
    time: float = 0.0
    bounds: Optional[np.ndarray] = None
    stretch_batch_compliance: Optional[np.ndarray] = None
    bend_batch_compliance: Optional[np.ndarray] = None

    def copy(self):
        c = copy.copy(self)
        for name in ("particles", "stretch", "stretch_batches", "bend", "bend_batches",
                     "tethers", "anchors", "triangles", "bounds", "stretch_batch_compliance",
                     "bend_batch_compliance"):
            v = getattr(self, name)
            setattr(c, name, None if v is None else v.copy())
        p = A.ClothParams()
        A.C.pointer(p)[0] = self.params
        c.params = p
        return c

    @property
    def positions(self):
        return self.particles["position"]

    def desc(self) -> A.ClothDesc:
        """A pxb_cloth_desc pointing into these arrays (valid while they are alive)."""
        for name in ("particles", "stretch", "stretch_batches", "bend", "bend_batches",
                     "tethers", "anchors", "triangles"):
            a = getattr(self, name)
            if not a.flags["C_CONTIGUOUS"]:
                setattr(self, name, np.ascontiguousarray(a))
        d = A.ClothDesc()
        d.particles = A.ptr(self.particles)
        d.n_particles = len(self.particles)
        d.stretch = A.ptr(self.stretch)
        d.n_stretch = len(self.stretch)
        d.stretch_batches = A.ptr(self.stretch_batches)
        d.n_stretch_batches = len(self.stretch_batches)
        d.bend = A.ptr(self.bend)
        d.n_bend = len(self.bend)
        d.bend_batches = A.ptr(self.bend_batches)
        d.n_bend_batches = len(self.bend_batches)
        d.tethers = A.ptr(self.tethers)
        d.n_tethers = len(self.tethers)
        d.anchors = A.ptr(self.anchors)
        d.n_anchors = len(self.anchors)
        d.triangles = A.ptr(self.triangles)
        d.n_triangle_indices = len(self.triangles)
        d.columns = self.columns
        d.rows = self.rows
        d.params = self.params
        d.time = self.time
        d.stretch_batch_compliance = A.ptr(self.stretch_batch_compliance)
        d.bend_batch_compliance = A.ptr(self.bend_batch_compliance)
        return d

    @classmethod
    def from_desc(cls, d: A.ClothDesc, bounds=None):
        """Copies the arrays a pxb_cloth_desc points at."""
        def grab(addr, n, dtype):
            if n == 0 or not addr:
                return np.zeros(0, dtype)
            buf = (A.C.c_char * (n * dtype.itemsize)).from_address(addr)
            return np.frombuffer(bytes(buf), dtype).copy()
        params = A.ClothParams()
        A.C.pointer(params)[0] = d.params
        sbc = grab(d.stretch_batch_compliance, d.n_stretch_batches, np.dtype("<f4")) \
            if d.stretch_batch_compliance else None
        bbc = grab(d.bend_batch_compliance, d.n_bend_batches, np.dtype("<f4")) \
            if d.bend_batch_compliance else None
        return cls(particles=grab(d.particles, d.n_particles, A.PARTICLE),
                   stretch=grab(d.stretch, d.n_stretch, A.CONSTRAINT),
                   stretch_batches=grab(d.stretch_batches, d.n_stretch_batches, A.BATCH),
                   bend=grab(d.bend, d.n_bend, A.CONSTRAINT),
                   bend_batches=grab(d.bend_batches, d.n_bend_batches, A.BATCH),
                   tethers=grab(d.tethers, d.n_tethers, A.TETHER),
                   anchors=grab(d.anchors, d.n_anchors, A.ANCHOR),
                   triangles=grab(d.triangles, d.n_triangle_indices, np.dtype("<u4")),
                   columns=d.columns, rows=d.rows, params=params, time=d.time, bounds=bounds,
                   stretch_batch_compliance=sbc, bend_batch_compliance=bbc)


@dataclass
class StrandArrays:
    particles: np.ndarray
    stretch: np.ndarray
    stretch_batches: np.ndarray
    rest_local: np.ndarray   # (n, 3) float32
    rest_offset: np.ndarray  # (n, 3) float32
    strands: np.ndarray
    params: A.StrandParams = field(default_factory=A.StrandParams.defaults)
    time: float = 0.0
    bounds: Optional[np.ndarray] = None

    def copy(self):
        s = copy.copy(self)
        for name in ("particles", "stretch", "stretch_batches", "rest_local", "rest_offset",
                     "strands", "bounds"):
            v = getattr(self, name)
            setattr(s, name, None if v is None else v.copy())
        p = A.StrandParams()
        A.C.pointer(p)[0] = self.params
        s.params = p
        return s

    def desc(self) -> A.StrandSetDesc:
        d = A.StrandSetDesc()
        self.rest_local = np.ascontiguousarray(self.rest_local, np.float32)
        self.rest_offset = np.ascontiguousarray(self.rest_offset, np.float32)
        d.particles = A.ptr(self.particles)
        d.n_particles = len(self.particles)
        d.stretch = A.ptr(self.stretch)
        d.n_stretch = len(self.stretch)
        d.stretch_batches = A.ptr(self.stretch_batches)
        d.n_stretch_batches = len(self.stretch_batches)
        d.rest_local = A.ptr(self.rest_local)
        d.rest_offset = A.ptr(self.rest_offset)
        d.strands = A.ptr(self.strands)
        d.n_strands = len(self.strands)
        d.params = self.params
        d.time = self.time
        return d


# ------------------------------------------------------------------------------------------
# Collider snapshots
# ------------------------------------------------------------------------------------------

IDENTITY = (0.0, 0.0, 0.0, 1.0)  # (x, y, z, w)


def _qrot(q, v):
    """Unit-quaternion rotation in float32, v + 2*(w*(u x v) + u x (u x v))."""
    q = np.asarray(q, np.float32)
    v = np.asarray(v, np.float32)
    u = q[:3]
    uv = np.cross(u, v).astype(np.float32)
    uuv = np.cross(u, uv).astype(np.float32)
    return (v + ((uv * q[3]) + uuv) * np.float32(2.0)).astype(np.float32)


def _qmul(p, q):
    px, py, pz, pw = [np.float32(x) for x in p]
    qx, qy, qz, qw = [np.float32(x) for x in q]
    return np.array([pw * qx + px * qw + py * qz - pz * qy,
                     pw * qy + py * qw + pz * qx - px * qz,
                     pw * qz + pz * qw + px * qy - py * qx,
                     pw * qw - px * qx - py * qy - pz * qz], np.float32)


def _axes(q):
    x, y, z, w = [np.float32(v) for v in q]
    one, two = np.float32(1), np.float32(2)
    xx, yy, zz, xz, xy, yz = x * x, y * y, z * z, x * z, x * y, y * z
    wx, wy, wz = w * x, w * y, w * z
    return (np.array([one - two * (yy + zz), two * (xy + wz), two * (xz - wy)], np.float32),
            np.array([two * (xy - wz), one - two * (xx + zz), two * (yz + wx)], np.float32),
            np.array([two * (xz + wy), two * (yz - wx), one - two * (xx + yy)], np.float32))


def _world_bounds(c):
    """collision::world_bounds (shape.h:198-228) for sphere / box / capsule."""
    pos = c["position"]
    rot = c["orientation"]
    center = (pos + _qrot(rot, c["local_center"])).astype(np.float32)
    if c["type"] == A.SHAPE_SPHERE:
        r = np.float32(c["radius"])
        return center - r, center + r
    if c["type"] == A.SHAPE_CAPSULE:
        axis_local = np.zeros(3, np.float32)
        axis_local[int(c["capsule_axis"])] = 1.0
        axis_world = _qrot(_qmul(rot, c["local_rotation"]), axis_local)
        hh = np.float32(c["capsule_half_height"])
        a = center - axis_world * hh
        b = center + axis_world * hh
        r = np.float32(c["capsule_radius"])
        return np.minimum(a, b) - r, np.maximum(a, b) + r
    if c["type"] == A.SHAPE_BOX:
        # OBB::bounds (obb.h:42-52): the 8 corners of the box transformed and re-fitted.
        orient = _qmul(rot, c["local_rotation"])
        ax, ay, az = _axes(orient)
        he = c["half_extents"]
        lo = np.full(3, np.finfo(np.float32).max, np.float32)
        hi = -lo
        for i in range(8):
            corner = np.array([he[0] if i & 1 else -he[0], he[1] if i & 2 else -he[1],
                               he[2] if i & 4 else -he[2]], np.float32)
            w = ax * corner[0] + ay * corner[1] + az * corner[2] + center
            lo = np.minimum(lo, w)
            hi = np.maximum(hi, w)
        return lo, hi
    if c["type"] in (A.SHAPE_TRIANGLE_MESH, A.SHAPE_CONVEX_HULL):
        raise ValueError("mesh and hull bounds need the geometry: use hull_collider / mesh_collider")
    raise ValueError("unsupported collider type")


def _posed_bounds(lo_local, hi_local, center, orient, scale):
    """world_bounds of a TriangleMesh / ConvexHull (shape.h:216-225): the 8 corners of the local
    bounds through rotation * scale, plus the posed centre, re-fitted (AABB::transform)."""
    ax, ay, az = _axes(orient)
    s = np.float32(scale)
    lo = np.full(3, np.finfo(np.float32).max, np.float32)
    hi = -lo
    for i in range(8):
        corner = np.array([hi_local[0] if i & 1 else lo_local[0], hi_local[1] if i & 2 else lo_local[1],
                           hi_local[2] if i & 4 else lo_local[2]], np.float32)
        w = ((ax * s) * corner[0] + (ay * s) * corner[1]) + ((az * s) * corner[2] + center)
        lo = np.minimum(lo, w)
        hi = np.maximum(hi, w)
    return lo.astype(np.float32), hi.astype(np.float32)


class Hull:
    """geometry::ConvexHull's arrays (physxcoopa/geometry/convex_hull.h:41-57): vertices, face
    planes (outward unit normal, offset), and each face's vertex indices CCW about its normal."""

    def __init__(self, vertices, face_planes, face_starts, face_vertices):
        self.vertices = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        self.face_planes = np.ascontiguousarray(face_planes, np.float32).reshape(-1, 4)
        self.face_starts = np.ascontiguousarray(face_starts, np.uint32).reshape(-1)
        self.face_vertices = np.ascontiguousarray(face_vertices, np.uint32).reshape(-1)

    def desc(self):
        d = A.HullDesc()
        d.vertices = A.ptr(self.vertices)
        d.n_vertices = len(self.vertices)
        d.face_planes = A.ptr(self.face_planes)
        d.n_faces = len(self.face_planes)
        d.face_starts = A.ptr(self.face_starts)
        d.face_vertices = A.ptr(self.face_vertices)
        return d

    def local_bounds(self):
        return self.vertices.min(axis=0), self.vertices.max(axis=0)


class Mesh:
    """geometry::TriangleMesh's vertices, triangle indices and face normals
    (physxcoopa/geometry/triangle_mesh.h:70-96). normals None: computed on registration as
    TriangleMesh::from_triangles does."""

    def __init__(self, vertices, indices, normals=None):
        self.vertices = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)

    def desc(self):
        d = A.MeshDesc()
        d.vertices = A.ptr(self.vertices)
        d.n_vertices = len(self.vertices)
        d.indices = A.ptr(self.indices)
        d.n_indices = len(self.indices)
        d.normals = A.ptr(self.normals)
        return d

    def local_bounds(self):
        return self.vertices.min(axis=0), self.vertices.max(axis=0)


class HeightGrid:
    """geometry::HeightGrid's samples (physxcoopa/geometry/height_grid.h): nx x ny heights, row j
    at j * nx, sample (i, j) at (i * cell_x, j * cell_y, height); used as a TriangleMesh through
    TriangleMesh::from_height_grid (triangle_mesh.h:210-215), two triangles per cell."""

    def __init__(self, nx, ny, cell, heights):
        self.nx, self.ny = int(nx), int(ny)
        self.cell = (float(cell[0]), float(cell[1]))
        self.heights = np.ascontiguousarray(heights, np.float32).reshape(-1)

    def desc(self):
        d = A.HeightGridDesc()
        d.nx, d.ny = self.nx, self.ny
        d.cell_x, d.cell_y = self.cell
        d.heights = A.ptr(self.heights)
        d.n_heights = len(self.heights)
        return d

    def local_bounds(self):
        """HeightGrid::bounds(): the box of every sample (heights padded with zeros)."""
        nx, ny = max(2, self.nx), max(2, self.ny)
        h = np.zeros(nx * ny, np.float32)
        h[:min(len(self.heights), nx * ny)] = self.heights[:nx * ny]
        lo = np.array([0.0, 0.0, h.min()], np.float32)
        hi = np.array([np.float32(nx - 1) * np.float32(self.cell[0]), np.float32(ny - 1) * np.float32(self.cell[1]),
                       h.max()], np.float32)
        return lo, hi


def make_collider(shape_type, position=(0, 0, 0), orientation=IDENTITY, *, radius=0.5,
                  half_extents=(0.5, 0.5, 0.5), capsule_radius=0.5, capsule_half_height=0.5,
                  capsule_axis=2, local_center=(0, 0, 0), local_rotation=IDENTITY,
                  sweep=(0, 0, 0), end_orientation=None, enabled=True):
    """One pxb_collider record, with ClothCollider::bounds computed as world_bounds."""
    c = np.zeros((), A.COLLIDER)
    c["type"] = shape_type
    c["enabled"] = 1 if enabled else 0
    c["position"] = position
    c["orientation"] = orientation
    c["local_center"] = local_center
    c["local_rotation"] = local_rotation
    c["radius"] = radius
    c["half_extents"] = half_extents
    c["capsule_radius"] = capsule_radius
    c["capsule_half_height"] = capsule_half_height
    c["capsule_axis"] = capsule_axis
    c["sweep"] = sweep
    c["end_orientation"] = orientation if end_orientation is None else end_orientation
    lo, hi = _world_bounds(c)
    if np.dot(np.asarray(sweep, np.float32), np.asarray(sweep, np.float32)) > 0:
        end = c.copy()
        end["position"] = np.asarray(position, np.float32) + np.asarray(sweep, np.float32)
        end["orientation"] = c["end_orientation"]
        lo2, hi2 = _world_bounds(end)
        lo, hi = np.minimum(lo, lo2), np.maximum(hi, hi2)
    c["bounds_min"] = lo
    c["bounds_max"] = hi
    return c


def sphere(radius, position=(0, 0, 0), **kw):
    return make_collider(A.SHAPE_SPHERE, position, radius=radius, **kw)


def box(half_extents, position=(0, 0, 0), orientation=IDENTITY, **kw):
    return make_collider(A.SHAPE_BOX, position, orientation, half_extents=half_extents, **kw)


def capsule(radius, half_height, position=(0, 0, 0), orientation=IDENTITY, axis=2, **kw):
    return make_collider(A.SHAPE_CAPSULE, position, orientation, capsule_radius=radius,
                         capsule_half_height=half_height, capsule_axis=axis, **kw)


def _geometry_collider(shape_type, geometry_id, geometry, position, orientation, scale, local_center,
                       local_rotation, enabled):
    c = np.zeros((), A.COLLIDER)
    c["type"] = shape_type
    c["enabled"] = 1 if enabled else 0
    c["position"] = position
    c["orientation"] = orientation
    c["local_center"] = local_center
    c["local_rotation"] = local_rotation
    c["end_orientation"] = orientation
    c["geometry"] = geometry_id
    c["geometry_scale"] = scale
    center = (np.asarray(position, np.float32) + _qrot(orientation, local_center)).astype(np.float32)
    lo, hi = geometry.local_bounds()
    c["bounds_min"], c["bounds_max"] = _posed_bounds(lo, hi, center, _qmul(orientation, local_rotation), scale)
    return c


def hull_collider(geometry_id, hull, position=(0, 0, 0), orientation=IDENTITY, *, scale=1.0,
                  local_center=(0, 0, 0), local_rotation=IDENTITY, enabled=True):
    """A ConvexHull collider (Shape::make_hull, shape.h:147-155) naming the geometry id a context
    returned for `hull`, with ClothCollider::bounds as world_bounds computes it."""
    return _geometry_collider(A.SHAPE_CONVEX_HULL, geometry_id, hull, position, orientation, scale,
                              local_center, local_rotation, enabled)


def mesh_collider(geometry_id, mesh, position=(0, 0, 0), orientation=IDENTITY, *, scale=1.0,
                  local_center=(0, 0, 0), local_rotation=IDENTITY, enabled=True):
    """A TriangleMesh collider (Shape::make_mesh, shape.h:138-145; meshes are static, so it is
    never swept) naming the geometry id a context returned for `mesh`."""
    return _geometry_collider(A.SHAPE_TRIANGLE_MESH, geometry_id, mesh, position, orientation, scale,
                              local_center, local_rotation, enabled)


def collider_array(records):
    return np.ascontiguousarray(np.array(list(records), A.COLLIDER).reshape(-1))


def gravity_sources(records):
    """records: iterable of (centre, strength, radius, range)."""
    out = np.zeros(len(records), A.GRAVITY_SOURCE)
    for i, (c, s, r, rg) in enumerate(records):
        out[i]["centre"] = c
        out[i]["strength"] = s
        out[i]["radius"] = r
        out[i]["range"] = rg
    return out
