"""Loads the test-side checkers built by oracle/Makefile.

  liboracle.so  -- the C restatement of the reference algorithm (oracle/xpbd_oracle.c)
  libpxbref.so  -- the reference's own headers compiled against the glm-subset shim

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
import ctypes as C
import os

import numpy as np

from physxcoopa_b200 import _abi as A
from physxcoopa_b200.arrays import ClothArrays, StrandArrays

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libpxbref.so")
# the same reference sources built -O3 -march=native (the CPU baseline's second build mode)
REF_SO_NATIVE = os.path.join(ROOT, "oracle", "_ref", "libpxbref_native.so")

f32p = C.POINTER(C.c_float)
P = C.c_void_p


class OrcCloth(C.Structure):
    _fields_ = [("particles", P), ("n_particles", A.u32), ("stretch", P), ("n_stretch", A.u32),
                ("stretch_batches", P), ("n_stretch_batches", A.u32), ("bend", P),
                ("n_bend", A.u32), ("bend_batches", P), ("n_bend_batches", A.u32),
                ("tethers", P), ("n_tethers", A.u32), ("anchors", P), ("n_anchors", A.u32),
                ("triangles", P), ("n_triangle_indices", A.u32), ("columns", A.u32),
                ("rows", A.u32), ("params", A.ClothParams), ("time", A.f32),
                ("stretch_batch_compliance", P), ("bend_batch_compliance", P),
                ("bounds_min", A.f32 * 3), ("bounds_max", A.f32 * 3)]


class OrcStrandSet(C.Structure):
    _fields_ = [("particles", P), ("n_particles", A.u32), ("stretch", P), ("n_stretch", A.u32),
                ("stretch_batches", P), ("n_stretch_batches", A.u32), ("rest_local", P),
                ("rest_offset", P), ("strands", P), ("n_strands", A.u32),
                ("params", A.StrandParams), ("time", A.f32), ("bounds_min", A.f32 * 3),
                ("bounds_max", A.f32 * 3)]


_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        lib = C.CDLL(ORACLE_SO)
        lib.orc_solve_cloth.argtypes = [C.POINTER(OrcCloth), P, A.u32, f32p, A.u32, A.u32, A.f32]
        lib.orc_step_cloth.argtypes = [C.POINTER(OrcCloth), P, A.u32, f32p, P, A.u32, A.u32,
                                       A.u32, A.f32]
        lib.orc_project_particle.argtypes = [P, A.f32, f32p, f32p, f32p, P]
        lib.orc_gravity_at.argtypes = [f32p, P, A.u32, f32p, f32p]
        lib.orc_cloth_centre.argtypes = [P, A.u32, f32p]
        lib.orc_max_particle_speed.argtypes = [P, A.u32]
        lib.orc_max_particle_speed.restype = A.f32
        lib.orc_frame_substeps.argtypes = [A.f32, A.f32, A.u32]
        lib.orc_frame_substeps.restype = A.u32
        lib.orc_solve_strands.argtypes = [C.POINTER(OrcStrandSet), P, A.u32, f32p, A.u32, A.u32,
                                          A.f32]
        lib.orc_step_strands.argtypes = [C.POINTER(OrcStrandSet), P, A.u32, f32p, P, A.u32,
                                         A.u32, A.u32, A.f32]
        lib.orc_set_strand_roots.argtypes = [C.POINTER(OrcStrandSet), P, A.u32, P, A.u32]
        lib.orc_world_step_cloth.argtypes = [C.POINTER(OrcCloth), P, A.u32, C.c_int, P, A.u32, f32p, P, A.u32,
                                             A.f32, A.u32, A.u32, A.f32, C.POINTER(C.c_int), C.POINTER(A.f32)]
        lib.orc_world_step_strands.argtypes = [C.POINTER(OrcStrandSet), C.c_int, P, A.u32, f32p, P, A.u32,
                                               A.f32, A.u32, A.u32, A.f32, C.POINTER(C.c_int), C.POINTER(A.f32)]
        lib.orc_geometry_set_hull.argtypes = [A.u32, C.POINTER(A.HullDesc)]
        lib.orc_geometry_set_mesh.argtypes = [A.u32, C.POINTER(A.MeshDesc)]
        lib.orc_geometry_clear.argtypes = []
        lib.orc_geometry_clear.restype = None
        _oracle = lib
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = load_ref(REF_SO)
    return _ref


def load_ref(path):
    """Loads one build of the reference driver and declares its entry points."""
    lib = C.CDLL(path)
    lib.pxbref_cloth_make_grid.argtypes = [C.POINTER(A.GridClothDesc)]
    lib.pxbref_cloth_make_grid.restype = P
    lib.pxbref_cloth_from_desc.argtypes = [C.POINTER(A.ClothDesc)]
    lib.pxbref_cloth_from_desc.restype = P
    lib.pxbref_cloth_free.argtypes = [P]
    lib.pxbref_cloth_pin_static.argtypes = [P, f32p, A.f32]
    lib.pxbref_cloth_pin_static.restype = A.u32
    lib.pxbref_cloth_pin_to_body.argtypes = [P, A.u32, A.u32, f32p, f32p, f32p, A.f32]
    lib.pxbref_cloth_pin_to_body.restype = A.u32
    lib.pxbref_cloth_build_tethers.argtypes = [P]
    lib.pxbref_cloth_view.argtypes = [P, C.POINTER(A.ClothDesc)]
    lib.pxbref_cloth_bounds.argtypes = [P, f32p]
    lib.pxbref_solve_cloth.argtypes = [P, P, A.u32, f32p, A.u32, A.u32, A.f32]
    lib.pxbref_project_particle.argtypes = [P, A.f32, f32p, f32p, f32p, P]
    lib.pxbref_geometry_set_hull.argtypes = [A.u32, C.POINTER(A.HullDesc)]
    lib.pxbref_geometry_set_mesh.argtypes = [A.u32, C.POINTER(A.MeshDesc)]
    lib.pxbref_geometry_clear.argtypes = []
    lib.pxbref_geometry_clear.restype = None
    lib.pxbref_build_convex_hull.argtypes = [P, A.u32, P, A.u32, C.POINTER(A.u32), P, A.u32, P, P, A.u32]
    lib.pxbref_project_particle.restype = C.c_int
    lib.pxbref_bench_cloths.argtypes = [C.POINTER(P), A.u32, P, P, P, P, f32p, A.u32, A.u32,
                                        A.f32, A.u32, A.u32]
    lib.pxbref_bench_cloths.restype = C.c_double
    lib.pxbref_strands_make.argtypes = [A.u32, P, P, P, P, C.POINTER(A.StrandParams)]
    lib.pxbref_strands_make.restype = P
    lib.pxbref_strands_free.argtypes = [P]
    lib.pxbref_strands_view.argtypes = [P, C.POINTER(A.StrandSetDesc)]
    lib.pxbref_strands_bounds.argtypes = [P, f32p]
    lib.pxbref_strands_set_roots.argtypes = [P, P, A.u32, P, A.u32]
    lib.pxbref_solve_strands.argtypes = [P, P, A.u32, f32p, A.u32, A.u32, A.f32]
    return lib


def vec(x):
    return (C.c_float * 3)(*[float(v) for v in x])


# ------------------------------------------------------------------------------------------
# Oracle calls on ClothArrays / StrandArrays (advanced in place)
# ------------------------------------------------------------------------------------------

def _orc_cloth(c: ClothArrays):
    o = OrcCloth()
    o.particles = A.ptr(c.particles)
    o.n_particles = len(c.particles)
    o.stretch = A.ptr(c.stretch)
    o.n_stretch = len(c.stretch)
    o.stretch_batches = A.ptr(c.stretch_batches)
    o.n_stretch_batches = len(c.stretch_batches)
    o.bend = A.ptr(c.bend)
    o.n_bend = len(c.bend)
    o.bend_batches = A.ptr(c.bend_batches)
    o.n_bend_batches = len(c.bend_batches)
    o.tethers = A.ptr(c.tethers)
    o.n_tethers = len(c.tethers)
    o.anchors = A.ptr(c.anchors)
    o.n_anchors = len(c.anchors)
    o.triangles = A.ptr(c.triangles)
    o.n_triangle_indices = len(c.triangles)
    o.columns = c.columns
    o.rows = c.rows
    o.params = c.params
    o.time = c.time
    o.stretch_batch_compliance = A.ptr(c.stretch_batch_compliance)
    o.bend_batch_compliance = A.ptr(c.bend_batch_compliance)
    return o


def oracle_step_cloth(c: ClothArrays, colliders=None, gravity=(0, 0, -9.81), sources=None,
                      substeps=4, iterations=10, h=1.0 / 60.0):
    """One PhysicsWorld cloth step of the oracle: gravity at the cloth centre, then solve_cloth."""
    o = _orc_cloth(c)
    cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
    src = sources if sources is not None else np.zeros(0, A.GRAVITY_SOURCE)
    r = oracle().orc_step_cloth(C.byref(o), A.ptr(cols), len(cols), vec(gravity), A.ptr(src),
                                len(src), substeps, iterations, h)
    assert r == 0, "oracle refused the input"
    c.time = o.time
    c.bounds = np.array(list(o.bounds_min) + list(o.bounds_max), np.float32)
    return c


def oracle_world_step_cloth(c: ClothArrays, state, bodies=None, colliders=None, collider_moving=False,
                            gravity=(0, 0, -9.81), sources=None, fixed_dt=1.0 / 60.0, cloth_substeps=4,
                            cloth_iterations=10, dt=1.0 / 60.0):
    """One PhysicsWorld::step_cloths_ frame of the oracle for one cloth (anchors from body poses,
    sleep gate, solve, sleep bookkeeping). state: dict with "awake" and "sleep_timer", updated.
    Returns 1 when the cloth was solved, 0 when it slept."""
    o = _orc_cloth(c)
    cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
    src = sources if sources is not None else np.zeros(0, A.GRAVITY_SOURCE)
    bod = None if bodies is None else np.ascontiguousarray(bodies, A.BODY_POSE).reshape(-1)
    awake = C.c_int(int(state["awake"]))
    timer = A.f32(state["sleep_timer"])
    r = oracle().orc_world_step_cloth(C.byref(o), A.ptr(bod), 0 if bod is None else len(bod), int(collider_moving),
                                      A.ptr(cols), len(cols), vec(gravity), A.ptr(src), len(src), fixed_dt,
                                      cloth_substeps, cloth_iterations, dt, C.byref(awake), C.byref(timer))
    assert r >= 0, "oracle refused the input"
    state["awake"], state["sleep_timer"] = int(awake.value), np.float32(timer.value)
    if r == 1:
        c.time = o.time
        c.bounds = np.array(list(o.bounds_min) + list(o.bounds_max), np.float32)
    return r


def _orc_strands(s: StrandArrays):
    o = OrcStrandSet()
    o.particles = A.ptr(s.particles)
    o.n_particles = len(s.particles)
    o.stretch = A.ptr(s.stretch)
    o.n_stretch = len(s.stretch)
    o.stretch_batches = A.ptr(s.stretch_batches)
    o.n_stretch_batches = len(s.stretch_batches)
    o.rest_local = A.ptr(s.rest_local)
    o.rest_offset = A.ptr(s.rest_offset)
    o.strands = A.ptr(s.strands)
    o.n_strands = len(s.strands)
    o.params = s.params
    o.time = s.time
    if s.bounds is None:  # compute_bounds over the particles (strand.h:195-202)
        pos = s.particles["position"]
        s.bounds = np.concatenate([pos.min(axis=0), pos.max(axis=0)]).astype(np.float32)
    b = s.bounds
    o.bounds_min = (C.c_float * 3)(*b[:3])
    o.bounds_max = (C.c_float * 3)(*b[3:])
    return o


def oracle_step_strands(s: StrandArrays, colliders=None, gravity=(0, 0, -9.81), sources=None,
                        substeps=4, iterations=4, h=1.0 / 60.0):
    o = _orc_strands(s)
    cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
    src = sources if sources is not None else np.zeros(0, A.GRAVITY_SOURCE)
    r = oracle().orc_step_strands(C.byref(o), A.ptr(cols), len(cols), vec(gravity), A.ptr(src),
                                  len(src), substeps, iterations, h)
    assert r == 0, "oracle refused the input"
    s.time = o.time
    s.bounds = np.array(list(o.bounds_min) + list(o.bounds_max), np.float32)
    return s


def oracle_world_step_strands(s: StrandArrays, state, colliders=None, collider_moving=False, gravity=(0, 0, -9.81),
                              sources=None, fixed_dt=1.0 / 60.0, cloth_substeps=4, cloth_iterations=10,
                              dt=1.0 / 60.0):
    """One PhysicsWorld::step_strands_ frame of the oracle for one set (root-moved wake, sleep
    gate, solve, sleep bookkeeping). state: dict with "awake" and "sleep_timer", updated. Returns 1
    when the set was solved, 0 when it slept."""
    o = _orc_strands(s)
    cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
    src = sources if sources is not None else np.zeros(0, A.GRAVITY_SOURCE)
    awake = C.c_int(int(state["awake"]))
    timer = A.f32(state["sleep_timer"])
    r = oracle().orc_world_step_strands(C.byref(o), int(collider_moving), A.ptr(cols), len(cols), vec(gravity),
                                        A.ptr(src), len(src), fixed_dt, cloth_substeps, cloth_iterations, dt,
                                        C.byref(awake), C.byref(timer))
    assert r >= 0, "oracle refused the input"
    state["awake"], state["sleep_timer"] = int(awake.value), np.float32(timer.value)
    if r == 1:
        s.time = o.time
        s.bounds = np.array(list(o.bounds_min) + list(o.bounds_max), np.float32)
    return r


def oracle_set_strand_roots(s: StrandArrays, positions, orientations=None):
    o = _orc_strands(s)
    pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    rot = None if orientations is None else np.ascontiguousarray(orientations, np.float32).reshape(-1, 4)
    oracle().orc_set_strand_roots(C.byref(o), A.ptr(pos), len(pos), A.ptr(rot),
                                  0 if rot is None else len(rot))


def _start(motion_start):
    return None if motion_start is None else (C.c_float * 3)(*[float(x) for x in motion_start])


def oracle_project(collider, thickness, p, motion_start=None):
    pp = (C.c_float * 3)(*[float(x) for x in p])
    n = (C.c_float * 3)()
    d = C.c_float(0.0)
    col = np.ascontiguousarray(np.asarray(collider, A.COLLIDER).reshape(1))
    r = oracle().orc_project_particle(A.ptr(col), thickness, pp, n, C.byref(d), _start(motion_start))
    return r, np.array(pp[:], np.float32), np.array(n[:], np.float32), np.float32(d.value)


# ------------------------------------------------------------------------------------------
# Reference (oracle/_ref) objects
# ------------------------------------------------------------------------------------------

def _copy_view(view, fields):
    out = {}
    for name, count, dtype in fields:
        n = getattr(view, count)
        addr = getattr(view, name)
        if n == 0 or not addr:
            out[name] = np.zeros(0, dtype)
        else:
            buf = (C.c_char * (n * dtype.itemsize)).from_address(addr)
            out[name] = np.frombuffer(bytes(buf), dtype).copy()
    return out


class RefCloth:
    """A cloth::Cloth owned by the reference driver."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def make_grid(cls, desc: A.GridClothDesc):
        return cls(ref().pxbref_cloth_make_grid(C.byref(desc)))

    @classmethod
    def from_arrays(cls, c: ClothArrays):
        d = c.desc()
        return cls(ref().pxbref_cloth_from_desc(C.byref(d)))

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.pxbref_cloth_free(self.h)
            self.h = None

    def pin_static(self, point, radius):
        return ref().pxbref_cloth_pin_static(self.h, vec(point), radius)

    def pin_to_body(self, body_index, body_generation, body_position, body_orientation, point, radius):
        return ref().pxbref_cloth_pin_to_body(self.h, body_index, body_generation, vec(body_position),
                                              (C.c_float * 4)(*[float(x) for x in body_orientation]), vec(point),
                                              radius)

    def build_tethers(self):
        ref().pxbref_cloth_build_tethers(self.h)

    def solve(self, colliders=None, gravity=(0, 0, -9.81), substeps=4, iterations=10, h=1 / 60):
        cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
        ref().pxbref_solve_cloth(self.h, A.ptr(cols), len(cols), vec(gravity), substeps,
                                 iterations, h)

    def arrays(self) -> ClothArrays:
        v = A.ClothDesc()
        ref().pxbref_cloth_view(self.h, C.byref(v))
        got = _copy_view(v, [("particles", "n_particles", A.PARTICLE),
                             ("stretch", "n_stretch", A.CONSTRAINT),
                             ("stretch_batches", "n_stretch_batches", A.BATCH),
                             ("bend", "n_bend", A.CONSTRAINT),
                             ("bend_batches", "n_bend_batches", A.BATCH),
                             ("tethers", "n_tethers", A.TETHER),
                             ("anchors", "n_anchors", A.ANCHOR),
                             ("triangles", "n_triangle_indices", np.dtype("<u4"))])
        b = (C.c_float * 6)()
        ref().pxbref_cloth_bounds(self.h, b)
        params = A.ClothParams()
        C.pointer(params)[0] = v.params
        return ClothArrays(columns=v.columns, rows=v.rows, params=params, time=v.time,
                           bounds=np.array(b[:], np.float32), **got)


class RefStrands:
    """A hair::StrandSet owned by the reference driver."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def make(cls, polylines, params, root_orientations=None, particle_masses=None):
        counts = np.array([len(p) for p in polylines], np.uint32)
        pts = np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 3)
                                                   for p in polylines]), np.float32)
        rot = None if root_orientations is None else np.ascontiguousarray(root_orientations, np.float32)
        mass = None if particle_masses is None else np.ascontiguousarray(particle_masses, np.float32)
        return cls(ref().pxbref_strands_make(len(counts), A.ptr(counts), A.ptr(pts), A.ptr(rot),
                                             A.ptr(mass), C.byref(params)))

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.pxbref_strands_free(self.h)
            self.h = None

    def set_roots(self, positions, orientations=None):
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        rot = None if orientations is None else np.ascontiguousarray(orientations, np.float32).reshape(-1, 4)
        ref().pxbref_strands_set_roots(self.h, A.ptr(pos), len(pos), A.ptr(rot),
                                       0 if rot is None else len(rot))

    def solve(self, colliders=None, gravity=(0, 0, -9.81), substeps=4, iterations=4, h=1 / 60):
        cols = colliders if colliders is not None else np.zeros(0, A.COLLIDER)
        ref().pxbref_solve_strands(self.h, A.ptr(cols), len(cols), vec(gravity), substeps,
                                   iterations, h)

    def arrays(self, params) -> StrandArrays:
        v = A.StrandSetDesc()
        ref().pxbref_strands_view(self.h, C.byref(v))
        got = _copy_view(v, [("particles", "n_particles", A.PARTICLE),
                             ("stretch", "n_stretch", A.CONSTRAINT),
                             ("stretch_batches", "n_stretch_batches", A.BATCH),
                             ("strands", "n_strands", A.STRAND)])
        n = v.n_particles
        rl = np.frombuffer(bytes((C.c_char * (12 * n)).from_address(v.rest_local)), np.float32).copy() if n else np.zeros(0, np.float32)
        ro = np.frombuffer(bytes((C.c_char * (12 * n)).from_address(v.rest_offset)), np.float32).copy() if n else np.zeros(0, np.float32)
        b = (C.c_float * 6)()
        ref().pxbref_strands_bounds(self.h, b)
        return StrandArrays(rest_local=rl.reshape(-1, 3), rest_offset=ro.reshape(-1, 3),
                            params=params, time=v.time, bounds=np.array(b[:], np.float32), **got)


def ref_project(collider, thickness, p, motion_start=None):
    pp = (C.c_float * 3)(*[float(x) for x in p])
    n = (C.c_float * 3)()
    d = C.c_float(0.0)
    col = np.ascontiguousarray(np.asarray(collider, A.COLLIDER).reshape(1))
    r = ref().pxbref_project_particle(A.ptr(col), thickness, pp, n, C.byref(d), _start(motion_start))
    return r, np.array(pp[:], np.float32), np.array(n[:], np.float32), np.float32(d.value)


# ------------------------------------------------------------------------------------------
# Collider geometry, registered under the same id in the oracle and the reference
# ------------------------------------------------------------------------------------------

def register_geometry(gid, geometry):
    """Registers a Hull or Mesh (physxcoopa_b200.arrays) under `gid` with the oracle and, when
    it is built, the reference driver, so colliders naming `gid` mean the same shape to both."""
    from physxcoopa_b200.arrays import HeightGrid, Hull
    if isinstance(geometry, HeightGrid):
        args = (gid, geometry.nx, geometry.ny, C.c_float(geometry.cell[0]), C.c_float(geometry.cell[1]),
                A.ptr(geometry.heights), len(geometry.heights))
        assert oracle().orc_geometry_set_height_grid(*args) == 0
        if ref_available():
            assert ref().pxbref_geometry_set_height_grid(*args) == 0
        return
    d = geometry.desc()
    if isinstance(geometry, Hull):
        assert oracle().orc_geometry_set_hull(gid, C.byref(d)) == 0
        if ref_available():
            assert ref().pxbref_geometry_set_hull(gid, C.byref(d)) == 0
    else:
        assert oracle().orc_geometry_set_mesh(gid, C.byref(d)) == 0
        if ref_available():
            assert ref().pxbref_geometry_set_mesh(gid, C.byref(d)) == 0


def ref_build_convex_hull(points):
    """geometry::build_convex_hull (the reference's own builder) over `points`, as a Hull."""
    from physxcoopa_b200.arrays import Hull
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    cap_v, cap_f, cap_fv = 256, 512, 4096
    verts = np.zeros((cap_v, 3), np.float32)
    planes = np.zeros((cap_f, 4), np.float32)
    starts = np.zeros(cap_f + 1, np.uint32)
    fverts = np.zeros(cap_fv, np.uint32)
    nv = A.u32(0)
    nf = ref().pxbref_build_convex_hull(A.ptr(pts), len(pts), A.ptr(verts), cap_v, C.byref(nv), A.ptr(planes),
                                        cap_f, A.ptr(starts), A.ptr(fverts), cap_fv)
    assert nf > 0, "degenerate point cloud or capacity too small"
    return Hull(verts[:nv.value], planes[:nf], starts[:nf + 1], fverts[:starts[nf]])
