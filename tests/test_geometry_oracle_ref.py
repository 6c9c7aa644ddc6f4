"""Mesh and convex-hull colliders: the oracle's restatement of the TriangleMesh and ConvexHull
branches of cloth::project_particle (cloth_collision.h:205-354, over MeshBVH and hull_vs_sphere)
pinned bit for bit to the reference's own code (oracle/_ref), on single projections and through
whole cloth and strand solves, plus the reference tests' known answers for mesh colliders
(tests/cloth_collision_test.cpp:218-395) against the oracle."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import scenes as S
from physxcoopa_b200.arrays import HeightGrid, collider_array, hull_collider, mesh_collider, sphere

import _checkers as K

pytestmark = pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")

QUATS = [(0.0, 0.0, 0.0, 1.0), (0.1, 0.7, 0.1, 0.7), (0.3, -0.2, 0.5, 0.7874008)]


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def unit(q):
    q = np.asarray(q, np.float32)
    return tuple(float(x) for x in (q / np.float32(np.sqrt(np.dot(q, q)))).astype(np.float32))


def hulls():
    cube_pts = np.array([[x, y, z] for x in (-.5, .5) for y in (-.5, .5) for z in (-.5, .5)], np.float32)
    rng = np.random.default_rng(4)
    return {"cube_ref": K.ref_build_convex_hull(cube_pts),
            "cloud_ref": K.ref_build_convex_hull(rng.normal(size=(60, 3)).astype(np.float32) * 0.3),
            "prism7": S.prism_hull(7, 0.35, 0.25),
            "random": S.random_hull(30, 0.4, seed=5)}


def meshes():
    return {"floor": S.floor_mesh(), "corner": S.corner_mesh(), "terrain": S.terrain_mesh(12, 2.0, 0.2, seed=3),
            "terrain_from_triangles": S.terrain_mesh(6, 2.0, 0.3, seed=9)}


def compare(col, thickness, pts, starts=None):
    hits = 0
    for i, p in enumerate(pts):
        st = None if starts is None else starts[i]
        a = K.oracle_project(col, thickness, p, st)
        b = K.ref_project(col, thickness, p, st)
        assert a[0] == b[0], (i, p, st)
        if a[0] == 1:
            hits += 1
            for x, y in zip(a[1:], b[1:]):
                assert same(x, y), (i, p, st, x, y)
    return hits


@pytest.mark.parametrize("name", ["cube_ref", "cloud_ref", "prism7", "random"])
def test_hull_projection_matches_reference(name):
    hull = hulls()[name]
    K.register_geometry(7, hull)
    rng = np.random.default_rng(11)
    total = 0
    for q in QUATS:
        for scale in (1.0, 0.7):
            col = hull_collider(7, hull, (0.1, -0.2, 0.3), unit(q), scale=scale, local_center=(0.05, 0.0, -0.02),
                                local_rotation=unit((0.0, 0.2, 0.0, 0.98)))
            pts = rng.uniform(-0.7, 0.7, (300, 3)).astype(np.float32) + np.float32([0.1, -0.2, 0.3])
            total += compare(col, 0.03, pts)
    assert total > 50  # inside and near-surface points both reached


@pytest.mark.parametrize("name", ["floor", "corner", "terrain", "terrain_from_triangles"])
def test_mesh_projection_matches_reference(name):
    mesh = meshes()[name]
    if name == "terrain_from_triangles":
        mesh.normals = None
    K.register_geometry(8, mesh)
    rng = np.random.default_rng(12)
    lo, hi = mesh.local_bounds()
    total = 0
    for q in QUATS[:2]:
        for scale in (1.0, 1.3):
            col = mesh_collider(8, mesh, (0.2, 0.1, -0.1), unit(q), scale=scale, local_center=(0.0, 0.1, 0.0))
            # near the surface: points in the local box grown by 5 cm, mapped through the pose
            local = rng.uniform(lo - 0.05, hi + 0.05, (250, 3)).astype(np.float32)
            world = np.array([K_pose(col, p) for p in local], np.float32)
            total += compare(col, 0.05, world)
            # swept crossings: starts 0.2 m away along random directions
            d = rng.normal(size=(250, 3)).astype(np.float32)
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            total += compare(col, 0.05, world, (world + 0.2 * d).astype(np.float32))
    assert total > 100


def K_pose(col, p):
    """world = position + rot * (local_center + local_rotation * (scale * p)), float32."""
    from physxcoopa_b200.arrays import _qmul, _qrot
    rot = col["orientation"]
    q = _qmul(rot, col["local_rotation"])
    return (col["position"] + _qrot(rot, col["local_center"]) + _qrot(q, np.float32(col["geometry_scale"]) * p))


def test_geometry_zero_and_disabled_never_collide():
    mesh = S.floor_mesh()
    K.register_geometry(9, mesh)
    for col in (mesh_collider(0, mesh), mesh_collider(9, mesh, enabled=False),
                hull_collider(0, S.prism_hull())):
        for impl in (K.oracle_project, K.ref_project):
            assert impl(col, 0.03, (0.0, 0.0, 0.01), (0.0, 0.0, 0.5))[0] == 0


# ------------------------------------------------------------------------------------------
# The reference tests' known answers (tests/cloth_collision_test.cpp:218-395)
# ------------------------------------------------------------------------------------------

@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_mesh_collider_returns_a_tunnelling_particle_to_its_entry_side(impl):
    proj = K.oracle_project if impl == "oracle" else K.ref_project
    K.register_geometry(10, S.floor_mesh())
    col = mesh_collider(10, S.floor_mesh())
    hit, p, n, _ = proj(col, 0.03, (0.0, 0.0, -0.5), (0.0, 0.0, 0.5))
    assert hit == 1 and abs(p[2] - 0.03) < 1e-4
    np.testing.assert_allclose(n, (0, 0, 1), atol=1e-4)
    hit, q, n, _ = proj(col, 0.03, (0.0, 0.0, 0.5), (0.0, 0.0, -0.5))
    assert hit == 1 and abs(q[2] + 0.03) < 1e-4
    np.testing.assert_allclose(n, (0, 0, -1), atol=1e-4)


@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_mesh_collider_projects_shallow_particles_out_the_front_face(impl):
    proj = K.oracle_project if impl == "oracle" else K.ref_project
    K.register_geometry(10, S.floor_mesh())
    col = mesh_collider(10, S.floor_mesh())
    hit, p, n, _ = proj(col, 0.03, (0.0, 0.0, -0.01))
    assert hit == 1 and abs(p[2] - 0.03) < 1e-4
    np.testing.assert_allclose(n, (0, 0, 1), atol=1e-4)
    hit, p, n, _ = proj(col, 0.03, (0.0, 0.0, 0.01))
    assert hit == 1 and abs(p[2] - 0.03) < 1e-4
    np.testing.assert_allclose(n, (0, 0, 1), atol=1e-4)
    # beyond the standoff, and a motion shorter than the thickness: untouched
    assert proj(col, 0.03, (0.0, 0.0, 0.10), (0.0, 0.0, 0.11))[0] == 0


@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_mesh_collider_concave_pocket_is_not_flipped(impl):
    proj = K.oracle_project if impl == "oracle" else K.ref_project
    K.register_geometry(11, S.corner_mesh())
    col = mesh_collider(11, S.corner_mesh())
    hit, p, _, _ = proj(col, 0.03, (-0.002, 0.0, 0.02))
    assert hit == 1 and p[0] <= 0.0 and p[2] >= 0.0
    hit, q, _, _ = proj(col, 0.03, (-0.002, 0.0, -0.002))
    assert hit == 1 and (q[0] > 0.0 or q[2] > 0.0)


# ------------------------------------------------------------------------------------------
# Whole solves through the collision stage
# ------------------------------------------------------------------------------------------

def _register(scene):
    for k, g in enumerate(scene.geometries):
        K.register_geometry(k + 1, g)


def test_cloth_on_terrain_and_hull_matches_reference_bitwise():
    sc = S.terrain_drape(side=16, params=A.ClothParams.defaults())  # no shear-compliance extension
    _register(sc)
    ref = K.RefCloth.from_arrays(sc.cloths[0])
    orc = sc.cloths[0].copy()
    cols = sc.colliders[0]
    for step in range(60):
        ref.solve(cols, substeps=4, iterations=6)
        K.oracle_step_cloth(orc, cols, substeps=4, iterations=6)
        if step % 20 == 19:
            got = ref.arrays()
            for f in ("position", "prev_position", "velocity"):
                assert same(orc.particles[f], got.particles[f]), (step, f)
    got = ref.arrays()
    # it came to rest on the colliders, above the terrain's lowest point
    assert got.particles["position"][:, 2].min() > -0.12


def test_fast_sheet_does_not_tunnel_through_a_mesh_floor():
    """cloth_collision_test.cpp:253-289 (mesh_collider_stops_tunnelling_through_the_solver): a 5 x 5
    sheet fired at -60 m/s onto a mesh floor stays above it, oracle and reference alike."""
    p = A.ClothParams.defaults()
    p.thickness = 0.03
    p.air_drag = 0.0
    p.air_lift = 0.0
    ref = K.RefCloth.make_grid(_grid(5, (0.0, 0.0, 1.0), 1.0, p))
    arr = ref.arrays()
    arr.particles["velocity"] = (0.0, 0.0, -60.0)
    ref = K.RefCloth.from_arrays(arr)
    orc = ref.arrays()
    K.register_geometry(12, S.floor_mesh())
    cols = collider_array([mesh_collider(12, S.floor_mesh())])
    for _ in range(120):
        ref.solve(cols, substeps=4, iterations=10)
        K.oracle_step_cloth(orc, cols, substeps=4, iterations=10)
    got = ref.arrays()
    assert same(orc.particles["position"], got.particles["position"])
    assert (got.particles["position"][:, 2] > 0.0).all()


def test_sheet_settles_on_mesh_floor_at_thickness():
    """cloth_collision_test.cpp:371-395: a 9 x 9 sheet settles on a mesh floor at the standoff."""
    p = A.ClothParams.defaults()
    p.thickness = 0.03
    ref = K.RefCloth.make_grid(_grid(9, (0.0, 0.0, 0.6), 2.0, p))
    orc = ref.arrays()
    K.register_geometry(12, S.floor_mesh())
    cols = collider_array([mesh_collider(12, S.floor_mesh())])
    for _ in range(300):
        ref.solve(cols, substeps=4, iterations=10)
        K.oracle_step_cloth(orc, cols, substeps=4, iterations=10)
    got = ref.arrays()
    assert same(orc.particles["position"], got.particles["position"])
    lowest = got.particles["position"][:, 2].min()
    assert lowest >= 0.0 and abs(lowest - 0.03) < 5e-3


def _grid(res, center, width, params):
    import ctypes as C
    d = A.GridClothDesc()
    d.columns = res
    d.rows = res
    d.width = width
    d.height = width
    d.center = (C.c_float * 3)(*center)
    d.orientation = (C.c_float * 4)(0, 0, 0, 1)
    d.total_mass = 1.0
    d.shear = 1
    d.params = params
    return d


def test_strands_over_a_mesh_and_hull_match_reference_bitwise():
    terrain = S.terrain_mesh(10, 1.0, 0.1, seed=2)
    rock = S.prism_hull(5, 0.1, 0.08)
    K.register_geometry(13, terrain)
    K.register_geometry(14, rock)
    cols = collider_array([mesh_collider(13, terrain, (0.0, 0.0, 0.0)),
                           hull_collider(14, rock, (0.05, 0.0, 0.1), unit((0.2, 0.1, 0.0, 0.97))),
                           sphere(0.05, (-0.1, 0.05, 0.1))])
    p = A.StrandParams.defaults()
    lines = [np.array([[0.02 * i - 0.1, 0.01 * i, 0.3 - 0.015 * k] for k in range(12)], np.float32) for i in range(9)]
    ref = K.RefStrands.make(lines, p)
    orc = ref.arrays(p)
    for _ in range(60):
        ref.solve(cols, substeps=4, iterations=4)
        K.oracle_step_strands(orc, cols, substeps=4, iterations=4)
    got = ref.arrays(p)
    for f in ("position", "velocity", "prev_position"):
        assert same(orc.particles[f], got.particles[f]), f


def grids():
    """Height grids of one coarse block, of several (the 64-cell blocks and the ragged 8-cell
    blocks at their edges), and flat with a spike (equal distances to many triangles)."""
    flat = np.zeros(24 * 20, np.float32)
    flat[10 * 24 + 11] = 0.3
    return {"small": S.height_grid_terrain(20, 17, 0.1, 0.15, seed=2),
            "multi_block": S.height_grid_terrain(140, 75, 0.02, 0.05, seed=3),
            "flat_spike": HeightGrid(24, 20, (0.05, 0.07), flat)}


@pytest.mark.parametrize("name", ["small", "multi_block", "flat_spike"])
def test_height_grid_projection_matches_reference(name):
    """TriangleMesh::from_height_grid (triangle_mesh.h:210-215): queries walk the grid's block
    pyramid (height_grid.h), not a MeshBVH; the oracle restates it and equals the reference."""
    grid = grids()[name]
    K.register_geometry(9, grid)
    rng = np.random.default_rng(13)
    lo, hi = grid.local_bounds()
    total = 0
    for q in QUATS[:2]:
        for scale in (1.0, 0.8):
            col = mesh_collider(9, grid, (0.1, -0.3, 0.05), unit(q), scale=scale, local_center=(-0.4, -0.3, 0.0))
            local = rng.uniform(lo - 0.04, hi + 0.04, (300, 3)).astype(np.float32)
            world = np.array([K_pose(col, p) for p in local], np.float32)
            total += compare(col, 0.04, world)
            d = rng.normal(size=(300, 3)).astype(np.float32)
            d /= np.linalg.norm(d, axis=1, keepdims=True)
            total += compare(col, 0.04, world, (world + 0.25 * d).astype(np.float32))
    assert total > 100


def test_cloth_on_height_grid_matches_reference_bitwise():
    sc = S.height_grid_drape(side=16, params=A.ClothParams.defaults())
    _register(sc)
    ref = K.RefCloth.from_arrays(sc.cloths[0])
    orc = sc.cloths[0].copy()
    cols = sc.colliders[0]
    for step in range(60):
        ref.solve(cols, substeps=4, iterations=6)
        K.oracle_step_cloth(orc, cols, substeps=4, iterations=6)
        if step % 20 == 19:
            got = ref.arrays()
            for f in ("position", "prev_position", "velocity"):
                assert same(orc.particles[f], got.particles[f]), (step, f)
    # it came to rest on the terrain
    assert ref.arrays().particles["position"][:, 2].min() > -0.2


def test_height_grid_floor_batch_matches_reference_bitwise():
    """The benchmark's height-grid floor (the 2048-triangle floor's 33 x 33 samples through
    TriangleMesh::from_height_grid) with sheets resting on it, under the reference's default
    parameters (no shear-compliance extension)."""
    sc = S.mesh_floor_batch(n=2, side=25, height_grid=True, params=A.ClothParams.defaults())
    _register(sc)
    for cloth, cols in zip(sc.cloths, sc.colliders):
        ref = K.RefCloth.from_arrays(cloth)
        orc = cloth.copy()
        for _ in range(20):
            ref.solve(cols, substeps=4, iterations=10)
            K.oracle_step_cloth(orc, cols, substeps=4, iterations=10)
        got = ref.arrays()
        for f in ("position", "prev_position", "velocity"):
            assert same(orc.particles[f], got.particles[f]), f
        assert got.particles["position"][:, 2].min() > -0.03
