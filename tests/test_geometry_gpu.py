"""Mesh and convex-hull colliders on the device, against the oracle (oracle/xpbd_oracle.c, itself
pinned bit for bit to the reference in test_geometry_oracle_ref.py).

The device evaluates the ConvexHull branch over a hull posed on the host once per step, and the
TriangleMesh branch over a hierarchy built on the host by MeshBVH::build's rule, walked in its
recursion order; both in the reference's operation order with IEEE single precision. So every
case here is asserted EQUAL to the oracle: the projection primitive on thousands of points, and
cloth and strand steps on every launch path (one CTA, a thread-block cluster, the whole-GPU
kernel, the captured graph).
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes as S
from physxcoopa_b200.arrays import Hull, collider_array, hull_collider, mesh_collider, sphere

import _checkers as K
from test_cloth_gpu import assert_equal_particles, maxdiff
from test_strands_oracle_ref import params, straight

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def register(ctx, geometry):
    gid = ctx.create_geometry(geometry)
    K.register_geometry(gid, geometry)
    return gid


def unit(q):
    q = np.asarray(q, np.float32)
    return tuple(float(x) for x in (q / np.float32(np.sqrt(np.dot(q, q)))).astype(np.float32))


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                          np.ascontiguousarray(b, np.float32).view(np.uint32))


def check_projection(ctx, col, thickness, pts, starts=None):
    hit, out, nrm, dep = ctx.project_particles(col, thickness, pts, starts)
    n_hit = 0
    for i, p in enumerate(pts):
        r, q, n, d = K.oracle_project(col, thickness, p, None if starts is None else starts[i])
        assert hit[i] == r, (i, p)
        if r == 1:
            n_hit += 1
            assert same(out[i], q) and same(nrm[i], n) and same(dep[i], d), (i, p, out[i], q)
    return n_hit


GEOMETRIES = {
    "prism7": lambda: S.prism_hull(7, 0.35, 0.25),
    "random_hull": lambda: S.random_hull(40, 0.4, seed=8),
    "floor": S.floor_mesh,
    "corner": S.corner_mesh,
    "terrain": lambda: S.terrain_mesh(20, 2.0, 0.2, seed=3),
    "terrain_computed_normals": lambda: S.terrain_mesh(9, 2.0, 0.3, seed=4),
    # TriangleMesh::from_height_grid: one 64-cell block; several, with ragged 8-cell blocks
    "height_grid": lambda: S.height_grid_terrain(20, 17, 0.1, 0.15, seed=2),
    "height_grid_blocks": lambda: S.height_grid_terrain(140, 75, 0.02, 0.05, seed=3),
}


@pytest.mark.parametrize("name", sorted(GEOMETRIES))
def test_projection_equals_oracle(ctx, name):
    g = GEOMETRIES[name]()
    if name == "terrain_computed_normals":
        g.normals = None
    gid = register(ctx, g)
    rng = np.random.default_rng(21)
    lo, hi = g.local_bounds()
    total = 0
    try:
        for q in [(0.0, 0.0, 0.0, 1.0), unit((0.1, 0.7, 0.1, 0.7))]:
            for scale in (1.0, 0.8):
                make = hull_collider if isinstance(g, Hull) else mesh_collider
                col = make(gid, g, (0.1, -0.2, 0.3), q, scale=scale, local_center=(0.02, 0.0, -0.01))
                from test_geometry_oracle_ref import K_pose
                local = rng.uniform(lo - 0.08, hi + 0.08, (1500, 3)).astype(np.float32)
                pts = np.array([K_pose(col, p) for p in local], np.float32)
                total += check_projection(ctx, col, 0.04, pts)
                d = rng.normal(size=pts.shape).astype(np.float32)
                d /= np.linalg.norm(d, axis=1, keepdims=True)
                total += check_projection(ctx, col, 0.04, pts, (pts + 0.25 * d).astype(np.float32))
    finally:
        ctx.destroy_geometry(gid)
    assert total > 200


def test_reference_mesh_known_answers_on_device(ctx):
    """cloth_collision_test.cpp:218-362 on the device primitive."""
    floor = register(ctx, S.floor_mesh())
    corner = register(ctx, S.corner_mesh())
    try:
        col = mesh_collider(floor, S.floor_mesh())
        pts = np.array([[0, 0, -0.5], [0, 0, 0.5], [0, 0, -0.01], [0, 0, 0.01], [0, 0, 0.10]], np.float32)
        st = np.array([[0, 0, 0.5], [0, 0, -0.5], [0, 0, -0.01], [0, 0, 0.01], [0, 0, 0.11]], np.float32)
        hit, out, nrm, _ = ctx.project_particles(col, 0.03, pts, st)
        assert list(hit) == [1, 1, 1, 1, 0]
        np.testing.assert_allclose(out[:4, 2], [0.03, -0.03, 0.03, 0.03], atol=1e-4)
        np.testing.assert_allclose(nrm[:4, 2], [1, -1, 1, 1], atol=1e-4)
        col = mesh_collider(corner, S.corner_mesh())
        hit, out, _, _ = ctx.project_particles(col, 0.03, np.array([[-0.002, 0, 0.02], [-0.002, 0, -0.002]], np.float32))
        assert list(hit) == [1, 1]
        assert out[0, 0] <= 0.0 and out[0, 2] >= 0.0
        assert out[1, 0] > 0.0 or out[1, 2] > 0.0
    finally:
        ctx.destroy_geometry(floor)
        ctx.destroy_geometry(corner)


def _scene_with_oracle(ctx, scene):
    ids = S.register_geometries(ctx, scene)
    for gid, g in zip(ids, scene.geometries):
        K.register_geometry(gid, g)
    return ids


def run_scene(ctx, scene, steps, iterations=10, graph=False):
    orc = [c.copy() for c in scene.cloths]
    ids = [ctx.add_cloth(c) for c in scene.cloths]
    try:
        d, keep = ctx.make_step(ids, scene.colliders, substeps=4, iterations=iterations)
        for _ in range(steps):
            if graph:
                ctx.step_graph_desc(d)
            else:
                ctx.step_desc(d)
            for c, cols in zip(orc, scene.colliders):
                K.oracle_step_cloth(c, cols, substeps=4, iterations=iterations)
        gpu = [ctx.read_particles(i, len(c.particles)) for i, c in zip(ids, scene.cloths)]
    finally:
        for i in ids:
            ctx.remove_cloth(i)
    return gpu, orc


def test_terrain_drape_equals_oracle_1_and_300_steps(ctx):
    sc = S.terrain_drape(side=32)
    gids = _scene_with_oracle(ctx, sc)
    try:
        gpu, orc = run_scene(ctx, sc, 1)
        assert maxdiff(gpu[0]["position"], orc[0].particles["position"]) <= 1e-5
        assert_equal_particles(gpu[0], orc[0].particles, "step 1")
        gpu, orc = run_scene(ctx, sc, 300)
        assert maxdiff(gpu[0]["position"], orc[0].particles["position"]) <= 1e-3
        assert_equal_particles(gpu[0], orc[0].particles, "step 300")
        # it came to rest on the terrain and the rock, nothing below the terrain's lowest point
        assert gpu[0]["position"][:, 2].min() > -0.12
    finally:
        for g in gids:
            ctx.destroy_geometry(g)


@pytest.mark.parametrize("side", [100, 128, 140, 160, 200])
def test_cluster_and_whole_gpu_paths_with_mesh_and_hull(ctx, side):
    """100 x 100 runs lean on one CTA, 128 x 128 lean on one CTA as float arrays, 140 x 140 lean
    on two CTAs, 160 x 160 on a cluster of eight, 200 x 200 on the whole-GPU kernel."""
    sc = S.terrain_drape(side=side, seed=5)
    plan = R.plan_cloth(sc.cloths[0])
    want = {100: (1, 1), 128: (1, 2), 140: (2, 1), 160: (8, 0), 200: (0, 0)}[side]
    assert (plan["n_ranks"], plan["lean"]) == want, plan
    gids = _scene_with_oracle(ctx, sc)
    try:
        gpu, orc = run_scene(ctx, sc, 3 if side == 200 else 12)
        assert_equal_particles(gpu[0], orc[0].particles, f"{side}^2")
    finally:
        for g in gids:
            ctx.destroy_geometry(g)


def test_graph_step_with_posed_hull_equals_eager(ctx):
    """The posed hull travels in the step's staging, which a captured graph re-uploads each replay:
    a rotating rock (new pose every step) through the graph equals the oracle."""
    rock = S.prism_hull(6, 0.3, 0.2)
    gid = register(ctx, rock)
    try:
        sc = S.single_drape(seed=3)
        cloth = sc.cloths[0]
        orc = cloth.copy()
        cid = ctx.add_cloth(cloth)
        try:
            for s in range(6):
                ang = 0.2 * s
                col = collider_array([hull_collider(gid, rock, (0.0, 0.05, 0.78), (0.0, 0.0, float(np.sin(ang / 2)),
                                                                                   float(np.cos(ang / 2))))])
                d, keep = ctx.make_step([cid], [col], substeps=4, iterations=10)
                ctx.step_graph_desc(d)
                K.oracle_step_cloth(orc, col, substeps=4, iterations=10)
            gpu = ctx.read_particles(cid, len(cloth.particles))
        finally:
            ctx.remove_cloth(cid)
        assert_equal_particles(gpu, orc.particles, "graph")
    finally:
        ctx.destroy_geometry(gid)


def test_strands_over_mesh_and_hull_equal_oracle(ctx):
    terrain = S.terrain_mesh(10, 1.0, 0.1, seed=2)
    rock = S.prism_hull(5, 0.1, 0.08)
    t_id, r_id = register(ctx, terrain), register(ctx, rock)
    try:
        cols = collider_array([mesh_collider(t_id, terrain),
                               hull_collider(r_id, rock, (0.05, 0.0, 0.1), unit((0.2, 0.1, 0.0, 0.97))),
                               sphere(0.05, (-0.1, 0.05, 0.1))])
        p = params(global_shape=0.0, local_shape=0.0)
        lines = [np.array([[0.02 * i - 0.1, 0.01 * i, 0.3 - 0.015 * k] for k in range(12)], np.float32)
                 for i in range(9)]
        s = R.make_strands(lines, p)
        orc = s.copy()
        sid = ctx.add_strands(s)
        try:
            for _ in range(60):
                ctx.step_strands([sid], [cols], iterations=4)
                K.oracle_step_strands(orc, cols, iterations=4)
            gpu = ctx.read_strand_particles(sid, len(s.particles))
        finally:
            ctx.remove_strands(sid)
        for f in ("position", "velocity", "prev_position"):
            assert np.array_equal(gpu[f], orc.particles[f]), f
    finally:
        ctx.destroy_geometry(t_id)
        ctx.destroy_geometry(r_id)


def test_geometry_refusals_and_lifetime(ctx):
    cloth = S.single_drape().cloths[0]
    cid = ctx.add_cloth(cloth)
    try:
        mesh = S.floor_mesh()
        gid = ctx.create_mesh(mesh)
        hid = ctx.create_hull(S.prism_hull())
        # a collider naming a hull id with the mesh type is refused
        with pytest.raises(R.PxbError) as e:
            ctx.step([cid], [collider_array([mesh_collider(hid, mesh)])])
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
        ctx.destroy_geometry(gid)
        with pytest.raises(R.PxbError) as e:
            ctx.step([cid], [collider_array([mesh_collider(gid, mesh)])])
        assert e.value.status == A.PXB_ERR_INVALID_HANDLE
        with pytest.raises(R.PxbError):
            ctx.destroy_geometry(gid)
        ctx.destroy_geometry(hid)
        # geometry 0 never collides, like a null Shape::mesh
        orc = cloth.copy()
        ctx.step([cid], [collider_array([mesh_collider(0, mesh)])])
        K.oracle_step_cloth(orc, collider_array([mesh_collider(0, mesh)]))
        assert np.array_equal(ctx.read_particles(cid, len(cloth.particles))["position"], orc.particles["position"])
    finally:
        ctx.remove_cloth(cid)
    bad = [Hull([[0, 0, 0]], np.zeros((0, 4)), [0], []),                           # no face
           Hull([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 0, 1, 0]], [0, 3], [0, 1, 5]),  # index out of range
           Hull([[0, 0, 0]], [[0, 0, 1, 0]], [0, 161], np.zeros(161))]                # face over 160 vertices
    for h in bad:
        with pytest.raises(R.PxbError) as e:
            ctx.create_hull(h)
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    from physxcoopa_b200.arrays import Mesh
    with pytest.raises(R.PxbError) as e:
        ctx.create_mesh(Mesh([[0, 0, 0]], [0, 0, 1]))
    assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    empty = ctx.create_mesh(Mesh(np.zeros((0, 3)), np.zeros(0)))  # accepted; never collides
    ctx.destroy_geometry(empty)


def test_height_grid_drape_equals_oracle_1_and_300_steps(ctx):
    """A cloth settling on TriangleMesh::from_height_grid: the device walks the grid's block
    pyramid in the reference's order (height_grid.h), so every step equals the oracle."""
    sc = S.height_grid_drape(side=24)
    gids = _scene_with_oracle(ctx, sc)
    try:
        gpu, orc = run_scene(ctx, sc, 1)
        assert_equal_particles(gpu[0], orc[0].particles, "step 1")
        gpu, orc = run_scene(ctx, sc, 300)
        assert maxdiff(gpu[0]["position"], orc[0].particles["position"]) <= 1e-3
        assert_equal_particles(gpu[0], orc[0].particles, "step 300")
        assert gpu[0]["position"][:, 2].min() > -0.2
    finally:
        for g in gids:
            ctx.destroy_geometry(g)
