"""General-topology cloths on the device (PxbClothDev::topology 1): cloths built from arbitrary
triangle meshes, and make_grid_cloth's lists in batches other than its own, stepped through the
C-ABI and compared bit for bit with the oracle, whose solve_cloth restatement is pinned to the
reference's on the same cloths (test_mesh_cloth_cpu.py)."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes as S
from physxcoopa_b200.arrays import collider_array, hull_collider, mesh_collider, sphere

import _checkers as K
from test_cloth_gpu import assert_equal_particles
from test_consumers_gpu import fnv1a, state_bytes, FNV_BASIS
from test_frame_oracle_ref import FIXED_DT, body_poses
from test_mesh_cloth_cpu import self_colliding_mesh, self_colliding_regrid, unbatched

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def run_against_oracle(ctx, cloths, cols, steps, check_every=10, iterations=10, graph=False, what=""):
    """Steps the cloths together on the device and one by one in the oracle; compares every
    particle every `check_every` steps and the compliant lists' lambdas at the end."""
    orc = [c.copy() for c in cloths]
    ids = [ctx.add_cloth(c) for c in cloths]
    try:
        d, keep = ctx.make_step(ids, cols, iterations=iterations)
        for s in range(steps):
            if graph:
                ctx.step_graph_desc(d)
            else:
                ctx.step_desc(d)
            for o, col in zip(orc, cols):
                K.oracle_step_cloth(o, col, iterations=iterations)
            if (s + 1) % check_every == 0 or s + 1 == steps:
                for k, (cid, o) in enumerate(zip(ids, orc)):
                    assert_equal_particles(ctx.read_particles(cid, len(o.particles)), o.particles,
                                           f"{what} cloth {k} step {s}")
        for cid, o in zip(ids, orc):
            ls, lb = ctx.read_lambdas(cid, len(o.stretch), len(o.bend))
            if o.params.stretch_compliance != 0.0 and o.stretch_batch_compliance is None:
                assert np.array_equal(ls, o.stretch["lambda"])
            if o.params.bend_compliance != 0.0 and o.bend_batch_compliance is None:
                assert np.array_equal(lb, o.bend["lambda"])
            res = ctx.read_results([cid])[0]
            assert np.array_equal(np.array(res["bounds_min"], np.float32), o.bounds[:3])
            assert np.array_equal(np.array(res["bounds_max"], np.float32), o.bounds[3:])
        del keep
    finally:
        for cid in ids:
            ctx.remove_cloth(cid)
    return orc


def test_mesh_drape_equals_oracle(ctx):
    sc = S.mesh_drape(rings=12, seed=1)
    assert R.plan_cloth(sc.cloths[0])["topology"] == 1
    run_against_oracle(ctx, sc.cloths, sc.colliders, steps=60, what="mesh drape")


def test_mesh_cloths_compliant_stretch_no_bend_and_aero(ctx):
    """Compliant stretch (lambdas kept for both lists), a bend-free mesh, strong wind with
    turbulence (the aerodynamic gather over the triangle index), several sizes in one launch."""
    p = S.cloth_params(stretch_compliance=2e-6, air_drag=0.3, air_lift=0.2, wind_turbulence=1.5)
    p.wind[0], p.wind[1] = 3.0, 1.0
    cloths = [S.mesh_cloth(r, 0.4, (1.5 * k, 0.0, 1.0), seed=r, params=p,
                           pins=[((1.5 * k - 0.4, 0.0, 1.0), 0.3 * 0.4 / r)], bend=(k != 1))
              for k, r in enumerate((5, 9, 16))]
    cols = [collider_array([sphere(0.15, (1.5 * k, 0.05, 0.7))]) for k in range(3)]
    run_against_oracle(ctx, cloths, cols, steps=40, what="aero")


@pytest.mark.parametrize("variant", ["serial", "shuffled", "triangles", "partial", "compliance"])
def test_grid_lists_in_other_batches_equal_oracle(ctx, variant):
    """make_grid_cloth's cloth with its lists walked in other ways: every list in one batch
    (serial Gauss-Seidel), the stretch list shuffled and re-coloured, the triangles wound the
    other way, half the bend batches dropped (those constraints are never solved), and per-batch
    compliance on re-coloured batches."""
    sc = S.single_drape(seed=2)
    g = sc.cloths[0]
    g.params.has_shear_compliance = 0
    g.stretch_batch_compliance = None
    if variant == "serial":
        c = unbatched(g)
    elif variant == "shuffled":
        c = g.copy()
        rng = np.random.default_rng(5)
        c.stretch = c.stretch[rng.permutation(len(c.stretch))].copy()
        c.stretch_batches = np.array([(0, len(c.stretch))], A.BATCH)
    elif variant == "triangles":
        c = g.copy()
        c.triangles = c.triangles.reshape(-1, 3)[:, [0, 2, 1]].reshape(-1).copy()
    elif variant == "partial":
        c = g.copy()
        c.bend_batches = c.bend_batches[::2].copy()
    else:
        c = unbatched(g)
        n = len(c.stretch)
        c.stretch_batches = np.array([(0, n // 3), (n // 3, n)], A.BATCH)
        c.stretch_batch_compliance = np.array([0.0, 3e-6], np.float32)
    assert R.plan_cloth(c)["topology"] == 1
    run_against_oracle(ctx, [c], sc.colliders, steps=30, what=variant)


def test_mesh_cloths_beside_grid_cloths_and_graph_replay(ctx):
    """General-topology and grid cloths in one step call, eager and replayed from the graph."""
    grid = S.single_drape(seed=3)
    mesh = S.mesh_drape(rings=10, seed=3)
    cloths = [grid.cloths[0], mesh.cloths[0], S.mesh_drape(rings=6, seed=4).cloths[0]]
    cols = [grid.colliders[0], mesh.colliders[0], mesh.colliders[0]]
    run_against_oracle(ctx, cloths, cols, steps=20, check_every=5, graph=True, what="graph")


def test_mesh_cloth_on_mesh_and_hull_colliders(ctx):
    """A mesh cloth dropped on a terrain mesh with a hull rock: the swept mesh query and the
    hull branch on the general-topology path."""
    terrain = S.terrain_mesh(16, 2.0, 0.1, seed=9)
    rock = S.prism_hull(6, 0.2, 0.12)
    sc = S.ClothScene("mesh on terrain", [S.mesh_cloth(10, 0.45, (0.0, 0.0, 0.35), seed=9)],
                      [collider_array([mesh_collider(1, terrain), hull_collider(2, rock, (0.1, 0.0, 0.1))])],
                      geometries=[terrain, rock])
    ids = S.register_geometries(ctx, sc)
    for gid, g in zip(ids, sc.geometries):
        K.register_geometry(gid, g)
    try:
        run_against_oracle(ctx, sc.cloths, sc.colliders, steps=45, check_every=15, what="terrain")
    finally:
        for gid in ids:
            ctx.destroy_geometry(gid)


def test_mesh_cloth_frames_follow_a_body(ctx):
    """pxb_cloths_step_frame on a mesh cloth pinned to a moving body."""
    h = R.HostCloth.from_mesh(*S.disc_mesh(0.4, 8, (0.0, 0.0, 2.0), jitter=0.2, seed=2),
                              params=S.cloth_params(damping=1.0))
    h.pin_to_body(0, 0, (0.0, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.4, 2.0), 0.12)
    c = h.arrays()
    cid = ctx.add_cloth(c)
    orc = c.copy()
    state = {"awake": 1, "sleep_timer": np.float32(0.0)}
    try:
        for frame in range(60):
            bodies = body_poses([((0.01 * frame, 0.0, 2.0), (0.0, 0.0, np.sin(0.01 * frame), np.cos(0.01 * frame)))])
            ctx.step_frame([cid], bodies, fixed_dt=FIXED_DT, cloth_substeps=4, cloth_iterations=3, dt=FIXED_DT)
            K.oracle_world_step_cloth(orc, state, bodies, fixed_dt=FIXED_DT, cloth_substeps=4, cloth_iterations=3,
                                      dt=FIXED_DT)
        assert_equal_particles(ctx.read_particles(cid, len(c.particles)), orc.particles, "frames")
        assert np.array_equal(ctx.read_anchors(cid, len(c.anchors)).view(np.uint8), orc.anchors.view(np.uint8))
    finally:
        ctx.remove_cloth(cid)


def render_restated(pos, triangles):
    """Vertex normals over an arbitrary triangle list in the device's float32 operation order:
    per particle, cross(b - a, c - a) of its triangles in ascending order, then v / |v|."""
    f = np.float32
    n = np.zeros((len(pos), 3), f)
    for t in triangles.reshape(-1, 3):
        a, b, c = (pos[int(i)] for i in t)
        u, v = b - a, c - a
        cr = np.array([u[1] * v[2] - v[1] * u[2], u[2] * v[0] - v[2] * u[0], u[0] * v[1] - v[0] * u[1]], f)
        for i in t:
            n[int(i)] = n[int(i)] + cr
    out = np.zeros((len(pos), 6), f)
    out[:, :3] = pos
    for i in range(len(pos)):
        l2 = f(f(n[i, 0] * n[i, 0] + n[i, 1] * n[i, 1]) + n[i, 2] * n[i, 2])
        s = f(1.0) / np.sqrt(l2) if l2 > 0 else f(0.0)
        out[i, 3:] = n[i] * s
    return out


def test_mesh_render_buffer_and_state_hash(ctx):
    sc = S.mesh_drape(rings=8, seed=6)
    c = sc.cloths[0]
    cid = ctx.add_cloth(c)
    orc = c.copy()
    try:
        flat = ctx.read_render_buffer([cid], len(c.particles))
        assert np.allclose(flat[:, 5], 1.0, atol=1e-3)  # a near-flat disc in the xy plane faces +z
        for _ in range(20):
            ctx.step([cid], sc.colliders)
            K.oracle_step_cloth(orc, sc.colliders[0])
        buf = ctx.read_render_buffer([cid], len(c.particles))
        pos = ctx.read_particles(cid, len(c.particles))["position"]
        assert np.array_equal(buf.view(np.uint32), render_restated(pos, c.triangles).view(np.uint32))
        assert ctx.state_hash([cid]) == fnv1a(FNV_BASIS, state_bytes(orc.particles))
    finally:
        ctx.remove_cloth(cid)


@pytest.mark.parametrize("scene", [self_colliding_mesh, self_colliding_regrid])
def test_self_collision_on_general_topology_equals_oracle(ctx, scene):
    """Self-collision (cloth_solver.h:291-366) on general-topology cloths in shared memory, pushes
    on every substep: the 1-ring exemption reads the cloth's own columns (0 for a mesh)."""
    c, col = scene()
    orc = run_against_oracle(ctx, [c], [col], steps=20, check_every=5, what=scene.__name__)
    off = c.copy()
    off.params.self_collision = 0
    for _ in range(20):
        K.oracle_step_cloth(off, col)
    assert not np.array_equal(off.particles["position"], orc[0].particles["position"])  # the stage acted


def test_general_topology_refusals(ctx):
    c = S.mesh_cloth(34, tethers=False)  # state in HBM: no shared memory for the hash tables
    c.params.self_collision = 1
    cid = ctx.add_cloth(c)
    try:
        with pytest.raises(R.PxbError) as e:
            ctx.step([cid])
        assert e.value.status == A.PXB_ERR_UNSUPPORTED
        p = A.ClothParams()
        A.C.pointer(p)[0] = c.params
        p.self_collision = 0
        ctx.set_params(cid, p)
        ctx.step([cid])  # steps once the stage is off
        with pytest.raises(R.PxbError) as e:
            ctx.step_warm([cid], warm_iterations=0)
        assert e.value.status == A.PXB_ERR_UNSUPPORTED
    finally:
        ctx.remove_cloth(cid)


def test_cloths_beyond_shared_memory_solve_in_hbm(ctx):
    """Mesh cloths whose state exceeds one CTA's shared memory (topology 2: positions, rest
    lengths and lambdas read in place in HBM) beside one that fits, equal to the oracle."""
    big = S.mesh_drape(rings=34, seed=5)
    huge = S.mesh_cloth(44, 0.6, (3.0, 0.0, 1.0), seed=6, pins=[((2.4, 0.0, 1.0), 0.3 * 0.6 / 44)])
    small = S.mesh_drape(rings=8, seed=7)
    assert R.plan_cloth(big.cloths[0])["topology"] == 2 and R.plan_cloth(huge)["topology"] == 2
    cloths = [big.cloths[0], huge, small.cloths[0]]
    cols = [big.colliders[0], collider_array([sphere(0.2, (3.0, 0.1, 0.6))]), small.colliders[0]]
    run_against_oracle(ctx, cloths, cols, steps=12, check_every=4, what="hbm")


def test_mesh_cloth_beyond_16_bit_slots_equals_oracle(ctx):
    """A mesh cloth of more than 65535 layout slots (a disc of 150 rings: 67,951 particles) keeps
    its constraint endpoints as two 32-bit words per item instead of one packed word; solved in
    HBM, equal to the oracle."""
    sc = S.mesh_drape(rings=150, seed=9)
    cloth = sc.cloths[0]
    assert len(cloth.particles) > 65535
    plan = R.plan_cloth(cloth)
    assert plan["topology"] == 2 and plan["layout_slots"] > 65535
    run_against_oracle(ctx, [cloth], [sc.colliders[0]], steps=3, check_every=3, what="wide")
