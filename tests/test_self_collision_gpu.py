"""Self-collision on the device (stage 6 of solve_cloth, cloth_solver.h:291-366) against the oracle,
which equals the compiled reference bit for bit on its self-collision scenes (test_oracle_ref.py).

The reference pass is serial (each push moves two particles before the next pair is tested);
the device keeps its order exactly (one warp walks the particles in index order over a hash
built in shared memory), so every scene here is asserted EQUAL to the oracle, plus the reference
tests' own properties: a collapsed blob is pushed apart (cloth_solver_test.cpp:246-295) and a
self-collision push cannot leave a particle inside a collider (cloth_collision_test.cpp:76-126).
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes as S
from physxcoopa_b200.arrays import capsule, collider_array, sphere

import _checkers as K
from test_cloth_gpu import assert_equal_particles, maxdiff

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def self_params(distance_scale=None, **kw):
    p = S.cloth_params(**kw)
    p.self_collision = 1
    p.self_distance = 0.0 if distance_scale is None else distance_scale * S.SPACING  # 0: the builder's 0.6 x spacing
    return p


def folding_sheet(side, distance_scale=2.2, seed=0):
    """A sheet pinned at two corners, blown by a gusting wind and draped over a thin capsule,
    with self_distance 2.2 x the spacing: particles two rows apart (0.1 m at rest) are closer
    than that, so the serial pushes run on every substep, against the constraints."""
    p = self_params(distance_scale, wind=(0.0, -3.0, 1.0), wind_turbulence=0.8)
    width = (side - 1) * S.SPACING
    h = R.HostCloth(side, side, width, width, center=(0.0, 0.0, 1.0), params=p, jitter=1e-3, seed=seed)
    h.pin_static((-width / 2, width / 2, 1.0), 0.3 * S.SPACING)
    h.pin_static((width / 2, width / 2, 1.0), 0.3 * S.SPACING)
    h.build_tethers()
    cols = collider_array([capsule(0.04, width, (0.0, 0.1 * width, 0.7), axis=0)])
    return h.arrays(), cols


def run_pair(ctx, cloth, cols, steps, iterations=10):
    orc = cloth.copy()
    cid = ctx.add_cloth(cloth)
    try:
        for _ in range(steps):
            ctx.step([cid], None if cols is None else [cols], iterations=iterations)
            K.oracle_step_cloth(orc, cols, iterations=iterations)
        gpu = ctx.read_particles(cid, len(cloth.particles))
    finally:
        ctx.remove_cloth(cid)
    return gpu, orc


@pytest.mark.parametrize("side", [9, 24, 48, 64, 80])
def test_folding_sheet_equals_oracle(ctx, side):
    """Up to 44 the sheet is all in shared memory. At 48 an SM would hold one CTA of the whole
    sheet but two of the lean one with its hash tables, so it is lean (positions only in shared
    memory, rest lengths and lambdas in HBM, the hash tables after the positions). At 64 the lean
    sheet with its tables leaves one CTA per SM too, so it stays whole. At 80 only the lean layout
    fits."""
    cloth, cols = folding_sheet(side)
    plan = R.plan_cloth(cloth)
    assert plan["n_ranks"] == 1 and plan["self_collision"] == 1 and plan["lean"] == (side in (48, 80))
    gpu, orc = run_pair(ctx, cloth, cols, 1)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    assert_equal_particles(gpu, orc.particles, "step 1")
    steps = 60 if side <= 24 else 25
    gpu, orc = run_pair(ctx, cloth, cols, steps)
    assert_equal_particles(gpu, orc.particles, f"step {steps}")
    # the stage did something: without it the same steps end elsewhere
    plain = cloth.copy()
    plain.params.self_collision = 0
    for _ in range(steps):
        K.oracle_step_cloth(plain, cols)
    assert maxdiff(plain.particles["position"], orc.particles["position"]) > 1e-4


def _cleared(side, p, center):
    """make_test_sheet with every constraint list cleared, as the reference's tests set it up."""
    c = R.HostCloth(side, side, 4.0, 4.0, center=center, params=p).arrays()
    for f in ("stretch", "bend", "stretch_batches", "bend_batches"):
        setattr(c, f, getattr(c, f)[:0].copy())
    return c


def _violations(pos, cols, d_min):
    n = len(pos)
    bad = 0
    for i in range(n):
        for j in range(i + 1, n):
            if abs(i % cols - j % cols) <= 1 and abs(i // cols - j // cols) <= 1:
                continue
            if np.linalg.norm(pos[i].astype(np.float64) - pos[j]) < d_min * 0.8:
                bad += 1
    return bad


def test_collapsed_blob_is_pushed_apart(ctx):
    """cloth_solver_test.cpp:246-295: every particle of a 9 x 9 sheet collapsed into a 1 cm blob,
    no constraints, no gravity: after 60 steps no non-neighbouring pair is closer than
    0.8 x self_distance with self-collision, and many are without it."""
    results = {}
    for on in (1, 0):
        p = A.ClothParams.defaults()
        p.self_collision = on
        p.gravity_scale = 0.0
        p.air_drag = 0.0
        p.air_lift = 0.0
        c = _cleared(9, p, (0.0, 0.0, 5.0))
        d_min = float(c.params.self_distance)
        assert d_min > 0.0  # derived from the grid spacing at build time
        f = np.arange(len(c.particles), dtype=np.float32) * np.float32(0.013)
        blob = np.stack([np.sin(f) * np.float32(0.01), np.cos(f) * np.float32(0.01),
                         np.float32(5.0) + np.sin(f * np.float32(2.0)) * np.float32(0.01)], 1).astype(np.float32)
        c.particles["position"] = blob
        c.particles["prev_position"] = blob
        c.particles["velocity"] = 0.0
        if on:
            plan = R.plan_cloth(c)
            assert plan["n_colours"] == 0 and plan["self_smem_bytes"] > plan["smem_bytes"]  # tables after the lambdas
        gpu, orc = run_pair(ctx, c, None, 60)
        assert_equal_particles(gpu, orc.particles, f"self_collision={on}")
        results[on] = _violations(gpu["position"], 9, d_min)
    assert results[1] == 0
    assert results[0] > 0


def test_self_collision_cannot_push_a_particle_into_a_collider(ctx):
    """cloth_collision_test.cpp:76-126: two non-neighbouring particles 2 cm apart just outside a
    sphere, self_distance 20 cm, one substep: they are pushed apart, and the collision stage (run
    after self-collision) leaves both at the full standoff outside the sphere."""
    p = A.ClothParams.defaults()
    p.self_collision = 1
    p.self_distance = 0.2
    p.gravity_scale = 0.0
    p.air_drag = 0.0
    p.air_lift = 0.0
    p.thickness = 0.03
    p.substeps = 1
    c = _cleared(9, p, (0.0, 0.0, 50.0))
    a, b = 0, 5 * 9 + 5
    for i, x in ((a, 1.06), (b, 1.04)):
        c.particles["position"][i] = (x, 0.0, 0.0)
        c.particles["prev_position"][i] = (x, 0.0, 0.0)
        c.particles["velocity"][i] = 0.0
    cols = collider_array([sphere(1.0)])
    gpu, orc = run_pair(ctx, c, cols, 1)
    assert_equal_particles(gpu, orc.particles, "one substep")
    pa, pb = gpu["position"][a].astype(np.float64), gpu["position"][b].astype(np.float64)
    assert np.linalg.norm(pa - pb) > 0.05
    assert np.linalg.norm(pa) >= 1.0 + 0.03 - 1e-4 and np.linalg.norm(pb) >= 1.0 + 0.03 - 1e-4


def test_mixed_batch_with_self_collision_and_plain_cloths(ctx):
    """Self-colliding cloths launch the extended kernel, the others the plain one, in one step;
    every cloth equals its oracle."""
    cloths, cols = [], []
    for k, side in enumerate((16, 32, 20)):
        c, col = folding_sheet(side, seed=k)
        cloths.append(c)
        cols.append(col)
    plain = S.single_drape(seed=4)
    cloths.append(plain.cloths[0])
    cols.append(plain.colliders[0])
    orcs = [c.copy() for c in cloths]
    ids = [ctx.add_cloth(c) for c in cloths]
    try:
        for _ in range(20):
            ctx.step(ids, cols)
            for o, col in zip(orcs, cols):
                K.oracle_step_cloth(o, col)
        for cid, c, o in zip(ids, cloths, orcs):
            assert_equal_particles(ctx.read_particles(cid, len(c.particles)), o.particles, "batch")
    finally:
        for cid in ids:
            ctx.remove_cloth(cid)


def test_enabling_self_collision_with_set_params(ctx):
    cloth, cols = folding_sheet(24, seed=7)
    cloth.params.self_collision = 0
    orc = cloth.copy()
    cid = ctx.add_cloth(cloth)
    try:
        for k in range(30):
            if k == 10:
                p = A.ClothParams()
                A.C.pointer(p)[0] = orc.params
                p.self_collision = 1
                ctx.set_params(cid, p)
                orc.params.self_collision = 1
            ctx.step([cid], [cols])
            K.oracle_step_cloth(orc, cols)
        assert_equal_particles(ctx.read_particles(cid, len(cloth.particles)), orc.particles, "after set_params")
    finally:
        ctx.remove_cloth(cid)
