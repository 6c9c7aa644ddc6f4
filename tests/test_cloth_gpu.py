"""Parity of the device cloth solver with the oracle (oracle/xpbd_oracle.c).

Bars: pinned particles equal exactly; every particle within 1e-5 m after one step and within
1e-3 m after 300 steps. The kernel uses the reference's operation order with IEEE single
precision and no contraction, and the one reduction that feeds the solve (the cloth centre a
gravity source is evaluated at) is summed in the reference's sequential order, so every scene
here is also asserted EQUAL to the oracle, value for value.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes
from physxcoopa_b200.arrays import box, capsule, collider_array, gravity_sources, sphere

import _checkers as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def maxdiff(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)))) if a.size else 0.0


def assert_equal_particles(gpu, orc, what=""):
    for f in ("position", "velocity", "prev_position", "inv_mass"):
        x, y = gpu[f], orc[f]
        assert np.array_equal(x, y), f"{what} {f}: max |diff| {maxdiff(x, y)}"


def assert_pins_exact(gpu, orc):
    pinned = orc["inv_mass"] == 0.0
    assert np.array_equal(gpu["position"][pinned], orc["position"][pinned])


def run_pair(ctx, cloth, colliders=None, sources=None, steps=1, substeps=4, iterations=10,
             anchor_path=None):
    """Steps the same cloth on the device and in the oracle; returns (gpu particles, oracle)."""
    orc = cloth.copy()
    cid = ctx.add_cloth(cloth)
    try:
        for s in range(steps):
            if anchor_path is not None:
                w = anchor_path(s, orc.anchors["world_position"].copy())
                orc.anchors["world_position"] = w
                ctx.set_anchor_targets(cid, w)
            ctx.step([cid], None if colliders is None else [colliders],
                     sources=None if sources is None else [sources], substeps=substeps,
                     iterations=iterations)
            K.oracle_step_cloth(orc, colliders, sources=sources, substeps=substeps,
                                iterations=iterations)
        gpu = ctx.read_particles(cid, len(cloth.particles))
        res = ctx.read_results([cid])[0]
        lam = ctx.read_lambdas(cid, len(cloth.stretch), len(cloth.bend))
        t = ctx.read_time(cid)
    finally:
        ctx.remove_cloth(cid)
    return gpu, orc, res, lam, t


def test_single_drape_parity_1_and_300_steps(ctx):
    sc = scenes.single_drape(seed=0)
    cloth = sc.cloths[0]
    orc = cloth.copy()
    cid = ctx.add_cloth(cloth)
    ctx.step([cid], sc.colliders, substeps=4, iterations=10)
    K.oracle_step_cloth(orc, sc.colliders[0], substeps=4, iterations=10)
    gpu = ctx.read_particles(cid, len(cloth.particles))
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    assert_pins_exact(gpu, orc.particles)
    assert_equal_particles(gpu, orc.particles, "step 1")
    for _ in range(299):
        ctx.step([cid], sc.colliders, substeps=4, iterations=10)
        K.oracle_step_cloth(orc, sc.colliders[0], substeps=4, iterations=10)
    gpu = ctx.read_particles(cid, len(cloth.particles))
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-3
    assert_pins_exact(gpu, orc.particles)
    assert_equal_particles(gpu, orc.particles, "step 300")
    # the sheet really draped: it is below its start and outside the sphere
    centre = np.array([0, 0, 0.5], np.float32)
    assert np.all(np.linalg.norm(gpu["position"] - centre, axis=1) >= 0.3)
    assert gpu["position"][:, 2].min() < 0.5
    ctx.remove_cloth(cid)


def P(**kw):
    p = A.ClothParams.defaults()
    for k, v in kw.items():
        setattr(p, k, (A.C.c_float * 3)(*v) if isinstance(v, tuple) else v)
    return p


MATRIX = {
    "odd_5x5_sphere": dict(res=5, cols=[sphere(1.0, (0, 0, 0.6))]),
    "odd_13x13_capsule": dict(res=13, cols=[capsule(0.3, 0.5, (0, 0, 1.3), (0.2, 0.1, 0.0, 0.9746794))]),
    "rect_17x6_box": dict(res=(17, 6), cols=[box((0.6, 0.4, 0.3), (0.2, 0.0, 1.2), (0.0, 0.3826834, 0.0, 0.9238795))],
                          params=P(friction=0.9, thickness=0.05)),
    "three_colliders_22": dict(res=22, cols=[sphere(0.4, (-0.5, 0, 1.4)), capsule(0.2, 0.4, (0.6, 0, 1.5), axis=0),
                                             box((0.3, 0.3, 0.3), (0, 0.8, 1.4))]),
    "wind_turbulence_9": dict(res=9, params=P(wind=(0.4, 0.0, 0.1), wind_turbulence=0.6)),
    "no_shear_10": dict(res=10, shear=False, cols=[sphere(0.5, (0, 0, 1.3))]),
    "swept_colliders_8": dict(res=8, cols=[sphere(0.6, (0, -1, 1.3), sweep=(0, 1.0, 0)),
                                           box((0.3, 0.3, 0.3), (0.5, 0, 1.5), sweep=(0.2, 0, 0),
                                               end_orientation=(0, 0, 0.2588190, 0.9659258))]),
    "substep_override_6": dict(res=6, params=P(substeps=2, iterations=3)),
    "max_velocity_4": dict(res=4, params=P(max_velocity=0.5)),
    "pinned_tethered_11": dict(res=11, params=P(external_acceleration=(200.0, 0.0, 0.0)),
                               pins=[((0, 0, 2), 0.5)], tethers=True),
    "no_aero_2x2": dict(res=2, params=P(air_drag=0.0, air_lift=0.0), cols=[sphere(1.0, (0, 0, 0.5))]),
    "edge_pinned_64": dict(res=64, pins="edge", tethers=True, cols=[sphere(0.4, (0.1, 0.0, 1.3))],
                           params=scenes.cloth_params()),
}


@pytest.mark.parametrize("name", sorted(MATRIX))
def test_scene_matrix_equals_oracle(ctx, name):
    sc = MATRIX[name]
    res = sc["res"]
    cols_n, rows_n = (res, res) if isinstance(res, int) else res
    width = 4.0 if cols_n < 40 else 0.05 * (cols_n - 1)
    h = R.HostCloth(cols_n, rows_n, width, 4.0 if rows_n < 40 else 0.05 * (rows_n - 1),
                    center=(0, 0, 2), shear=sc.get("shear", True), params=sc.get("params"),
                    jitter=1e-3, seed=5)
    pins = sc.get("pins", [])
    if pins == "edge":
        arr = h.arrays()
        top = arr.particles["position"][(rows_n - 1) * cols_n:]
        pins = [(tuple(p), 0.01) for p in top]
    for p, r in pins:
        h.pin_static(p, r)
    if sc.get("tethers"):
        h.build_tethers()
    cloth = h.arrays()
    cols = collider_array(sc["cols"]) if sc.get("cols") else None
    gpu, orc, res_, lam, t = run_pair(ctx, cloth, cols, steps=25, iterations=4)
    assert_equal_particles(gpu, orc.particles, name)
    assert np.float32(t) == np.float32(orc.time)
    # per-cloth results: bounds and max speed (cloth.h:319-336)
    assert np.array_equal(res_["bounds_min"], orc.bounds[:3])
    assert np.array_equal(res_["bounds_max"], orc.bounds[3:])
    assert np.float32(res_["max_speed"]) == K.oracle().orc_max_particle_speed(
        A.ptr(orc.particles), len(orc.particles))
    # lambdas of compliant batches (zero-compliance batches keep none on the device)
    bend_comp = cloth.params.bend_compliance
    if bend_comp != 0.0:
        assert np.array_equal(lam[1], orc.bend["lambda"])


def test_moving_anchor_follows_targets(ctx):
    """A kinematic anchor target moving every frame (cloth_solver_test.cpp:190-233)."""
    h = R.HostCloth(15, 15, 4.0, 4.0, center=(0, 0, 4.05))
    h.pin_static((0, 0, 4.0), 0.4)
    h.build_tethers()
    cloth = h.arrays()
    col = collider_array([sphere(1.0, (0, 0, 3))])

    def path(s, w):
        w[:, 0] += 4.0 * (1 / 60) * (0.9 if s % 2 == 0 else 1.1)
        return w
    gpu, orc, _, _, _ = run_pair(ctx, cloth, col, steps=40, iterations=1, anchor_path=path)
    assert_equal_particles(gpu, orc.particles, "moving anchor")
    anc = orc.anchors
    np.testing.assert_array_equal(gpu["position"][anc["particle"]], anc["world_position"])


def test_gravity_sources_equal_oracle(ctx):
    """Gravity from a source evaluated at the cloth's mean position (world.h:1833, 2048-2076).
    The device sums the centre in the reference's sequential order, so even this chaotic drape
    (an unpinned sheet sliding off a sphere) stays equal to the oracle."""
    h = R.HostCloth(20, 20, 2.0, 2.0, center=(0, 0, 2), jitter=1e-3, seed=3)
    cloth = h.arrays()
    src = gravity_sources([((0.3, -0.2, -1.0), 9.81, 1.0, 10.0), ((5.0, 0.0, 0.0), 20.0, 0.5, 3.0)])
    col = collider_array([sphere(0.5, (0, 0, 1.0))])
    gpu, orc, _, _, _ = run_pair(ctx, cloth, col, sources=src, steps=1)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    assert_equal_particles(gpu, orc.particles, "sources, 1 step")
    gpu, orc, _, _, _ = run_pair(ctx, cloth, col, sources=src, steps=120)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-3
    assert_equal_particles(gpu, orc.particles, "sources, 120 steps")


def test_kernel_variants_agree_and_autotune_restores_state(ctx):
    """Every block-size variant in both launch forms (one CTA per cloth; persistent CTAs popping
    a work queue) gives the same bits; the autotuner leaves the cloths where they were."""
    sc = scenes.uniform_batch(n=6, side=40, seed=4)
    outs = []
    for mode in (0, 1):
        for variant in range(3):
            ids = [ctx.add_cloth(c) for c in sc.cloths]
            ctx.set_cloth_variant(variant)
            ctx.set_launch_mode(mode)
            for _ in range(5):
                ctx.step(ids, sc.colliders)
            outs.append([ctx.read_particles(i, len(c.particles)).tobytes() for i, c in zip(ids, sc.cloths)])
            for i in ids:
                ctx.remove_cloth(i)
    assert all(o == outs[0] for o in outs)
    ctx.set_launch_mode(1)
    ids = [ctx.add_cloth(c) for c in sc.cloths]
    d, keep = ctx.make_step(ids, sc.colliders)
    best, ms = ctx.autotune(d, trials=2)
    assert best in range(6) and len(ms) == 6 and all(m > 0 for m in ms)
    for i, c in zip(ids, sc.cloths):  # tuning did not advance the cloths
        assert np.array_equal(ctx.read_particles(i, len(c.particles))["position"], c.particles["position"])
        assert ctx.read_time(i) == np.float32(c.time)
    for _ in range(5):
        ctx.step_desc(d)
    assert [ctx.read_particles(i, len(c.particles)).tobytes() for i, c in zip(ids, sc.cloths)] == outs[0]
    for i in ids:
        ctx.remove_cloth(i)
    ctx.set_cloth_variant(0)


def test_batch_of_mixed_sizes_in_one_call(ctx):
    cloths, cols = [], []
    for k, side in enumerate([5, 16, 33, 64, 2, 47]):
        h = R.HostCloth(side, side, 0.05 * (side - 1), 0.05 * (side - 1), center=(0, 0, 1),
                        params=scenes.cloth_params(), jitter=1e-3, seed=k)
        half = 0.05 * (side - 1) / 2
        h.pin_static((-half, half, 1), 0.02)
        h.pin_static((half, half, 1), 0.02)
        h.build_tethers()
        cloths.append(h.arrays())
        cols.append(collider_array([sphere(0.2 + 0.05 * k, (0.05 * k, 0, 0.6))]))
    orcs = [c.copy() for c in cloths]
    ids = [ctx.add_cloth(c) for c in cloths]
    n0 = ctx.launch_count
    for _ in range(10):
        ctx.step(ids, cols, substeps=4, iterations=10)
        for o, c in zip(orcs, cols):
            K.oracle_step_cloth(o, c, substeps=4, iterations=10)
    # one launch per (cluster size, CTAs per SM) group: at most one per cloth, fewer here
    assert 10 <= ctx.launch_count - n0 < 10 * len(cloths)
    total = sum(len(c.particles) for c in cloths)
    out = np.zeros(3 * total, np.float32)
    ctx.read_positions(ids, out)
    off = 0
    for cid, o in zip(ids, orcs):
        g = ctx.read_particles(cid, len(o.particles))
        assert_equal_particles(g, o.particles, f"cloth {cid}")
        n = len(o.particles)
        assert np.array_equal(out[off:off + 3 * n].reshape(-1, 3), o.particles["position"])
        off += 3 * n
    for cid in ids:
        ctx.remove_cloth(cid)


def test_uniform_batch_config_sample_equals_oracle(ctx):
    sc = scenes.uniform_batch(n=8, side=64, seed=1)
    orcs = [c.copy() for c in sc.cloths]
    ids = [ctx.add_cloth(c) for c in sc.cloths]
    for _ in range(3):
        ctx.step(ids, sc.colliders, substeps=4, iterations=10)
        for o, c in zip(orcs, sc.colliders):
            K.oracle_step_cloth(o, c, substeps=4, iterations=10)
    for cid, o in zip(ids, orcs):
        assert_equal_particles(ctx.read_particles(cid, len(o.particles)), o.particles, "uniform")
        ctx.remove_cloth(cid)


def test_drop_in_solve_cloth_on_host_arrays(ctx):
    h = R.HostCloth(12, 12, 2.0, 2.0, center=(0, 0, 2), params=scenes.cloth_params(),
                    jitter=1e-3, seed=9)
    h.pin_static((-1, 1, 2), 0.05)
    h.build_tethers()
    mine = h.arrays()
    orc = mine.copy()
    col = collider_array([capsule(0.3, 0.4, (0, 0, 1.4), axis=0)])
    for _ in range(12):
        ctx.solve_cloth_host(mine, col, substeps=4, iterations=6)
        K.oracle_step_cloth(orc, col, substeps=4, iterations=6)
    assert_equal_particles(mine.particles, orc.particles, "drop-in")
    assert np.array_equal(mine.bend["lambda"], orc.bend["lambda"])
    sb = mine.stretch_batches
    for b, comp in enumerate(mine.stretch_batch_compliance):
        if comp != 0.0:
            s, e = sb[b]["begin"], sb[b]["end"]
            assert np.array_equal(mine.stretch["lambda"][s:e], orc.stretch["lambda"][s:e])
    assert np.array_equal(mine.anchors["prev_world_position"], orc.anchors["prev_world_position"])
    assert np.float32(mine.time) == np.float32(orc.time)
    assert np.array_equal(mine.bounds, orc.bounds)


def test_project_particles_known_answers_and_random(ctx):
    hit, p, n, d = ctx.project_particles(sphere(1.0), 0.03, [(0.5, 0, 0), (2.0, 0, 0)])
    assert list(hit) == [1, 0]
    np.testing.assert_allclose(p[0], (1.03, 0, 0), atol=1e-5)
    np.testing.assert_allclose(n[0], (1, 0, 0), atol=1e-5)
    assert abs(d[0] - 0.53) < 1e-5
    rng = np.random.default_rng(4)
    pts = rng.uniform(-1.2, 1.2, size=(500, 3)).astype(np.float32)
    for col in (sphere(0.7, (0.1, 0.2, 0.3)), capsule(0.25, 0.6, orientation=(0.1, 0.7, 0.1, 0.7), axis=1),
                box((0.4, 0.2, 0.6), (0, 0, 0.2), (0.3, 0.1, 0.2, 0.9273618)),
                box((0.4, 0.2, 0.6), sweep=(0.3, 0, 0), end_orientation=(0, 0, 0.3826834, 0.9238795)),
                sphere(0.5, sweep=(0.5, 0.2, 0.0))):
        hit, p, n, d = ctx.project_particles(col, 0.03, pts)
        for i in range(len(pts)):
            r = K.oracle_project(col, 0.03, pts[i])
            assert hit[i] == r[0]
            if r[0]:
                assert np.array_equal(p[i], r[1]) and np.array_equal(n[i], r[2]) and d[i] == r[3]


def test_refusals_and_handles(ctx):
    p = A.ClothParams.defaults()
    p.self_collision = 1
    p.self_distance = 0.1
    big = R.HostCloth(100, 100, 5.0, 5.0, params=p).arrays()  # a cluster: no self-collision there
    bid = ctx.add_cloth(big)
    with pytest.raises(R.PxbError) as e:
        ctx.step([bid])
    assert e.value.status == 2  # UNSUPPORTED: no CPU fallback
    ctx.remove_cloth(bid)
    ok = R.HostCloth(5, 5, 1.0, 1.0).arrays()
    cid = ctx.add_cloth(ok)
    mesh = np.zeros(1, A.COLLIDER)
    mesh["type"] = A.SHAPE_TRIANGLE_MESH
    mesh["enabled"] = 1
    mesh["geometry"] = 999  # no such registered geometry
    with pytest.raises(R.PxbError) as e:
        ctx.step([cid], [mesh])
    assert e.value.status == 5
    ctx.remove_cloth(cid)
    with pytest.raises(R.PxbError) as e:
        ctx.step([cid])
    assert e.value.status == 5  # stale handle
    past = ok.copy()
    past.bend_batches = past.bend_batches.copy()
    past.bend_batches[0]["end"] = len(past.bend) + 1  # a batch past its list
    with pytest.raises(R.PxbError) as e:
        ctx.add_cloth(past)
    assert e.value.status == 2
    empty = ok.copy()
    empty.particles = empty.particles[:0]
    with pytest.raises(R.PxbError) as e:
        ctx.add_cloth(empty)
    assert e.value.status == 1


def test_two_runs_are_bitwise_identical(ctx):
    sc = scenes.uniform_batch(n=4, side=48, seed=3)
    outs = []
    for _ in range(2):
        ids = [ctx.add_cloth(c) for c in sc.cloths]
        for _ in range(20):
            ctx.step(ids, sc.colliders)
        outs.append([ctx.read_particles(i, len(c.particles)).tobytes() for i, c in zip(ids, sc.cloths)])
        for i in ids:
            ctx.remove_cloth(i)
    assert outs[0] == outs[1]


def test_reference_drape_pin_through_the_device(ctx):
    """cloth_collision_test.cpp:27-64 on the device path: no particle inside the sphere,
    stretch < 1.25, and the sheet wraps below the centre."""
    centre = np.array([0, 0, 3], np.float32)
    h = R.HostCloth(21, 21, 4.0, 4.0, center=tuple(centre + (0, 0, 1.05)))
    h.pin_static(tuple(centre + (0, 0, 1.05)), 0.4)
    h.build_tethers()
    c = h.arrays()
    cid = ctx.add_cloth(c)
    col = collider_array([sphere(1.0, tuple(centre))])
    for _ in range(300):
        ctx.step([cid], [col], substeps=4, iterations=1)
    g = ctx.read_particles(cid, len(c.particles))
    pos = g["position"]
    assert np.all(np.linalg.norm(pos - centre, axis=1) >= 1.0)
    st = c.stretch
    assert (np.linalg.norm(pos[st["a"]] - pos[st["b"]], axis=1) / st["rest_length"]).max() < 1.25
    assert ctx.read_results([cid])[0]["bounds_min"][2] < centre[2]
    ctx.remove_cloth(cid)


# --- cloths split over a thread-block cluster --------------------------------------------------

def clustered_sheet(cols, rows, seed, pins="corners", params=None):
    w, hgt = 0.05 * (cols - 1), 0.05 * (rows - 1)
    h = R.HostCloth(cols, rows, w, hgt, center=(0, 0, 1), params=params or scenes.cloth_params(),
                    jitter=1e-3, seed=seed)
    arr = h.arrays()
    if pins == "edge":
        for p in arr.particles["position"][(rows - 1) * cols:]:
            h.pin_static(tuple(p), 0.01)
    else:
        h.pin_static((-w / 2, hgt / 2, 1), 0.02)
        h.pin_static((w / 2, hgt / 2, 1), 0.02)
    h.build_tethers()
    return h.arrays()


CLUSTERED = {
    # (columns, rows) and the layout the planner gives: (CTAs, lean). Lean: only the positions in
    # shared memory, rest lengths and lambdas read in place in HBM; lean 2: as float arrays.
    "lean1_65": dict(shape=(65, 65), layout=(1, 1), cols=[sphere(0.5, (0.1, 0, 0.4))]),
    "lean1_100_sources": dict(shape=(100, 100), layout=(1, 1), cols=[capsule(0.2, 0.5, (0, 0, 0.5), axis=0)],
                              sources=[((0.5, -0.3, -2.0), 9.81, 1.0, 10.0)]),
    "arrays_128_edge": dict(shape=(128, 128), layout=(1, 2), pins="edge",
                           cols=[box((0.6, 0.5, 0.4), (0.2, 0.1, 0.3), (0.0, 0.3826834, 0.0, 0.9238795))]),
    "lean1_tall_40x180": dict(shape=(40, 180), layout=(1, 1), cols=[sphere(0.6, (0, 0.5, 0.2))]),
    "arrays_wind_150x97": dict(shape=(150, 97), layout=(1, 2), params=dict(wind=(0.5, 0.2, 0.0), wind_turbulence=0.5)),
    "lean2_wind_150x130": dict(shape=(150, 130), layout=(2, 1), params=dict(wind=(0.5, 0.2, 0.0), wind_turbulence=0.5)),
    "c8_160": dict(shape=(160, 160), layout=(8, 0), cols=[sphere(0.8, (0, 0, 0.2))]),
}


@pytest.mark.parametrize("name", sorted(CLUSTERED))
def test_clustered_cloth_equals_oracle(ctx, name):
    """Cloths too large for one CTA's shared memory run lean (positions only in shared memory) on
    one CTA or two, or on a cluster of CTAs (rows split, the neighbour rows read through
    distributed shared memory); results equal the oracle's."""
    sc = CLUSTERED[name]
    params = scenes.cloth_params(**{k: (A.C.c_float * 3)(*v) if isinstance(v, tuple) else v
                                    for k, v in sc.get("params", {}).items()})
    cloth = clustered_sheet(*sc["shape"], seed=11, pins=sc.get("pins", "corners"), params=params)
    plan = R.plan_cloth(cloth)
    assert (plan["n_ranks"], plan["lean"]) == sc["layout"], plan
    cols = collider_array(sc["cols"]) if sc.get("cols") else None
    src = gravity_sources(sc["sources"]) if sc.get("sources") else None
    gpu, orc, res_, lam, t = run_pair(ctx, cloth, cols, sources=src, steps=1)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    assert_pins_exact(gpu, orc.particles)
    gpu, orc, res_, lam, t = run_pair(ctx, cloth, cols, sources=src, steps=30)
    assert_equal_particles(gpu, orc.particles, name)
    assert np.float32(t) == np.float32(orc.time)
    assert np.array_equal(res_["bounds_min"], orc.bounds[:3])
    assert np.array_equal(res_["bounds_max"], orc.bounds[3:])
    assert np.float32(res_["max_speed"]) == K.oracle().orc_max_particle_speed(
        A.ptr(orc.particles), len(orc.particles))
    assert np.array_equal(lam[1], orc.bend["lambda"])
    # stretch list: structural batches (compliance 0, no lambda kept on the device) and shear
    # batches (compliance 1e-6), compared where the batch is compliant
    keep = compliant_mask(cloth.stretch_batches, cloth.stretch_batch_compliance, len(cloth.stretch))
    assert keep.any() and not keep.all()
    assert np.array_equal(lam[0][keep], orc.stretch["lambda"][keep])
    assert not lam[0][~keep].any()


def compliant_mask(batches, compliance, n):
    m = np.zeros(n, bool)
    for b, c in zip(batches, compliance):
        if c != 0.0:
            m[b["begin"]:b["end"]] = True
    return m


def test_batch_of_every_cluster_size(ctx):
    """One step call over cloths of every layout (one CTA, lean on one CTA as float4 or as float
    arrays or on two CTAs, a cluster of eight): at least one launch per layout and at most one per
    cloth (a launch groups cloths of one layout and residency), all equal to the oracle, positions
    gathered in the caller's order."""
    shapes = [(20, 20), (128, 128), (64, 64), (65, 65), (100, 100), (16, 16), (150, 130), (160, 160)]
    cloths = [clustered_sheet(c, r, seed=k) for k, (c, r) in enumerate(shapes)]
    sizes = {(R.plan_cloth(c)["n_ranks"], R.plan_cloth(c)["lean"]) for c in cloths}
    assert sizes == {(1, 0), (1, 1), (1, 2), (2, 1), (8, 0)}
    cols = [collider_array([sphere(0.3 + 0.05 * k, (0.05 * k, 0, 0.4))]) for k in range(len(cloths))]
    orcs = [c.copy() for c in cloths]
    ids = [ctx.add_cloth(c) for c in cloths]
    n0 = ctx.launch_count
    for _ in range(5):
        ctx.step(ids, cols)
        for o, c in zip(orcs, cols):
            K.oracle_step_cloth(o, c, substeps=4, iterations=10)
    assert 5 * len(sizes) <= ctx.launch_count - n0 <= 5 * len(cloths)
    total = sum(len(c.particles) for c in cloths)
    out = np.zeros(3 * total, np.float32)
    ctx.read_positions(ids, out)
    res = ctx.read_results(ids)
    off = 0
    for k, (cid, o) in enumerate(zip(ids, orcs)):
        g = ctx.read_particles(cid, len(o.particles))
        assert_equal_particles(g, o.particles, f"cloth {shapes[k]}")
        n = len(o.particles)
        assert np.array_equal(out[off:off + 3 * n].reshape(-1, 3), o.particles["position"])
        assert np.array_equal(res[k]["bounds_min"], o.bounds[:3])
        off += 3 * n
    for cid in ids:
        ctx.remove_cloth(cid)



# --- cloths beyond a cluster: every SM on one cloth, state in global memory ---------------------

def test_whole_gpu_cloth_equals_oracle(ctx):
    """A 200 x 200 sheet (beyond an 8-CTA cluster) with a gravity source and a box: the
    cooperative whole-GPU kernel equals the oracle, value for value, with lambdas and results."""
    cloth = clustered_sheet(200, 200, seed=21, pins="edge")
    assert R.plan_cloth(cloth)["n_ranks"] == 0
    cols = collider_array([box((0.8, 0.6, 0.5), (0.3, 0.1, -0.2), (0.0, 0.3826834, 0.0, 0.9238795))])
    src = gravity_sources([((0.5, -0.3, -3.0), 9.81, 1.0, 10.0)])
    gpu, orc, res_, lam, t = run_pair(ctx, cloth, cols, sources=src, steps=3)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    assert_pins_exact(gpu, orc.particles)
    assert_equal_particles(gpu, orc.particles, "200x200")
    assert np.array_equal(res_["bounds_min"], orc.bounds[:3])
    assert np.array_equal(res_["bounds_max"], orc.bounds[3:])
    assert np.float32(res_["max_speed"]) == K.oracle().orc_max_particle_speed(
        A.ptr(orc.particles), len(orc.particles))
    assert np.array_equal(lam[1], orc.bend["lambda"])


def test_large_cloth_512_one_step_equals_oracle(ctx):
    """The large-cloth configuration's sheet: 512 x 512, 20 iterations, draped on a capsule."""
    cloth = clustered_sheet(512, 512, seed=3)
    cols = collider_array([capsule(0.4, 3.0, (0.0, 0.0, 0.4), axis=0)])
    gpu, orc, res_, lam, t = run_pair(ctx, cloth, cols, steps=1, iterations=20)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    assert_pins_exact(gpu, orc.particles)
    assert_equal_particles(gpu, orc.particles, "512x512")


def test_batch_with_a_whole_gpu_cloth(ctx):
    """Whole-GPU and shared-memory cloths in one step call."""
    cloths = [clustered_sheet(c, c, seed=k) for k, c in enumerate((30, 190, 70))]
    cols = [collider_array([sphere(0.4, (0.0, 0.0, 0.4))]) for _ in cloths]
    orcs = [c.copy() for c in cloths]
    ids = [ctx.add_cloth(c) for c in cloths]
    for _ in range(2):
        ctx.step(ids, cols)
        for o, c in zip(orcs, cols):
            K.oracle_step_cloth(o, c, substeps=4, iterations=10)
    res = ctx.read_results(ids)
    for k, (cid, o) in enumerate(zip(ids, orcs)):
        assert_equal_particles(ctx.read_particles(cid, len(o.particles)), o.particles, f"cloth {k}")
        assert np.array_equal(res[k]["bounds_max"], o.bounds[3:])
    for cid in ids:
        ctx.remove_cloth(cid)


def test_graph_steps_equal_eager_steps(ctx):
    """pxb_cloths_step_graph: captured on the second call of a shape, replayed after; results
    identical to pxb_cloths_step across cluster sizes and the whole-GPU path, recaptured when the
    shape changes (a cloth removed, another list)."""
    cloths = [clustered_sheet(c, c, seed=30 + k) for k, c in enumerate((12, 40, 64, 90, 130, 185))]
    cols = [collider_array([sphere(0.3, (0.02 * k, 0, 0.4))]) for k in range(len(cloths))]
    srcs = [gravity_sources([((0.5, 0.2, -2.0), 9.81, 1.0, 10.0)]) if k % 2 else None for k in range(len(cloths))]

    def trajectory(use_graph, steps=5):
        ids = [ctx.add_cloth(c) for c in cloths]
        d, keep = ctx.make_step(ids, cols, sources=srcs)
        out = []
        for _ in range(steps):
            (ctx.step_graph_desc if use_graph else ctx.step_desc)(d)
            out.append([ctx.read_particles(i, len(c.particles)).tobytes() for i, c in zip(ids, cloths)])
        ctx.remove_cloth(ids[0])
        d2, keep2 = ctx.make_step(ids[1:], cols[1:], sources=srcs[1:])
        for _ in range(3):
            (ctx.step_graph_desc if use_graph else ctx.step_desc)(d2)
        out.append([ctx.read_particles(i, len(c.particles)).tobytes() for i, c in zip(ids[1:], cloths[1:])])
        res = ctx.read_results(ids[1:]).tobytes()
        flat = np.zeros(3 * sum(len(c.particles) for c in cloths[1:]), np.float32)
        ctx.read_positions(ids[1:], flat)  # a launch after replays: no error left behind by them
        for i in ids[1:]:
            ctx.remove_cloth(i)
        del keep, keep2
        return out, res, flat.tobytes()

    eager = trajectory(False)
    graph = trajectory(True)
    assert graph == eager
