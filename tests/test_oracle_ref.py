"""Pins the C restatement (oracle/xpbd_oracle.c) to the reference itself.

`oracle/_ref/libpxbref.so` is the reference's own cloth / hair headers compiled unmodified
against the glm-subset shim. The oracle must reproduce it BIT FOR BIT on every scene below:
same stage order, same operation order, same single-precision rounding. The reference's own
test known-answers (tests/cloth_solver_test.cpp, cloth_collision_test.cpp, gravity_test.cpp)
are re-expressed at the end against the oracle.
"""
import ctypes as C

import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200.arrays import box, capsule, collider_array, gravity_sources, sphere

import _checkers as K

pytestmark = pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")


def grid_desc(res, center=(0, 0, 2), width=4.0, height=4.0, params=None, shear=True, jitter=0.0,
              seed=7, orientation=(0, 0, 0, 1), mass=1.0):
    """cloth_fixtures.h make_test_sheet: a 4 x 4 m sheet, 1 kg (tests/support/cloth_fixtures.h:18-28)."""
    d = A.GridClothDesc()
    d.columns = res
    d.rows = res
    d.width = width
    d.height = height
    d.center = (C.c_float * 3)(*center)
    d.orientation = (C.c_float * 4)(*orientation)
    d.total_mass = mass
    d.shear = 1 if shear else 0
    d.params = params if params is not None else A.ClothParams.defaults()
    d.jitter = jitter
    d.jitter_seed = seed
    return d


def assert_cloth_bitwise(a, b):
    for f in ("position", "prev_position", "velocity", "inv_mass"):
        x, y = a.particles[f], b.particles[f]
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), \
            f"{f}: max |diff| {np.max(np.abs(x - y))}"
    assert np.array_equal(a.stretch["lambda"].view(np.uint32), b.stretch["lambda"].view(np.uint32))
    assert np.array_equal(a.bend["lambda"].view(np.uint32), b.bend["lambda"].view(np.uint32))
    assert np.array_equal(a.anchors.view(np.uint8), b.anchors.view(np.uint8))
    assert np.float32(a.time) == np.float32(b.time)
    assert np.array_equal(a.bounds, b.bounds)


# ------------------------------------------------------------------------------------------
# Builder topology (cloth_solver_test.cpp:35-76)
# ------------------------------------------------------------------------------------------

@pytest.mark.parametrize("res", [2, 3, 5, 9, 16])
def test_reference_grid_topology_and_disjoint_batches(res):
    c = K.RefCloth.make_grid(grid_desc(res)).arrays()
    assert len(c.particles) == res * res
    assert len(c.stretch) == 2 * (res - 1) * res + 2 * (res - 1) * (res - 1)
    assert len(c.bend) == 2 * max(res - 2, 0) * res
    assert len(c.triangles) == (res - 1) * (res - 1) * 6
    for lst, batches in ((c.stretch, c.stretch_batches), (c.bend, c.bend_batches)):
        covered = 0
        for b in batches:
            ks = lst[b["begin"]:b["end"]]
            ends = np.concatenate([ks["a"], ks["b"]])
            assert len(np.unique(ends)) == len(ends), "a batch shares a particle"
            covered += b["end"] - b["begin"]
        assert covered == len(lst)


# ------------------------------------------------------------------------------------------
# Oracle == reference, bit for bit
# ------------------------------------------------------------------------------------------

def _params(**kw):
    p = A.ClothParams.defaults()
    for k, v in kw.items():
        if isinstance(v, (tuple, list)):
            setattr(p, k, (C.c_float * len(v))(*v))
        else:
            setattr(p, k, v)
    return p


SCENES = {
    "plain_sphere": dict(res=9, params=_params(), colliders=[sphere(1.0, (0, 0, 0.5))]),
    "iterations_10_jitter": dict(res=12, params=_params(bend_compliance=1e-4), jitter=1e-3,
                                 colliders=[sphere(0.3, (0.1, -0.2, 1.5))], iterations=10),
    "no_aero_capsule": dict(res=8, params=_params(air_drag=0.0, air_lift=0.0),
                            colliders=[capsule(0.3, 0.5, (0, 0, 1.3), (0.2, 0.1, 0.0, 0.9746794))]),
    "rotated_box_friction": dict(res=10, params=_params(friction=0.9, thickness=0.05),
                                 colliders=[box((0.6, 0.4, 0.3), (0.2, 0.0, 1.2),
                                                (0.0, 0.3826834, 0.0, 0.9238795))]),
    "three_colliders": dict(res=11, colliders=[sphere(0.4, (-0.5, 0, 1.4)),
                                               capsule(0.2, 0.4, (0.6, 0, 1.5), axis=0),
                                               box((0.3, 0.3, 0.3), (0, 0.8, 1.4))]),
    "wind_turbulence": dict(res=7, params=_params(wind=(0.4, 0.0, 0.1), wind_turbulence=0.6)),
    "pinned_tethered": dict(res=11, params=_params(external_acceleration=(200.0, 0.0, 0.0)),
                            pin=[((0, 0, 2), 0.5)], tethers=True),
    "corners_pinned_sphere": dict(res=9, pin=[((-2, 2, 2), 0.1), ((2, 2, 2), 0.1)],
                                  tethers=True, colliders=[sphere(0.5, (0, 0, 1.4))]),
    "no_shear": dict(res=6, shear=False, colliders=[sphere(0.5, (0, 0, 1.3))]),
    "swept_colliders": dict(res=8, colliders=[sphere(0.6, (0, -1, 1.3), sweep=(0, 1.0, 0)),
                                              box((0.3, 0.3, 0.3), (0.5, 0, 1.5),
                                                  sweep=(0.2, 0, 0),
                                                  end_orientation=(0, 0, 0.2588190, 0.9659258))]),
    "substep_override": dict(res=6, params=_params(substeps=2, iterations=3)),
    "self_collision": dict(res=7, params=_params(self_collision=1),
                           colliders=[sphere(0.8, (0, 0, 1.0))]),
    "max_velocity_clamp": dict(res=5, params=_params(max_velocity=0.5)),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_oracle_matches_reference_bitwise(name):
    sc = SCENES[name]
    ref = K.RefCloth.make_grid(grid_desc(sc["res"], params=sc.get("params"),
                                         shear=sc.get("shear", True), jitter=sc.get("jitter", 0.0)))
    for point, radius in sc.get("pin", []):
        ref.pin_static(point, radius)
    if sc.get("tethers"):
        ref.build_tethers()
    orc = ref.arrays()
    cols = collider_array(sc.get("colliders", [])) if sc.get("colliders") else None
    iters = sc.get("iterations", 1)
    for step in range(25):
        ref.solve(cols, substeps=4, iterations=iters)
        K.oracle_step_cloth(orc, cols, substeps=4, iterations=iters)
        if step % 8 == 7:
            assert_cloth_bitwise(orc, ref.arrays())
    assert_cloth_bitwise(orc, ref.arrays())


def test_oracle_matches_reference_with_moving_anchor():
    """A kinematic anchor target that moves every frame (cloth_solver_test.cpp:190-233)."""
    ref = K.RefCloth.make_grid(grid_desc(9, center=(0, 0, 4.05)))
    ref.pin_static((0, 0, 4.05), 0.6)
    ref.build_tethers()
    for frame in range(20):
        arr = ref.arrays()
        arr.anchors["world_position"][:, 0] += 0.05  # the body moved 5 cm this frame
        ref = K.RefCloth.from_arrays(arr)
        orc = arr.copy()
        ref.solve(collider_array([sphere(1.0, (0, 0, 3))]), substeps=4, iterations=2)
        K.oracle_step_cloth(orc, collider_array([sphere(1.0, (0, 0, 3))]), substeps=4,
                            iterations=2)
        assert_cloth_bitwise(orc, ref.arrays())


# ------------------------------------------------------------------------------------------
# project_particle known answers (cloth_collision_test.cpp:135-217)
# ------------------------------------------------------------------------------------------

@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_still_sphere_projection_is_exact(impl):
    proj = K.oracle_project if impl == "oracle" else K.ref_project
    col = sphere(1.0)
    hit, p, n, d = proj(col, 0.03, (0.5, 0.0, 0.0))
    assert hit == 1
    np.testing.assert_allclose(p, (1.03, 0, 0), atol=1e-5)
    np.testing.assert_allclose(n, (1, 0, 0), atol=1e-5)
    assert abs(d - 0.53) < 1e-5
    hit, p, _, _ = proj(col, 0.03, (2.0, 0.0, 0.0))
    assert hit == 0
    np.testing.assert_allclose(p, (2, 0, 0), atol=1e-6)


@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_swept_collider_projects_out_of_the_motion_path(impl):
    proj = K.oracle_project if impl == "oracle" else K.ref_project
    still = sphere(1.0)
    hit, p, _, _ = proj(still, 0.03, (1.5, 0.5, 0.0))
    assert hit == 0
    moving = sphere(1.0, sweep=(2.0, 0.0, 0.0))
    hit, p, n, _ = proj(moving, 0.03, (1.5, 0.5, 0.0))
    assert hit == 1
    np.testing.assert_allclose(p, (1.5, 1.03, 0.0), atol=1e-5)
    np.testing.assert_allclose(n, (0, 1, 0), atol=1e-5)
    moving_box = box((0.5, 0.5, 0.5), sweep=(2.0, 0.0, 0.0))
    still_box = box((0.5, 0.5, 0.5))
    hit, _, _, _ = proj(still_box, 0.03, (1.52, 0.0, 0.0))
    assert hit == 0
    hit, b, n, _ = proj(moving_box, 0.03, (1.52, 0.0, 0.0))
    assert hit == 1
    assert abs(b[0] - (2.0 - 0.53)) < 1e-5
    np.testing.assert_allclose(n, (-1, 0, 0), atol=1e-5)


def test_projection_oracle_matches_reference_on_random_points():
    rng = np.random.default_rng(3)
    cols = [sphere(0.7, (0.1, 0.2, 0.3)),
            capsule(0.25, 0.6, (0.0, 0.1, 0.0), (0.1, 0.7, 0.1, 0.7), axis=1),
            capsule(0.2, 0.0, (0.3, 0.0, 0.0)),
            box((0.4, 0.2, 0.6), (0.0, 0.0, 0.2), (0.3, 0.1, 0.2, 0.9273618)),
            box((0.4, 0.2, 0.6), (0.0, 0.0, 0.2), sweep=(0.3, 0.0, 0.0),
                end_orientation=(0.0, 0.0, 0.3826834, 0.9238795))]
    for col in cols:
        for p in rng.uniform(-1.2, 1.2, size=(400, 3)).astype(np.float32):
            a = K.oracle_project(col, 0.03, p)
            b = K.ref_project(col, 0.03, p)
            assert a[0] == b[0]
            if a[0] == 1:
                for x, y in zip(a[1:], b[1:]):
                    assert np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))


# ------------------------------------------------------------------------------------------
# Gravity field (gravity_test.cpp:50-96, restated from world.h:2048-2068)
# ------------------------------------------------------------------------------------------

def _gravity_at(g, sources, p):
    out = (C.c_float * 3)()
    K.oracle().orc_gravity_at(K.vec(g), A.ptr(sources), len(sources), K.vec(p), out)
    return np.array(out[:], np.float32)


def test_gravity_sources_strongest_pulls_and_falloff():
    src = gravity_sources([((0, 0, 0), 9.81, 5.0, 40.0), ((30, 0, 0), 9.81, 5.0, 40.0)])
    assert _gravity_at((0, 0, 0), src, (10, 0, 0))[0] < 0
    assert _gravity_at((0, 0, 0), src, (22, 0, 0))[0] > 0
    assert abs(np.linalg.norm(_gravity_at((0, 0, 0), src, (0, 10, 0))) - 9.81 * 0.25) < 1e-4
    assert np.array_equal(_gravity_at((0, 0, 0), src, (0, 0, 100)), np.zeros(3, np.float32))
    none = np.zeros(0, A.GRAVITY_SOURCE)
    assert np.array_equal(_gravity_at((1, 2, -9.81), none, (3, -7, 2)),
                          np.array([1, 2, -9.81], np.float32))


def test_frame_substeps_holds_the_internal_substep():
    fs = K.oracle().orc_frame_substeps
    assert fs(1 / 60, 1 / 60, 4) == 4
    assert fs(1 / 120, 1 / 60, 4) == 2
    assert fs(0.25, 1 / 60, 4) == 16
    assert fs(1e-5, 1 / 60, 4) == 1


# ------------------------------------------------------------------------------------------
# Reference test pins, against the oracle
# ------------------------------------------------------------------------------------------

def test_free_fall_matches_analytic():
    """cloth_solver_test.cpp:81-107: 60 frames of free fall, no damping / aero."""
    p = _params(damping=0.0, air_drag=0.0, air_lift=0.0)
    c = K.RefCloth.make_grid(grid_desc(5, center=(0, 0, 10), params=p)).arrays()
    start = c.particles["position"][0].copy()
    h = 1 / 60
    for _ in range(60):
        K.oracle_step_cloth(c, substeps=4, iterations=1, h=h)
    t = 60 * h
    hs = h / 4
    drop = 0.5 * 9.81 * t * t + 0.5 * 9.81 * t * hs
    assert abs((start[2] - c.particles["position"][0][2]) - drop) < 0.05
    assert abs(c.particles["position"][0][0] - start[0]) < 1e-4
    assert abs(c.particles["position"][0][1] - start[1]) < 1e-4


def test_static_anchors_hold_and_tethers_cap_distance():
    """cloth_solver_test.cpp:145-171."""
    p = _params(tether_scale=1.02, external_acceleration=(200.0, 0.0, 0.0))
    ref = K.RefCloth.make_grid(grid_desc(11, center=(0, 0, 5), params=p))
    ref.pin_static((0, 0, 5), 0.5)
    ref.build_tethers()
    c = ref.arrays()
    assert len(c.tethers) > 0
    for _ in range(180):
        K.oracle_step_cloth(c, substeps=4, iterations=1)
    pos = c.particles["position"]
    d = np.linalg.norm(pos[c.tethers["particle"]] - pos[c.tethers["anchor"]], axis=1)
    assert np.all(d <= c.tethers["max_length"] + 1e-3)
    for a in c.anchors:
        np.testing.assert_allclose(pos[a["particle"]], a["world_position"], atol=1e-5)
        assert c.particles["inv_mass"][a["particle"]] == 0.0


def test_sheet_drapes_over_sphere_without_penetrating():
    """cloth_collision_test.cpp:27-64."""
    centre = np.array([0, 0, 3], np.float32)
    ref = K.RefCloth.make_grid(grid_desc(21, center=tuple(centre + (0, 0, 1.05))))
    ref.pin_static(tuple(centre + (0, 0, 1.05)), 0.4)
    ref.build_tethers()
    c = ref.arrays()
    cols = collider_array([sphere(1.0, tuple(centre))])
    for _ in range(300):
        K.oracle_step_cloth(c, cols, substeps=4, iterations=1)
    pos = c.particles["position"]
    assert np.all(np.linalg.norm(pos - centre, axis=1) >= 1.0)
    st = c.stretch
    stretch = np.linalg.norm(pos[st["a"]] - pos[st["b"]], axis=1) / st["rest_length"]
    assert stretch.max() < 1.25
    assert c.bounds[2] < centre[2]
