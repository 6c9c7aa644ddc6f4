"""The caller glue of a cloth frame (PhysicsWorld::step_cloths_, world.h:1749-1847): the library's
pin_to_body builder against the reference's, and the oracle's restatement of the frame (anchors
from body poses, sleep gate, solve, sleep bookkeeping) against the reference test's known answers
(tests/cloth_solver_test.cpp:296-328, sleeps_when_settled_and_wakes_on_anchor_motion)."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R

import _checkers as K

FIXED_DT = 1.0 / 60.0  # util::k_default_fixed_dt; PhysicsConfig: 4 cloth substeps, 1 iteration


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def body_poses(records):
    """records: (position, orientation xyzw) per body index, generation 0, alive."""
    out = np.zeros(len(records), A.BODY_POSE)
    for k, (p, q) in enumerate(records):
        out[k]["position"] = p
        out[k]["orientation"] = q
        out[k]["alive"] = 1
    return out


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("radius", [0.3, 1.2, 3.0])
def test_pin_to_body_matches_reference_bitwise(radius):
    q = np.array([0.1, -0.3, 0.2, 0.9273618], np.float32)
    q /= np.float32(np.sqrt(np.dot(q, q)))
    body = ((0.4, -0.2, 5.3), tuple(float(v) for v in q))
    mine = R.HostCloth(9, 9, 4.0, 4.0, center=(0.0, 0.0, 5.0))
    desc = A.GridClothDesc()
    desc.columns = desc.rows = 9
    desc.width = desc.height = 4.0
    desc.center = (A.C.c_float * 3)(0.0, 0.0, 5.0)
    desc.orientation = (A.C.c_float * 4)(0.0, 0.0, 0.0, 1.0)
    desc.total_mass = 1.0
    desc.shear = 1
    desc.params = A.ClothParams.defaults()
    ref = K.RefCloth.make_grid(desc)
    n_mine = mine.pin_to_body(3, 7, body[0], body[1], (1.0, 0.5, 5.0), radius)
    n_ref = ref.pin_to_body(3, 7, body[0], body[1], (1.0, 0.5, 5.0), radius)
    assert n_mine == n_ref > 0
    a, b = mine.arrays(), ref.arrays()
    assert same(a.particles, b.particles)
    assert same(a.anchors, b.anchors)


def reference_sleep_scene():
    """cloth_solver_test.cpp:296-328: a 9 x 9, 4 m sheet at z = 5 pinned to a kinematic post within
    3 m of (0, 0, 5); damping 4, sleep_threshold 0.25 m/s, sleep_time 0.25 s."""
    p = A.ClothParams.defaults()
    p.damping = 4.0
    p.sleep_threshold = 0.25
    p.sleep_time = 0.25
    h = R.HostCloth(9, 9, 4.0, 4.0, center=(0.0, 0.0, 5.0), params=p)
    h.pin_to_body(0, 0, (0.0, 0.0, 5.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.0, 5.0), 3.0)
    return h.arrays()


def test_oracle_frame_sleeps_when_settled_and_wakes_on_anchor_motion():
    c = reference_sleep_scene()
    post = [((0.0, 0.0, 5.0), (0.0, 0.0, 0.0, 1.0))]
    state = {"awake": 1, "sleep_timer": np.float32(0.0)}
    for _ in range(600):
        K.oracle_world_step_cloth(c, state, body_poses(post), fixed_dt=FIXED_DT, cloth_iterations=1, dt=FIXED_DT)
    assert state["awake"] == 0
    before = c.particles["position"][-1].copy()
    for _ in range(60):
        assert K.oracle_world_step_cloth(c, state, body_poses(post), fixed_dt=FIXED_DT, cloth_iterations=1,
                                         dt=FIXED_DT) == 0
    np.testing.assert_allclose(c.particles["position"][-1], before, atol=1e-6)
    post[0] = ((0.5, 0.0, 5.0), (0.0, 0.0, 0.0, 1.0))
    K.oracle_world_step_cloth(c, state, body_poses(post), fixed_dt=FIXED_DT, cloth_iterations=1, dt=FIXED_DT)
    assert state["awake"] == 1
    # the anchors now follow the post
    np.testing.assert_allclose(c.anchors["world_position"][:, 0], c.anchors["local_position"][:, 0] + 0.5, atol=1e-5)


def test_frame_substeps_hold_the_internal_substep():
    f = K.oracle().orc_frame_substeps
    assert f(1.0 / 60.0, 1.0 / 60.0, 4) == 4
    assert f(1.0 / 30.0, 1.0 / 60.0, 4) == 8
    assert f(1.0 / 240.0, 1.0 / 60.0, 4) == 1
    assert f(1.0, 1.0 / 60.0, 4) == 16  # k_max_cloth_substeps
