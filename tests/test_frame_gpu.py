"""A whole cloth frame on the device (pxb_cloths_step_frame: PhysicsWorld::step_cloths_,
world.h:1749-1847, minus the collider gather) against the oracle's restatement of the same frame
(test_frame_oracle_ref.py): anchors follow their bodies, cloths fall asleep and wake, and every
particle, awake flag and sleep timer equals the oracle's frame after frame."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200.arrays import collider_array, sphere

import _checkers as K
from test_cloth_gpu import assert_equal_particles
from test_frame_oracle_ref import FIXED_DT, body_poses, reference_sleep_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def sheet(side, center, **params):
    p = A.ClothParams.defaults()
    for k, v in params.items():
        setattr(p, k, v)
    w = 0.08 * (side - 1)
    return R.HostCloth(side, side, w, w, center=center, params=p, jitter=1e-3, seed=side)


def poses_at(frame):
    """Body 0 slides along x for frames 0-39 and again from frame 160; body 1 turns about z for
    frames 0-29; body 2 never moves."""
    x0 = 0.01 * min(frame, 40) + (0.02 * (frame - 160) if frame >= 160 else 0.0)
    ang = 0.03 * min(frame, 30)
    return [((x0, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0)),
            ((1.5, 0.0, 2.0), (0.0, 0.0, float(np.sin(ang / 2)), float(np.cos(ang / 2)))),
            ((-1.5, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0))]


def test_frames_with_moving_bodies_sleep_and_wake_equal_oracle(ctx):
    sleepy = dict(damping=2.0, sleep_threshold=0.3, sleep_time=0.2)
    h0 = sheet(12, (0.0, 0.0, 2.0), **sleepy)
    h0.pin_to_body(0, 0, (0.0, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0), (0.0, 0.44, 2.0), 0.2)
    h1 = sheet(10, (1.5, 0.0, 2.0), **sleepy)
    h1.pin_to_body(1, 0, (1.5, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0), (1.5, 0.36, 2.0), 0.2)
    h2 = sheet(8, (-1.5, 0.0, 2.0), **sleepy)
    h2.pin_to_body(2, 0, (-1.5, 0.0, 2.0), (0.0, 0.0, 0.0, 1.0), (-1.5, 0.28, 2.0), 0.15)
    h3 = sheet(8, (0.0, 1.5, 2.0))  # static pins only, default sleep params
    h3.pin_static((-0.28, 1.78, 2.0), 0.05)
    cloths = [h.arrays() for h in (h0, h1, h2, h3)]
    cols = [collider_array([sphere(0.3, (0.0, 0.0, 1.2))]), None, None, collider_array([sphere(0.2, (0.0, 1.5, 1.4))])]
    ids = [ctx.add_cloth(c) for c in cloths]
    orc = [c.copy() for c in cloths]
    states = [{"awake": 1, "sleep_timer": np.float32(0.0)} for _ in cloths]
    slept = set()
    try:
        for frame in range(220):
            bodies = body_poses(poses_at(frame))
            awake = ctx.step_frame(ids, bodies, cols, fixed_dt=FIXED_DT, cloth_substeps=4, cloth_iterations=2,
                                   dt=FIXED_DT)
            for k, (o, st) in enumerate(zip(orc, states)):
                K.oracle_world_step_cloth(o, st, bodies, cols[k], fixed_dt=FIXED_DT, cloth_substeps=4,
                                          cloth_iterations=2, dt=FIXED_DT)
            assert list(awake) == [s["awake"] for s in states], frame
            slept |= {k for k, s in enumerate(states) if not s["awake"]}
            if frame % 20 == 19 or frame == 219:
                a, t = ctx.read_sleep_state(ids)
                assert np.array_equal(t, np.array([s["sleep_timer"] for s in states], np.float32)), frame
                for k, (cid, c, o) in enumerate(zip(ids, cloths, orc)):
                    assert_equal_particles(ctx.read_particles(cid, len(c.particles)), o.particles, f"cloth {k} frame {frame}")
                    assert np.array_equal(ctx.read_anchors(cid, len(c.anchors)).view(np.uint8), o.anchors.view(np.uint8))
        assert {0, 1, 2} <= slept          # they settled and slept
        assert states[0]["awake"] == 1     # body 0 moved again from frame 160 and woke its cloth
    finally:
        for cid in ids:
            ctx.remove_cloth(cid)


def test_reference_sleep_scene_on_device(ctx):
    """cloth_solver_test.cpp:296-328 through pxb_cloths_step_frame."""
    c = reference_sleep_scene()
    cid = ctx.add_cloth(c)
    try:
        post = [((0.0, 0.0, 5.0), (0.0, 0.0, 0.0, 1.0))]
        for _ in range(600):
            awake = ctx.step_frame([cid], body_poses(post), fixed_dt=FIXED_DT, cloth_substeps=4, cloth_iterations=1,
                                   dt=FIXED_DT)
        assert awake[0] == 0
        before = ctx.read_particles(cid, len(c.particles))["position"][-1].copy()
        for _ in range(60):
            ctx.step_frame([cid], body_poses(post), fixed_dt=FIXED_DT, cloth_substeps=4, cloth_iterations=1, dt=FIXED_DT)
        np.testing.assert_allclose(ctx.read_particles(cid, len(c.particles))["position"][-1], before, atol=1e-6)
        post[0] = ((0.5, 0.0, 5.0), (0.0, 0.0, 0.0, 1.0))
        awake = ctx.step_frame([cid], body_poses(post), fixed_dt=FIXED_DT, cloth_substeps=4, cloth_iterations=1,
                               dt=FIXED_DT)
        assert awake[0] == 1
    finally:
        ctx.remove_cloth(cid)


def test_a_moving_collider_wakes_a_sleeping_cloth(ctx):
    c = reference_sleep_scene()
    cid = ctx.add_cloth(c)
    try:
        post = body_poses([((0.0, 0.0, 5.0), (0.0, 0.0, 0.0, 1.0))])
        for _ in range(600):
            awake = ctx.step_frame([cid], post, fixed_dt=FIXED_DT, cloth_iterations=1, dt=FIXED_DT)
        assert awake[0] == 0
        awake = ctx.step_frame([cid], post, collider_moving=[1], fixed_dt=FIXED_DT, cloth_iterations=1, dt=FIXED_DT)
        assert awake[0] == 1
    finally:
        ctx.remove_cloth(cid)


def test_frame_refusals(ctx):
    c = reference_sleep_scene()
    cid = ctx.add_cloth(c)
    try:
        with pytest.raises(R.PxbError) as e:
            ctx.step_frame([cid], dt=0.0)
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    finally:
        ctx.remove_cloth(cid)
    with pytest.raises(R.PxbError) as e:
        ctx.step_frame([cid], dt=FIXED_DT)
    assert e.value.status == A.PXB_ERR_INVALID_HANDLE
