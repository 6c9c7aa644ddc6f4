"""A whole strand frame on the device (pxb_strands_step_frame: PhysicsWorld::step_strands_,
world.h:1861-1957, minus the collider gather) against the oracle's restatement of the same frame
(orc_world_step_strands): a groom whose roots move is woken by them, grooms come to rest and fall
asleep (velocities zeroed, roots' previous targets carried along while asleep), a moving collider
or a root target that moves again wakes them, and every particle, awake flag and sleep timer
equals the oracle's, frame after frame. The strands use no local shape and no turning roots (the
stages whose libm calls may differ from the host's in the last bit), so equality is exact."""
import numpy as np
import pytest

from physxcoopa_b200 import runtime as R
from physxcoopa_b200.arrays import collider_array, gravity_sources, sphere

import _checkers as K
from test_strands_oracle_ref import params, straight

pytestmark = pytest.mark.gpu

FIXED_DT = 1.0 / 60.0


def roots_of(lines, offset):
    return np.array([np.asarray(l[0], np.float32) + np.asarray(offset, np.float32) for l in lines], np.float32)


def test_strand_frames_wake_sleep_and_equal_the_oracle():
    ctx = R.Context(0)
    sleepy = dict(local_shape=0.0, global_shape=0.5, damping=6.0, sleep_threshold=0.1, sleep_time=0.25)
    lines_a = [straight((0.03 * i, 0.0, 1.0), 14, 0.02) for i in range(6)]      # roots driven along x
    lines_b = [straight((0.0, 0.5 + 0.03 * i, 1.0), 10, 0.02) for i in range(4)]  # still roots; a collider
    lines_c = [straight((1.0, 0.0, 1.0), 40, 0.01)]                              # long strand, gravity source
    sets = [R.make_strands(lines_a, params(**sleepy)), R.make_strands(lines_b, params(**sleepy)),
            R.make_strands(lines_c, params(**sleepy))]
    orcs = [s.copy() for s in sets]
    ids = [ctx.add_strands(s) for s in sets]
    states = [{"awake": 1, "sleep_timer": np.float32(0.0)} for _ in sets]
    src_c = gravity_sources([((1.0, 0.0, -2.0), 9.81, 1.0, 10.0)])
    slept, woke = set(), set()
    try:
        for f in range(180):
            # set A: the engine sets its roots every frame (set_strand_roots, from the scalp's
            # transform); they slide for the first 10 frames and again from frame 150
            x = 0.004 * min(f, 10) + (0.01 * (f - 149) if f >= 150 else 0.0)
            pos = roots_of(lines_a, (x, 0.0, 0.0))
            ctx.set_strand_roots(ids[0], pos)
            K.oracle_set_strand_roots(orcs[0], pos)
            cols = [None, collider_array([sphere(0.05, (0.02, 0.55, 0.85))]), None]
            moving = [0, 1 if f in (120, 121) else 0, 0]
            awake = ctx.step_strands_frame(ids, colliders=cols, collider_moving=moving,
                                           sources=[None, None, src_c], fixed_dt=FIXED_DT, cloth_substeps=4,
                                           cloth_iterations=6, dt=FIXED_DT)
            for k, (o, st) in enumerate(zip(orcs, states)):
                was = st["awake"]
                K.oracle_world_step_strands(o, st, colliders=cols[k], collider_moving=bool(moving[k]),
                                            sources=[None, None, src_c][k], fixed_dt=FIXED_DT, cloth_substeps=4,
                                            cloth_iterations=6, dt=FIXED_DT)
                if was and not st["awake"]:
                    slept.add(k)
                if not was and st["awake"]:
                    woke.add(k)
            a, t = ctx.read_strand_sleep_state(ids)
            assert list(a) == [st["awake"] for st in states] == list(awake), f
            assert np.array_equal(t, np.array([st["sleep_timer"] for st in states], np.float32)), f
            for k, (sid, o) in enumerate(zip(ids, orcs)):
                g = ctx.read_strand_particles(sid, len(o.particles))
                for fld in ("position", "velocity", "prev_position"):
                    assert np.array_equal(g[fld], o.particles[fld]), (f, k, fld)
        # the frames went through sleep and wake: A and B slept and woke again
        assert {0, 1} <= slept, slept
        assert {0, 1} <= woke, woke
    finally:
        ctx.close()
