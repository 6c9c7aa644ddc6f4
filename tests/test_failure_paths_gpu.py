"""Failure paths on the device, driven without faulting the GPU.

A cloth too large for an 8-CTA cluster steps on every SM with a grid barrier after every colour
and stage; every barrier wait is bounded. pxb_context_set_wait_test makes every grid barrier
unreachable (one more arrival than the launch has CTAs: a release that nothing sets) with a short
wait bound, so the expiry path runs: each CTA's first wait runs out and records the error word,
later barriers no longer wait, the launch ends, and the next synchronising call reports
PXB_ERR_DEVICE_STATUS and clears the word. The same context then steps correctly again, on the
whole-GPU path and on the one-CTA path.
"""
import time

import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes
from physxcoopa_b200.arrays import collider_array, sphere

import _checkers as K

pytestmark = pytest.mark.gpu


def sheet(side, seed):
    w = 0.05 * (side - 1)
    h = R.HostCloth(side, side, w, w, center=(0, 0, 1), params=scenes.cloth_params(), jitter=1e-3, seed=seed)
    h.pin_static((-w / 2, w / 2, 1), 0.02)
    h.pin_static((w / 2, w / 2, 1), 0.02)
    return h.arrays()


def test_expired_grid_barrier_reports_device_status_and_the_context_recovers():
    ctx = R.Context(0)
    try:
        big = sheet(200, 5)
        assert R.plan_cloth(big)["n_ranks"] == 0  # the whole-GPU path
        small = sheet(24, 6)
        col = collider_array([sphere(0.4, (0.0, 0.0, 0.4))])
        bid = ctx.add_cloth(big)
        sid = ctx.add_cloth(small)

        ctx.set_wait_test(grid_wait_polls=1 << 10, unreachable=True)
        t0 = time.perf_counter()
        ctx.step([bid], [col])
        with pytest.raises(R.PxbError) as e:
            ctx.synchronize()
        elapsed = time.perf_counter() - t0
        assert e.value.status == A.PXB_ERR_DEVICE_STATUS
        assert "queue wait expired" in str(e.value)
        assert elapsed < 30.0  # one expired wait per CTA, then the launch ran to its end
        # the word was cleared by the report: a synchronising call now succeeds
        ctx.synchronize()

        # back to normal bounds: the context steps correctly again (the failed step's state is
        # meaningless, so the big cloth is added afresh)
        ctx.set_wait_test()
        ctx.remove_cloth(bid)
        bid = ctx.add_cloth(big)
        orc_big, orc_small = big.copy(), small.copy()
        for _ in range(2):
            ctx.step([bid, sid], [col, col])
            K.oracle_step_cloth(orc_big, col, substeps=4, iterations=10)
            K.oracle_step_cloth(orc_small, col, substeps=4, iterations=10)
        g_big = ctx.read_particles(bid, len(big.particles))
        g_small = ctx.read_particles(sid, len(small.particles))
        assert np.array_equal(g_big["position"], orc_big.particles["position"])
        assert np.array_equal(g_small["position"], orc_small.particles["position"])
    finally:
        ctx.set_wait_test()
        ctx.close()


def test_wait_test_refuses_a_zero_bound():
    ctx = R.Context(0)
    try:
        with pytest.raises(R.PxbError) as e:
            ctx.set_wait_test(grid_wait_polls=0)
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    finally:
        ctx.close()
