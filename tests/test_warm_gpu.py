"""The warm-start solve (network displacement, a few iterations, residual check, fallback) and
the training-row recorder, held to exact properties against the plain solver:

* warm_iterations = 0 is the plain solve: positions equal the plain kernel's, bit for bit, and
  the reported residual is the max relative strain of the stretch constraints;
* a network that outputs zero followed by N warm iterations equals N plain iterations;
* a threshold below any residual falls back in every substep and equals the plain solve;
* continuing after a zero network until the plain count equals the plain solve too (the
  iterations resume where the warm ones stopped, lambdas included);
* recorded features are the quantities the solver sees (velocity at the start of the substep,
  predicted displacement), recorded rows are the free particles.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes
from physxcoopa_b200.arrays import collider_array, sphere

import _checkers as K

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def batch(sides=(16, 40, 64, 65, 100), seed=3):
    cloths, cols = [], []
    for k, side in enumerate(sides):
        w = 0.05 * (side - 1)
        h = R.HostCloth(side, side, w, w, center=(0, 0, 1), params=scenes.cloth_params(), jitter=1e-3, seed=seed + k)
        h.pin_static((-w / 2, w / 2, 1), 0.02)
        h.pin_static((w / 2, w / 2, 1), 0.02)
        h.build_tethers()
        cloths.append(h.arrays())
        cols.append(collider_array([sphere(0.3 + 0.03 * k, (0.05 * k, 0, 0.5))]))
    return cloths, cols


def random_net(rng, zero_out=False):
    W = {"w1": rng.normal(0, 0.2, (64, 24)), "b1": rng.normal(0, 0.1, 64),
         "w2": rng.normal(0, 0.125, (64, 64)), "b2": rng.normal(0, 0.1, 64),
         "w3": np.zeros((3, 64)) if zero_out else rng.normal(0, 0.125, (3, 64)),
         "b3": np.zeros(3) if zero_out else rng.normal(0, 0.1, 3),
         "in_mean": np.zeros(24), "in_scale": np.full(24, 100.0), "out_scale": np.full(3, 1e-4)}
    return A.MlpWeights.from_numpy(**W)


def run(ctx, cloths, cols, steps, fn):
    ids = [ctx.add_cloth(c) for c in cloths]
    try:
        for _ in range(steps):
            fn(ids)
        parts = [ctx.read_particles(i, len(c.particles)) for i, c in zip(ids, cloths)]
        warm = None
        try:
            warm = ctx.read_warm_results(ids)
        except R.PxbError:
            pass
    finally:
        for i in ids:
            ctx.remove_cloth(i)
    return parts, warm


def same(a, b):
    return all(np.array_equal(x[f], y[f]) for x, y in zip(a, b) for f in ("position", "velocity", "prev_position"))


def strain(c, parts):
    p = parts["position"]
    s = c.stretch
    d = p[s["a"]] - p[s["b"]]
    l = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    return np.abs(l / s["rest_length"] - np.float32(1.0)).max()


def test_plain_through_the_warm_kernel_is_the_plain_solve(ctx):
    cloths, cols = batch()
    plain, _ = run(ctx, cloths, cols, 5, lambda ids: ctx.step(ids, cols))
    warm0, res = run(ctx, cloths, cols, 5, lambda ids: ctx.step_warm(ids, cols, warm_iterations=0))
    assert same(plain, warm0)
    assert np.all(res["fallbacks"] == 0) and np.all(res["substeps"] == 4)
    # one substep, no colliders or tethers moving anything after the iterations: the residual
    # is the final strain
    free = [c.copy() for c in cloths]
    for c in free:
        c.tethers = c.tethers[:0]
    one, res1 = run(ctx, free, None, 1, lambda ids: ctx.step_warm(ids, None, substeps=1, warm_iterations=0))
    for c, p, r in zip(free, one, res1):
        assert np.float32(r["residual"]) == strain(c, p)


def test_zero_network_plus_n_iterations_equals_n_plain_iterations(ctx):
    cloths, cols = batch(seed=5)
    ctx.set_mlp(random_net(np.random.default_rng(1), zero_out=True))
    plain, _ = run(ctx, cloths, cols, 4, lambda ids: ctx.step(ids, cols, iterations=6))
    warm, res = run(ctx, cloths, cols, 4, lambda ids: ctx.step_warm(ids, cols, iterations=20, warm_iterations=6,
                                                                      threshold=np.inf))
    assert same(plain, warm)
    assert np.all(res["fallbacks"] == 0)


def test_fallback_everywhere_equals_the_plain_solve(ctx):
    cloths, cols = batch(seed=7)
    ctx.set_mlp(random_net(np.random.default_rng(2)))
    plain, _ = run(ctx, cloths, cols, 4, lambda ids: ctx.step(ids, cols, iterations=10))
    warm, res = run(ctx, cloths, cols, 4, lambda ids: ctx.step_warm(ids, cols, iterations=10, warm_iterations=3,
                                                                      threshold=-1.0))
    assert same(plain, warm)
    assert np.all(res["fallbacks"] == res["substeps"])


def test_network_moves_only_free_particles_and_reports_residuals(ctx):
    cloths, cols = batch(seed=9)
    ctx.set_mlp(random_net(np.random.default_rng(3)))
    warm, res = run(ctx, cloths, cols, 3, lambda ids: ctx.step_warm(ids, cols, warm_iterations=4, threshold=np.inf))
    plain, _ = run(ctx, cloths, cols, 3, lambda ids: ctx.step(ids, cols))
    for c, w, p in zip(cloths, warm, plain):
        pinned = c.particles["inv_mass"] == 0
        assert np.array_equal(w["position"][pinned], p["position"][pinned])
        assert np.all(np.isfinite(w["position"]))
    assert np.all(res["fallbacks"] == 0) and np.all(res["residual"] > 0)


def test_recorded_rows_are_what_the_solver_sees(ctx):
    cloths, cols = batch(sides=(20, 70), seed=11)
    ids = [ctx.add_cloth(c) for c in cloths]
    try:
        x, y = ctx.record(ids, cols, substep=0)
        n_free = sum(int((c.particles["inv_mass"] != 0).sum()) for c in cloths)
        assert len(x) == n_free and len(y) == n_free
        # from rest: the substep starts with zero velocity, and integration predicts a move of
        # v * hs with v = g * hs * damping (rounded against the position it is added to)
        P = cloths[0].params
        hs = np.float32(1.0 / 60.0) / np.float32(4)
        damping = np.float32(1.0) / (np.float32(1.0) + np.float32(P.damping) * hs)
        vz = (np.float32(0.0) + np.float32(-9.81) * np.float32(P.gravity_scale) * hs) * damping
        assert np.all(x[:, 3:6] == 0) and np.all(x[:, 0:2] == 0)
        assert np.allclose(x[:, 2], vz * hs, rtol=0, atol=2e-7)
        assert np.all(np.isfinite(y)) and np.abs(y).max() < 0.05
        # the recording step is a plain step
        after = [ctx.read_particles(i, len(c.particles)) for i, c in zip(ids, cloths)]
    finally:
        for i in ids:
            ctx.remove_cloth(i)
    plain, _ = run(ctx, cloths, cols, 1, lambda ids: ctx.step(ids, cols))
    assert same(after, plain)


def test_continued_iterations_after_a_zero_network_equal_the_plain_solve(ctx):
    cloths, cols = batch(seed=13)
    ctx.set_mlp(random_net(np.random.default_rng(4), zero_out=True))
    plain, _ = run(ctx, cloths, cols, 3, lambda ids: ctx.step(ids, cols, iterations=12))
    warm, res = run(ctx, cloths, cols, 3, lambda ids: ctx.step_warm(ids, cols, iterations=12, warm_iterations=4,
                                                                      threshold=-1.0, continue_iterations=True))
    assert same(plain, warm)
    assert np.all(res["fallbacks"] == res["substeps"]) and np.all(res["extra_iterations"] == 8 * res["substeps"])
