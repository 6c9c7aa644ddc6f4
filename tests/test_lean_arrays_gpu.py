"""The one-CTA float-array layout of the largest lean sheets (pxb_cloth_plan.lean == 2: x, y, z
arrays in shared memory and a byte per particle indexing the cloth's distinct inverse masses;
sides 110-128) against the layout it replaces (the same sheets on a 2-CTA cluster,
pxb_context_set_lean_arrays(0)) and against the oracle: equal bit for bit, step after step, with
the inverse masses from the table, from HBM (more distinct values than the table holds), after a
rewrite that moves a cloth from one to the other, and through the warm-start kernel.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes
from physxcoopa_b200.arrays import box, capsule, collider_array, sphere

import _checkers as K
from test_warm_gpu import random_net

pytestmark = pytest.mark.gpu

SIDES = (110, 117, 128)
FIELDS = ("position", "velocity", "prev_position")


def sheets(seed=5, many_masses=False):
    cloths, cols = [], []
    rng = np.random.default_rng(seed)
    for k, side in enumerate(SIDES):
        w = 0.02 * (side - 1)
        h = R.HostCloth(side, side, w, w, center=(0, 0, 1), params=scenes.reference_params(), jitter=1e-3,
                        seed=seed + k)
        h.pin_static((-w / 2, w / 2, 1), 0.02)
        h.pin_static((w / 2, w / 2, 1), 0.02)
        h.build_tethers()
        c = h.arrays()
        if many_masses:
            free = c.particles["inv_mass"] != 0.0
            c.particles["inv_mass"][free] = (rng.uniform(0.5, 2.0, int(free.sum())) * side * side).astype(np.float32)
        cloths.append(c)
        shapes = [sphere(0.4, (0.1 * k, 0.0, 0.3)), capsule(0.15, 0.4, (0.3, -0.2, 0.5)),
                  box((0.3, 0.2, 0.1), (-0.4, 0.3, 0.6))]
        cols.append(collider_array(shapes[: 1 + k]))
    return cloths, cols


@pytest.fixture(scope="module")
def ctxs():
    a = R.Context(0)        # float arrays (the default)
    b = R.Context(0)
    b.set_lean_arrays(False)  # 2-CTA clusters
    yield a, b
    a.close()
    b.close()


def test_plans():
    cloths, _ = sheets()
    for c, side in zip(cloths, SIDES):
        p = R.plan_cloth(c)
        assert (p["n_ranks"], p["lean"]) == (1, 2), (side, p)
        assert p["smem_bytes"] <= 227 * 1024


def read(ctx, ids, cloths):
    return [ctx.read_particles(i, len(c.particles)) for i, c in zip(ids, cloths)]


def same(x, y):
    return all(np.array_equal(p[f], q[f]) for p, q in zip(x, y) for f in FIELDS)


@pytest.mark.parametrize("many_masses", [False, True])
def test_arrays_equal_clusters_and_oracle(ctxs, many_masses):
    a, b = ctxs
    cloths, cols = sheets(many_masses=many_masses)
    if many_masses:
        assert all(len(np.unique(c.particles["inv_mass"])) > 256 for c in cloths)
    orcs = [c.copy() for c in cloths]
    ia = [a.add_cloth(c) for c in cloths]
    ib = [b.add_cloth(c) for c in cloths]
    try:
        for s in range(24):
            a.step(ia, cols)
            b.step(ib, cols)
            for o, c in zip(orcs, cols):
                K.oracle_step_cloth(o, c, substeps=4, iterations=10)
            ga, gb = read(a, ia, cloths), read(b, ib, cloths)
            assert same(ga, gb), s
            for g, o in zip(ga, orcs):
                for f in FIELDS:
                    assert np.array_equal(g[f], o.particles[f]), (s, f)
        for x, y, c in zip(ia, ib, cloths):
            la = a.read_lambdas(x, len(c.stretch), len(c.bend))
            lb = b.read_lambdas(y, len(c.stretch), len(c.bend))
            for u, v in zip(la, lb):
                assert np.array_equal(u, v)
        ra, rb = a.read_results(ia), b.read_results(ib)
        assert np.array_equal(ra, rb)
        # the sheets fell onto their colliders
        assert min(float(g["position"][:, 2].min()) for g in ga) < 0.9
    finally:
        for i in ia:
            a.remove_cloth(i)
        for i in ib:
            b.remove_cloth(i)


def test_rewritten_masses_switch_between_table_and_hbm(ctxs):
    a, b = ctxs
    cloths, cols = sheets(seed=9)
    many, _ = sheets(seed=9, many_masses=True)
    ia = [a.add_cloth(c) for c in cloths]
    ib = [b.add_cloth(c) for c in cloths]
    try:
        for phase, src in enumerate((many, cloths, many)):
            for x, y, s in zip(ia, ib, src):
                state = a.read_particles(x, len(s.particles))
                state["inv_mass"] = s.particles["inv_mass"]
                a.write_particles(x, state)
                b.write_particles(y, state)
            for _ in range(4):
                a.step(ia, cols)
                b.step(ib, cols)
            assert same(read(a, ia, cloths), read(b, ib, cloths)), phase
    finally:
        for i in ia:
            a.remove_cloth(i)
        for i in ib:
            b.remove_cloth(i)


def test_warm_start_kernel_equal_on_both_layouts(ctxs):
    a, b = ctxs
    cloths, cols = sheets(seed=13)
    net = random_net(np.random.default_rng(6))
    a.set_mlp(net)
    b.set_mlp(net)
    ia = [a.add_cloth(c) for c in cloths]
    ib = [b.add_cloth(c) for c in cloths]
    try:
        for s in range(6):
            for ctx, ids in ((a, ia), (b, ib)):
                ctx.step_warm(ids, cols, iterations=20, warm_iterations=4, threshold=2e-2, continue_iterations=True)
            assert same(read(a, ia, cloths), read(b, ib, cloths)), s
            wa, wb = a.read_warm_results(ia), b.read_warm_results(ib)
            assert np.array_equal(wa, wb), s
    finally:
        for i in ia:
            a.remove_cloth(i)
        for i in ib:
            b.remove_cloth(i)
