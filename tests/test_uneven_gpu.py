"""Parity on the benchmark's own batch: sheets of the uneven 4096-sheet batch (sides U{16..128},
1-3 sphere / capsule / box colliders, point gravity sources on half of them) stepped together in
one pxb_cloths_step call, i.e. through the launch grouping the benchmark times: sheets that fit
one CTA's shared memory, lean sheets on one CTA (positions in shared memory, rest lengths and
lambdas read in place) and the largest lean sheets on one CTA with their positions as float
arrays (sides 110-128), each group its own launch on a side stream.

Bars: pins exact, every particle within 1e-5 m after one step and within 1e-3 m after 300 steps;
the device is asserted equal to the oracle value for value at both points.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes

import _checkers as K

pytestmark = pytest.mark.gpu

PLAN = scenes.uneven_plan(4096, seed=2)


def layout_of(cloth):
    p = R.plan_cloth(cloth)
    if p["lean"] == 2:
        return "lean arrays"
    if p["lean"]:
        return f"lean x{p['n_ranks']}"
    return "shared memory" if p["n_ranks"] == 1 else f"cluster x{p['n_ranks']}"


def pick(per_layout):
    """Sheets of the batch, in batch order, until every layout has `per_layout` of them."""
    want = {"small": per_layout, "lean1": per_layout, "lean2": per_layout}
    out = []
    for i, s in enumerate(PLAN):
        key = "small" if s.side <= 44 else ("lean1" if s.side <= 109 else "lean2")
        if want[key] > 0:
            want[key] -= 1
            out.append(i)
        if not any(want.values()):
            break
    return out


def build(indices, params):
    specs = [PLAN[i] for i in indices]
    return ([scenes.build_sheet(s, params) for s in specs], [s.colliders for s in specs],
            [s.source for s in specs])


def step_both(ctx, cloths, colliders, sources, steps, check_every=None):
    orcs = [c.copy() for c in cloths]
    ids = [ctx.add_cloth(c) for c in cloths]
    d, keep = ctx.make_step(ids, colliders, (0.0, 0.0, -9.81), sources, 4, 10, 1.0 / 60.0)
    try:
        for s in range(steps):
            ctx.step_desc(d)
            for o, c, src in zip(orcs, colliders, sources):
                K.oracle_step_cloth(o, c, sources=src, substeps=4, iterations=10)
            if check_every and (s + 1) in check_every:
                check_every[s + 1](ids, orcs)
        got = [ctx.read_particles(i, len(o.particles)) for i, o in zip(ids, orcs)]
        res = ctx.read_results(ids)
    finally:
        del keep
        for i in ids:
            ctx.remove_cloth(i)
    return got, orcs, res


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def test_sample_covers_every_layout_colliders_and_sources():
    idx = pick(8)
    cloths, cols, srcs = build(idx, scenes.reference_params())
    kinds = {layout_of(c) for c in cloths}
    assert kinds == {"shared memory", "lean x1", "lean arrays"}, kinds
    types = {int(t) for c in cols for t in c["type"]}
    assert {A.SHAPE_SPHERE, A.SHAPE_CAPSULE, A.SHAPE_BOX} <= types
    assert sum(s is not None for s in srcs) >= 6


@pytest.mark.parametrize("params", ["reference", "three_compliances"])
def test_uneven_sample_one_step_equals_oracle(ctx, params):
    p = scenes.reference_params() if params == "reference" else scenes.cloth_params()
    idx = pick(8)
    cloths, cols, srcs = build(idx, p)
    got, orcs, res = step_both(ctx, cloths, cols, srcs, 1)
    for i, g, o in zip(idx, got, orcs):
        pinned = o.particles["inv_mass"] == 0.0
        assert np.array_equal(g["position"][pinned], o.particles["position"][pinned]), i
        d = float(np.max(np.abs(g["position"].astype(np.float64) - o.particles["position"])))
        assert d <= 1e-5, (i, PLAN[i].side, d)
        for f in ("position", "velocity", "prev_position"):
            assert np.array_equal(g[f], o.particles[f]), (i, PLAN[i].side, f)
    for r, o in zip(res, orcs):
        assert np.array_equal(np.concatenate([r["bounds_min"], r["bounds_max"]]), o.bounds)


def test_uneven_sample_300_steps_within_bar_and_equal(ctx):
    idx = pick(2)
    cloths, cols, srcs = build(idx, scenes.reference_params())
    assert {layout_of(c) for c in cloths} == {"shared memory", "lean x1", "lean arrays"}
    seen = {}

    def at_100(ids, orcs):
        seen[100] = max(float(np.max(np.abs(ctx.read_particles(i, len(o.particles))["position"]
                                            .astype(np.float64) - o.particles["position"])))
                        for i, o in zip(ids, orcs))

    got, orcs, _ = step_both(ctx, cloths, cols, srcs, 300, {100: at_100})
    assert seen[100] == 0.0
    for i, g, o in zip(idx, got, orcs):
        d = float(np.max(np.abs(g["position"].astype(np.float64) - o.particles["position"])))
        assert d <= 1e-3, (i, PLAN[i].side, d)
        pinned = o.particles["inv_mass"] == 0.0
        assert np.array_equal(g["position"][pinned], o.particles["position"][pinned])
        assert np.array_equal(g["position"], o.particles["position"]), (i, PLAN[i].side)
        # the sheets fell and met their colliders: not at rest where they started
        assert g["position"][:, 2].min() < 0.99
