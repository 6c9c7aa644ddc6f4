"""Parity of the device strand solver with the oracle (oracle/xpbd_oracle.c, solve_strands).

Stages without a transcendental call run in the reference's operation order in IEEE single
precision, and scenes that only use those (no local shape, no turning root, no wind) are asserted
EQUAL to the oracle, for strands of up to 32 particles (one lane per particle) and longer ones
(the long-strand kernel, lanes striding over the particles). The local-shape rotation (acos / sin / cos) and the slerp of a turning root
use CUDA's libm, which may differ from the host's by an ulp; those scenes are held to the bars:
within 1e-5 m after one step and 1e-3 m after many.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes
from physxcoopa_b200.arrays import box, capsule, collider_array, gravity_sources, sphere

import _checkers as K
from test_strands_oracle_ref import bent, params, straight

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def maxdiff(a, b):
    return float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)))) if a.size else 0.0


def run_pair(ctx, s, steps, cols=None, sources=None, iters=4, roots=None):
    orc = s.copy()
    sid = ctx.add_strands(s)
    try:
        for f in range(steps):
            if roots is not None:
                pos, rot = roots(f)
                ctx.set_strand_roots(sid, pos, rot)
                K.oracle_set_strand_roots(orc, pos, rot)
            ctx.step_strands([sid], None if cols is None else [cols],
                             sources=None if sources is None else [sources], iterations=iters)
            K.oracle_step_strands(orc, cols, sources=sources, iterations=iters)
        gpu = ctx.read_strand_particles(sid, len(s.particles))
        lam = ctx.read_strand_lambdas(sid, len(s.stretch))
        res = ctx.read_strand_results([sid])[0]
        t = ctx.read_strand_time(sid)
    finally:
        ctx.remove_strands(sid)
    return gpu, orc, lam, res, t


EXACT = {
    "hanging_no_shape": dict(lines=[straight((0, 0, 0), 10)], p=params(global_shape=0.0, local_shape=0.0)),
    "global_shape_only": dict(lines=[straight((0, 0, 0), 9), straight((0, 0.1, 0), 32)],
                              p=params(global_shape=0.5, global_shape_falloff=2.0, local_shape=0.0)),
    "collider_drape": dict(lines=[straight((0, 0, 0.6), 12)], p=params(global_shape=0.0, local_shape=0.0, thickness=0.02),
                           cols=[sphere(0.3)]),
    "three_colliders": dict(lines=[straight((0.02 * i, 0, 0.5), 10) for i in range(5)], p=params(local_shape=0.0),
                            cols=[sphere(0.2, (0.1, 0, 0.2)), capsule(0.1, 0.3, (0.2, 0.0, 0.3), axis=1),
                                  box((0.2, 0.2, 0.05), (0.1, 0.0, 0.1))]),
    "compliant": dict(lines=[straight((0, 0, 0), 16)], p=params(stretch_compliance=1e-5, local_shape=0.0), iters=7),
    "short_and_single": dict(lines=[straight((0, 0, 0), 2), straight((0, 0.2, 0), 3)], p=params(local_shape=0.0)),
    # strands longer than a warp (the long-strand kernel), alone and beside short ones
    "long_hanging": dict(lines=[straight((0, 0, 0), 100, 0.01)], p=params(global_shape=0.0, local_shape=0.0)),
    "long_mixed_drape": dict(lines=[straight((0, 0, 0.6), 40, 0.02), straight((0.05, 0, 0.6), 7, 0.02),
                                    straight((0.1, 0, 0.6), 65, 0.02), straight((0.15, 0.02, 0.6), 33, 0.02)],
                             p=params(local_shape=0.0, global_shape=0.3, thickness=0.02), cols=[sphere(0.3)]),
    "long_compliant": dict(lines=[straight((0, 0, 0), 257, 0.004)], p=params(stretch_compliance=1e-5, local_shape=0.0),
                           iters=7),
}


@pytest.mark.parametrize("name", sorted(EXACT))
def test_exact_scenes_equal_oracle(ctx, name):
    sc = EXACT[name]
    s = R.make_strands(sc["lines"], sc["p"])
    cols = collider_array(sc["cols"]) if "cols" in sc else None
    gpu, orc, lam, res, t = run_pair(ctx, s, 40, cols, iters=sc.get("iters", 4))
    for f in ("position", "velocity", "prev_position", "inv_mass"):
        assert np.array_equal(gpu[f], orc.particles[f]), f"{f}: {maxdiff(gpu[f], orc.particles[f])}"
    assert np.array_equal(lam, orc.stretch["lambda"])
    assert np.float32(t) == np.float32(orc.time)
    assert np.array_equal(res["bounds_min"], orc.bounds[:3]) and np.array_equal(res["bounds_max"], orc.bounds[3:])


TOLERANT = {
    "defaults": dict(lines=[straight((0, 0, 0))], p=params()),
    "local_shape_curl": dict(lines=[bent((0, 0, 0))], p=params(global_shape=0.0, local_shape=0.9)),
    "wind_turbulence": dict(lines=[straight((0, 0.02 * i, 0)) for i in range(4)],
                            p=params(wind=(1.0, 0.5, 0.0), wind_turbulence=0.7)),
    "many_with_collider": dict(lines=[straight((0.01 * i, 0.01 * (i % 7), 0.35), 32) for i in range(64)],
                               p=params(), cols=[sphere(0.3)]),
    # long strands hanging from their roots (combed straight down), local and global shape on
    "long_hanging_defaults": dict(lines=[np.array([[0.01 * i, 0.0, 0.35 - 0.01 * k] for k in range(48 + 17 * i)],
                                                  np.float32) for i in range(12)], p=params()),
}


@pytest.mark.parametrize("name", sorted(TOLERANT))
def test_transcendental_scenes_within_bars(ctx, name):
    sc = TOLERANT[name]
    s = R.make_strands(sc["lines"], sc["p"])
    cols = collider_array(sc["cols"]) if "cols" in sc else None
    gpu, orc, _, _, _ = run_pair(ctx, s, 1, cols)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    roots = orc.particles["inv_mass"] == 0
    assert np.array_equal(gpu["position"][roots], orc.particles["position"][roots])
    gpu, orc, _, _, _ = run_pair(ctx, s, 300, cols)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-3
    assert np.array_equal(gpu["position"][roots], orc.particles["position"][roots])


def test_long_strands_falling_onto_a_collider_one_step_bar(ctx):
    """Long strands (48 to 235 particles) falling from horizontal onto a sphere in a gusting wind:
    a chaotic multi-pendulum, in which an ulp of CUDA's libm against glibc's (local-shape
    rotation, gust) grows over the steps, so it is held to the one-step bar."""
    s = R.make_strands([straight((0.01 * i, 0.0, 0.35), 48 + 17 * i, 0.01) for i in range(12)],
                       params(wind=(0.5, 0.2, 0.0)))
    gpu, orc, _, _, _ = run_pair(ctx, s, 1, collider_array([sphere(0.3)]))
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    roots = orc.particles["inv_mass"] == 0
    assert np.array_equal(gpu["position"][roots], orc.particles["position"][roots])


def test_moving_and_turning_roots(ctx):
    s = R.make_strands([straight((0, 0, 0)), straight((0, 0.3, 0), 20)], params(global_shape=0.4))

    def roots(f):
        ang = 0.01 * f
        pos = np.array([[0.01 * f, 0, 0], [0.01 * f, 0.3, 0]], np.float32)
        rot = np.array([[0, 0, np.sin(ang / 2), np.cos(ang / 2)]] * 2, np.float32)
        return pos, rot
    gpu, orc, _, _, _ = run_pair(ctx, s, 120, roots=roots, iters=1)
    assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-3
    assert abs(gpu["position"][0][0] - 1.19) < 1e-3


def test_gravity_source_at_bounds_centre(ctx):
    s = R.make_strands([straight((0.05 * i, 0, 0), 12) for i in range(6)], params(local_shape=0.0))
    src = gravity_sources([((0.5, 0.3, -1.0), 9.81, 0.5, 10.0)])
    gpu, orc, _, _, _ = run_pair(ctx, s, 60, sources=src)
    assert np.array_equal(gpu["position"], orc.particles["position"])


def test_drop_in_solve_strands_on_host_arrays(ctx):
    mine = R.make_strands([straight((0, 0, 0.5), 12) for _ in range(3)], params(local_shape=0.0))
    orc = mine.copy()
    col = collider_array([sphere(0.3)])
    for _ in range(20):
        ctx.solve_strands_host(mine, col)
        K.oracle_step_strands(orc, col)
    assert np.array_equal(mine.particles["position"], orc.particles["position"])
    assert np.array_equal(mine.stretch["lambda"], orc.stretch["lambda"])
    assert np.float32(mine.time) == np.float32(orc.time)


def test_refusals(ctx):
    too_long = R.make_strands([straight((0, 0, 0), 8193, 0.001)])  # past one warp's shared memory
    with pytest.raises(R.PxbError) as e:
        ctx.add_strands(too_long)
    assert e.value.status == 7
    ok = R.make_strands([straight((0, 0, 0))])
    odd = ok.copy()
    odd.stretch = odd.stretch[::-1].copy()
    with pytest.raises(R.PxbError) as e:
        ctx.add_strands(odd)
    assert e.value.status == 2
    sid = ctx.add_strands(ok)
    ctx.remove_strands(sid)
    with pytest.raises(R.PxbError) as e:
        ctx.step_strands([sid])
    assert e.value.status == 5


def test_groom_sample_one_step_bar_and_physical_after_300(ctx):
    """A 256-strand sample of the groom workload (moving head, 20 iterations). The local-shape
    rotation calls acosf / sinf / cosf, whose CUDA results can differ from glibc's by an ulp; with
    contacts against a moving head that difference grows chaotically, so trajectory parity holds
    to the one-step bar (1e-5 m) and the 300-step state is checked for physical validity (roots
    exact; segment strain and head penetration no worse than the oracle's own on the same groom).
    The 300-step distance to the oracle is printed. The reference algorithm itself moves this
    groom by centimetres in 300 steps after a one-ulp change (test_strands_oracle_ref); stable
    hanging strands hold the 300-step bar (next test)."""
    sc = scenes.hair_groom(n_strands=256, iterations=20)
    s = sc.sets[0]
    orc = s.copy()
    sid = ctx.add_strands(s)
    roots = s.particles["inv_mass"] == 0
    for f in range(300):
        pos, rot = sc.root_path(f)
        ctx.set_strand_roots(sid, pos, rot)
        K.oracle_set_strand_roots(orc, pos, rot)
        cols = sc.meta["colliders_at"](f)
        ctx.step_strands([sid], [cols], iterations=sc.iterations)
        K.oracle_step_strands(orc, cols, iterations=sc.iterations)
        if f == 0:
            gpu = ctx.read_strand_particles(sid, len(s.particles))
            assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    gpu = ctx.read_strand_particles(sid, len(s.particles))
    print(f"groom sample, 300 steps: max |dp| to the oracle {maxdiff(gpu['position'], orc.particles['position']):.3g} m")
    pos = gpu["position"]
    assert np.array_equal(pos[roots], orc.particles["position"][roots])
    # physical state held to the oracle's own: segment strain and penetration of the head no
    # worse than the reference algorithm's on the same groom (with a small floor)
    st = s.stretch
    opos = orc.particles["position"]
    strain = np.abs(np.linalg.norm(pos[st["a"]] - pos[st["b"]], axis=1) / st["rest_length"] - 1.0)
    ostrain = np.abs(np.linalg.norm(opos[st["a"]] - opos[st["b"]], axis=1) / st["rest_length"] - 1.0)
    head = sc.meta["colliders_at"](299)[0]
    inside = (np.linalg.norm(pos - head["position"], axis=1) - head["radius"])[~roots].min()
    oinside = (np.linalg.norm(opos - head["position"], axis=1) - head["radius"])[~roots].min()
    print(f"max strain {strain.max():.4g} (oracle {ostrain.max():.4g}); deepest {inside:.4g} m "
          f"(oracle {oinside:.4g} m)")
    assert strain.max() <= max(0.01, 2.0 * ostrain.max())
    assert np.mean(strain) <= max(1e-3, 2.0 * np.mean(ostrain))
    assert inside >= min(-0.005, 2.0 * oinside)
    ctx.remove_strands(sid)


def test_hanging_strands_hold_300_step_bar(ctx):
    """Strands swinging to rest from tilted starts (a stable scene): the transcendental ulp
    differences stay damped and the 300-step state is within 1e-3 m of the oracle."""
    sc = scenes.hanging_strands(n_strands=256)
    s = sc.sets[0]
    orc = s.copy()
    sid = ctx.add_strands(s)
    roots = s.particles["inv_mass"] == 0
    for f in range(300):
        ctx.step_strands([sid], None, iterations=sc.iterations)
        K.oracle_step_strands(orc, None, iterations=sc.iterations)
        if f == 0:
            gpu = ctx.read_strand_particles(sid, len(s.particles))
            assert maxdiff(gpu["position"], orc.particles["position"]) <= 1e-5
    gpu = ctx.read_strand_particles(sid, len(s.particles))
    d = maxdiff(gpu["position"], orc.particles["position"])
    print(f"hanging strands, 300 steps: max |dp| to the oracle {d:.3g} m")
    assert d <= 1e-3
    assert np.array_equal(gpu["position"][roots], orc.particles["position"][roots])
    assert gpu["position"][:, 2].max() <= 1.0 + 1e-6  # hanging below the roots
    ctx.remove_strands(sid)
