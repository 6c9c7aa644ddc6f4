"""Hair: the oracle's solve_strands restatement and the library's make_strands, pinned to the
reference's own code (oracle/_ref) bit for bit, plus the reference hair tests' known answers
(tests/hair_solver_test.cpp) against the oracle."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200.arrays import box, capsule, collider_array, sphere

import _checkers as K

pytestmark = pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")


def straight(root, count=8, spacing=0.05):
    """hair_solver_test.cpp:42-48: a strand running +X from `root`."""
    return np.array([np.asarray(root, np.float32) + np.array([spacing * k, 0, 0], np.float32)
                     for k in range(count)], np.float32)


def bent(root, spacing=0.05):
    """hair_solver_test.cpp:57-66: out along +X, then along +Y."""
    r = np.asarray(root, np.float32)
    pts = [r + np.array([spacing * k, 0, 0], np.float32) for k in range(4)]
    pts += [r + np.array([spacing * 3, spacing * k, 0], np.float32) for k in range(1, 5)]
    return np.array(pts, np.float32)


def params(**kw):
    p = A.StrandParams.defaults()
    for k, v in kw.items():
        setattr(p, k, (A.C.c_float * 3)(*v) if isinstance(v, tuple) else v)
    return p


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


def test_builder_matches_reference_bitwise():
    rng = np.random.default_rng(0)
    lines = [straight((0.05 * i, 0, 0), count=int(rng.integers(2, 12))) for i in range(7)]
    lines.append(straight((0, 0, 1), count=1))  # fewer than two points: skipped
    lines.append(bent((0.3, 0.2, 0.1)))
    rot = np.array([[0, 0, 0.38268343, 0.9238795]] * len(lines), np.float32)
    mass = rng.uniform(0.0005, 0.002, len(lines)).astype(np.float32)
    p = params()
    ref = K.RefStrands.make(lines, p, rot, mass).arrays(p)
    mine = R.make_strands(lines, p, rot, mass)
    for f in ("particles", "stretch", "stretch_batches", "rest_local", "rest_offset", "strands"):
        assert same(getattr(ref, f), getattr(mine, f)), f


SCENES = {
    "defaults": dict(lines=lambda: [straight((0, 0, 0))], frames=60),
    "hanging_no_shape": dict(lines=lambda: [straight((0, 0, 0), 10)], p=params(global_shape=0.0, local_shape=0.0),
                             frames=60),
    "global_shape_falloff": dict(lines=lambda: [straight((0, 0, 0), 9)],
                                 p=params(global_shape=0.5, global_shape_falloff=2.0, local_shape=0.0), frames=60),
    "local_shape_curl": dict(lines=lambda: [bent((0, 0, 0))], p=params(global_shape=0.0, local_shape=0.9), frames=60),
    "collider_drape": dict(lines=lambda: [straight((0, 0, 0.6), 12)], p=params(global_shape=0.0, local_shape=0.0,
                                                                                thickness=0.02),
                           cols=lambda: [sphere(0.3)], frames=80),
    "three_colliders": dict(lines=lambda: [straight((0.02 * i, 0, 0.5), 10) for i in range(5)],
                            cols=lambda: [sphere(0.2, (0.1, 0, 0.2)), capsule(0.1, 0.3, (0.2, 0.0, 0.3), axis=1),
                                          box((0.2, 0.2, 0.05), (0.1, 0.0, 0.1))], frames=50),
    "wind_turbulence": dict(lines=lambda: [straight((0, 0.02 * i, 0)) for i in range(4)],
                            p=params(wind=(1.0, 0.5, 0.0), wind_turbulence=0.7), frames=40),
    "compliant_iters": dict(lines=lambda: [straight((0, 0, 0), 16)], p=params(stretch_compliance=1e-5),
                            frames=40, iters=7),
    "long_strands_curl_collider": dict(lines=lambda: [straight((0.01 * i, 0, 0.35), 40 + 29 * i, 0.01) for i in range(4)],
                                       p=params(wind=(0.5, 0.2, 0.0)), cols=lambda: [sphere(0.3)], frames=40),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_oracle_matches_reference_bitwise(name):
    sc = SCENES[name]
    p = sc.get("p", params())
    ref = K.RefStrands.make(sc["lines"](), p)
    orc = ref.arrays(p)
    cols = collider_array(sc["cols"]()) if "cols" in sc else None
    iters = sc.get("iters", 4)
    for _ in range(sc["frames"]):
        ref.solve(cols, substeps=4, iterations=iters)
        K.oracle_step_strands(orc, cols, substeps=4, iterations=iters)
    got = ref.arrays(p)
    for f in ("position", "velocity", "prev_position", "inv_mass"):
        assert same(orc.particles[f], got.particles[f]), f
    assert same(orc.stretch["lambda"], got.stretch["lambda"])
    assert np.float32(orc.time) == np.float32(got.time)
    assert same(orc.bounds, got.bounds)


def test_moving_and_turning_roots_match_reference():
    """hair_solver_test.cpp:183-203, with a turning root orientation added (slerp path)."""
    p = params(global_shape=0.4)
    ref = K.RefStrands.make([straight((0, 0, 0))], p)
    orc = ref.arrays(p)
    for i in range(120):
        pos = np.array([[0.01 * i, 0, 0]], np.float32)
        ang = 0.01 * i
        rot = np.array([[0, 0, np.sin(ang / 2), np.cos(ang / 2)]], np.float32)
        ref.set_roots(pos, rot)
        K.oracle_set_strand_roots(orc, pos, rot)
        ref.solve(None, substeps=4, iterations=1)
        K.oracle_step_strands(orc, None, substeps=4, iterations=1)
    got = ref.arrays(p)
    assert same(orc.particles["position"], got.particles["position"])
    assert abs(got.particles["position"][0][0] - 1.19) < 1e-3


# --- the reference's hair test known answers (hair_solver_test.cpp), on the oracle -----------

def _run(s, frames, cols=None, iters=4):
    for _ in range(frames):
        K.oracle_step_strands(s, cols, substeps=4, iterations=iters)
    return s


def _length(s, i=0):
    st = s.strands[i]
    pos = s.particles["position"][st["first"]:st["first"] + st["count"]]
    return float(np.sum(np.linalg.norm(np.diff(pos, axis=0), axis=1)))


def test_roots_pinned_and_the_rest_not():
    s = R.make_strands([straight((0, 0, 0))])
    assert s.particles["inv_mass"][0] == 0 and s.particles["inv_mass"][1] > 0 and len(s.stretch) == 7
    root = s.particles["position"][0].copy()
    _run(s, 60)
    assert np.linalg.norm(s.particles["position"][0] - root) < 1e-5
    assert s.particles["position"][7][2] < root[2] - 0.005


def test_hanging_strand_does_not_stretch():
    s = R.make_strands([straight((0, 0, 0), 10)], params(global_shape=0.0, local_shape=0.0))
    rest = _length(s)
    assert abs(rest - 0.45) < 1e-4
    _run(s, 180)
    assert abs(_length(s) - rest) < 0.01 * rest
    assert s.particles["position"][9][2] < -0.3


def test_strand_stays_out_of_a_collider():
    s = R.make_strands([straight((0, 0, 0.6), 12)], params(global_shape=0.0, local_shape=0.0, thickness=0.02))
    _run(s, 300, collider_array([sphere(0.3)]))
    assert (np.linalg.norm(s.particles["position"], axis=1) - 0.3).min() > -0.005


def _bumped_run(sc, steps, bump):
    """Steps a scene in the oracle; `bump` moves one particle per strand by one ulp first."""
    s = sc.sets[0].copy()
    if bump:
        p = s.particles["position"]
        idx = np.arange(5, len(p), 32)
        p[idx, 0] = np.nextafter(p[idx, 0], np.float32(1))
    for f in range(steps):
        if sc.root_path is not None:
            pos, rot = sc.root_path(f)
            K.oracle_set_strand_roots(s, pos, rot)
        K.oracle_step_strands(s, None, iterations=sc.iterations)
    return s.particles["position"].copy()


def test_groom_trajectories_amplify_one_ulp_in_the_reference_algorithm():
    """Why the groom's 300-step state is not held to 1e-3 m: in the reference algorithm itself
    (the oracle equals the compiled reference bit for bit), strands growing upward buckle under
    gravity, and a one-ulp change of one particle per strand grows to centimetres in 300 steps.
    An implementation whose acosf / sinf / cosf differ from glibc's in the last bit (the device's
    do) cannot stay within the bar there. Strands hanging from their roots are stable: the same
    one-ulp change stays at micrometres, and the device is held to the bar on them."""
    from physxcoopa_b200 import scenes
    groom = scenes.hair_groom(n_strands=64, iterations=20)
    d_groom = np.abs(_bumped_run(groom, 300, False) - _bumped_run(groom, 300, True)).max()
    hang = scenes.hanging_strands(n_strands=64)
    d_hang = np.abs(_bumped_run(hang, 300, False) - _bumped_run(hang, 300, True)).max()
    print(f"one-ulp bump after 300 steps: groom {d_groom:.3g} m, hanging {d_hang:.3g} m")
    assert d_groom > 1e-3
    assert d_hang < 1e-4
