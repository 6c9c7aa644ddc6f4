"""General-topology cloths on the host: the mesh builder (pxb_host_cloth_make_mesh) against a
Python restatement of its rule, the layout plan of cloths that are not make_grid_cloth's, and
the oracle against the reference's own solve_cloth (cloth_solver.h:158-460, which is
topology-agnostic) on such cloths. No GPU."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes as S
from physxcoopa_b200.arrays import collider_array, sphere

import _checkers as K

f32 = np.float32


def restated_mesh_cloth(v, ix, total_mass, bend):
    """pxb_host_cloth_make_mesh's rule in Python: returns (inv_mass, stretch pairs, stretch
    batches, bend pairs, bend batches) with the pairs in stored order."""
    n = len(v)
    mass = f32(total_mass) / f32(n) if total_mass > 1e-6 else f32(0)
    inv = f32(1) / mass if mass > f32(1e-6) else f32(0)
    edges, opposite, edge_of = [], [], {}
    t = ix.reshape(-1, 3)
    for tri in t:
        for e in range(3):
            a, b, o = int(tri[e]), int(tri[(e + 1) % 3]), int(tri[(e + 2) % 3])
            if a == b:
                continue
            k = (min(a, b), max(a, b))
            if k not in edge_of:
                edge_of[k] = len(edges)
                edges.append((a, b))
                opposite.append([])
            opposite[edge_of[k]].append(o)
    bends, seen = [], set()
    if bend:
        for e, opp in enumerate(opposite):
            if len(opp) != 2:
                continue
            a, b = opp
            k = (min(a, b), max(a, b))
            if a == b or k in edge_of or k in seen:
                continue
            seen.add(k)
            bends.append((a, b))

    def colour(pairs):
        used, of = [], []
        for a, b in pairs:
            c = 0
            while c < len(used) and (a in used[c] or b in used[c]):
                c += 1
            if c == len(used):
                used.append(set())
            used[c] |= {a, b}
            of.append(c)
        out, batches = [], []
        for c in range(len(used)):
            begin = len(out)
            out += [p for p, q in zip(pairs, of) if q == c]
            batches.append((begin, len(out)))
        return out, batches

    s, sb = colour(edges)
    b, bb = colour(bends)
    return inv, s, sb, b, bb


def rest_len(v, a, b):
    d = v[a] - v[b]
    return f32(np.sqrt(f32(f32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])))


@pytest.mark.parametrize("rings,bend", [(3, True), (9, True), (9, False)])
def test_mesh_builder_matches_its_rule(rings, bend):
    v, ix = S.disc_mesh(0.5, rings, (0.1, -0.2, 1.0), jitter=0.3, seed=rings)
    c = R.HostCloth.from_mesh(v, ix, total_mass=2.0, bend=bend).arrays()
    inv, s, sb, b, bb = restated_mesh_cloth(v, ix, 2.0, bend)
    assert np.array_equal(c.particles["position"], v) and np.array_equal(c.particles["prev_position"], v)
    assert np.all(c.particles["inv_mass"] == inv) and not c.particles["velocity"].any()
    assert [tuple(x) for x in c.stretch[["a", "b"]].tolist()] == s
    assert [tuple(x) for x in c.stretch_batches.tolist()] == sb
    assert [tuple(x) for x in c.bend[["a", "b"]].tolist()] == b
    assert [tuple(x) for x in c.bend_batches.tolist()] == bb
    for lst in (c.stretch, c.bend):
        want = np.array([rest_len(v, int(k["a"]), int(k["b"])) for k in lst], np.float32)
        assert np.array_equal(lst["rest_length"], want)
    assert np.array_equal(c.triangles, ix) and c.columns == 0 and c.rows == 0
    # every batch is particle-disjoint, the batches tile the list
    for lst, batches in ((c.stretch, c.stretch_batches), (c.bend, c.bend_batches)):
        assert (batches["begin"][1:] == batches["end"][:-1]).all() if len(batches) else len(lst) == 0
        for bt in batches:
            ends = np.concatenate([lst["a"][bt["begin"]:bt["end"]], lst["b"][bt["begin"]:bt["end"]]])
            assert len(np.unique(ends)) == len(ends)
    # the self-collision distance default: 0.6 x the mean edge length
    total = f32(0)
    for a, bb_ in s_first_order(v, ix):
        total = f32(total + rest_len(v, a, bb_))
    assert c.params.self_distance == f32(f32(0.6) * f32(total / f32(len(s))))


def s_first_order(v, ix):
    seen, out = set(), []
    for tri in ix.reshape(-1, 3):
        for e in range(3):
            a, b = int(tri[e]), int(tri[(e + 1) % 3])
            k = (min(a, b), max(a, b))
            if a != b and k not in seen:
                seen.add(k)
                out.append((a, b))
    return out


def test_mesh_builder_refusals():
    v, ix = S.disc_mesh(0.5, 2)
    with pytest.raises(R.PxbError):
        R.HostCloth.from_mesh(v, ix[:-1])          # not whole triangles
    bad = ix.copy()
    bad[4] = len(v)
    with pytest.raises(R.PxbError):
        R.HostCloth.from_mesh(v, bad)              # index past the vertices


def unbatched(c):
    """The same lists with every constraint in one batch per list: the reference then walks each
    list serially in list order."""
    u = c.copy()
    u.stretch_batches = np.array([(0, len(u.stretch))], A.BATCH)
    u.bend_batches = np.array([(0, len(u.bend))], A.BATCH)
    u.stretch_batch_compliance = None
    return u


def test_plan_general_topology():
    m = S.mesh_cloth(12)
    p = R.plan_cloth(m)
    assert p["topology"] == 1 and p["n_ranks"] == 1 and p["n_segments"] == 0 and p["self_collision"] == 1
    assert p["n_colours"] == len(m.stretch_batches) + len(m.bend_batches)  # one run per coloured batch
    g = S.single_drape().cloths[0]
    assert R.plan_cloth(g)["topology"] == 0
    u = R.plan_cloth(unbatched(g))
    # the grid's lists walked serially: a run ends where an item meets a particle of the run
    assert u["topology"] == 1 and u["n_colours"] == 12
    # non-grid triangles over grid lists: general layout
    t = g.copy()
    t.triangles = t.triangles.reshape(-1, 3)[:, [0, 2, 1]].reshape(-1).copy()
    assert R.plan_cloth(t)["topology"] == 1


def test_plan_general_topology_refusals():
    g = S.single_drape().cloths[0]
    twice = unbatched(g)
    twice.stretch_batches = np.array([(0, 10), (5, len(twice.stretch))], A.BATCH)
    with pytest.raises(R.PxbError) as e:
        R.plan_cloth(twice)
    assert e.value.status == A.PXB_ERR_UNSUPPORTED and "more than one batch" in str(e.value)
    past = unbatched(g)
    past.bend_batches = np.array([(0, len(past.bend) + 1)], A.BATCH)
    with pytest.raises(R.PxbError) as e:
        R.plan_cloth(past)
    assert e.value.status == A.PXB_ERR_UNSUPPORTED
    # 3571 particles, ~20k items: past one CTA's shared memory, so its state stays in HBM
    big = R.plan_cloth(S.mesh_cloth(34, tethers=False))
    assert big["topology"] == 2 and big["smem_bytes"] == 0 and big["n_ranks"] == 1 and big["threads"] <= 1024
    assert big["self_collision"] == 0  # its hash tables would need the shared memory it does not get
    # past the 16-bit slot of one packed endpoint word: two words per item, three times the
    # padded item count of rest-length and endpoint slots
    v, ix = S.disc_mesh(0.5, 149)  # 67,051 particles
    wide = R.plan_cloth(R.HostCloth.from_mesh(v, ix, bend=False).arrays())
    assert wide["topology"] == 2 and wide["layout_slots"] > 65535
    assert wide["constraint_slots"] % 3 == 0 and wide["constraint_slots"] // 3 % 4 == 0
    narrow = R.plan_cloth(S.mesh_cloth(34, tethers=False))
    assert narrow["constraint_slots"] % 2 == 0


def oracle_vs_reference(c, colliders, steps, iterations=10):
    ref = K.RefCloth.from_arrays(c)
    orc = c.copy()
    for _ in range(steps):
        ref.solve(colliders, iterations=iterations)
        K.oracle_step_cloth(orc, colliders, iterations=iterations)
    got = ref.arrays()
    for f in ("position", "velocity", "prev_position", "inv_mass"):
        assert np.array_equal(got.particles[f], orc.particles[f]), f
    assert np.array_equal(got.stretch["lambda"], orc.stretch["lambda"])
    assert np.array_equal(got.bend["lambda"], orc.bend["lambda"])


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")
def test_oracle_equals_reference_on_a_mesh_cloth():
    sc = S.mesh_drape(rings=8, seed=4)
    c = sc.cloths[0]
    c.params.has_shear_compliance = 0  # the reference has no per-batch compliance
    oracle_vs_reference(c, sc.colliders[0], steps=20)


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")
def test_oracle_equals_reference_on_a_mesh_cloth_past_16_bit_slots():
    """The 67,951-particle disc the device solves with two-word endpoints: oracle and compiled
    reference agree on it too."""
    sc = S.mesh_drape(rings=150, seed=9)
    c = sc.cloths[0]
    assert len(c.particles) > 65535
    c.params.has_shear_compliance = 0
    oracle_vs_reference(c, sc.colliders[0], steps=2)


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")
def test_oracle_equals_reference_on_serial_grid_lists():
    sc = S.single_drape(seed=6)
    c = unbatched(sc.cloths[0])
    c.params.has_shear_compliance = 0
    oracle_vs_reference(c, sc.colliders[0], steps=15)


def self_colliding_mesh(rings=10, seed=3):
    """A disc mesh pinned at one rim point with self_distance 2.2 x its mean edge: non-adjacent
    particles push on every substep (columns 0: no 1-ring exemption, as the reference reads it)."""
    p = S.cloth_params(self_collision=1, has_shear_compliance=0)
    c = S.mesh_cloth(rings, 0.5, (0.0, 0.0, 1.0), seed=seed, params=p, pins=[((0.5, 0.0, 1.0), 0.3 * 0.5 / rings)])
    c.params.self_distance = 2.2 * float(np.mean(c.stretch["rest_length"]))
    return c, collider_array([sphere(0.15, (0.1, 0.05, 0.7))])


def self_colliding_regrid():
    """The single drape's grid with its lists in one serial batch each and self_distance 2.2 x the
    spacing: general topology, the 1-ring exemption through the cloth's own columns (32)."""
    sc = S.single_drape(seed=9)
    c = unbatched(sc.cloths[0])
    c.params.has_shear_compliance = 0
    c.params.self_collision = 1
    c.params.self_distance = 2.2 * S.SPACING
    return c, sc.colliders[0]


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("scene", [self_colliding_mesh, self_colliding_regrid])
def test_oracle_equals_reference_with_self_collision_on_general_topology(scene):
    c, col = scene()
    assert R.plan_cloth(c)["topology"] == 1 and R.plan_cloth(c)["self_collision"] == 1
    oracle_vs_reference(c, col, steps=8)
