"""Device layout planning on the host (pxb_cloth_plan_layout): no GPU needed.

pxb_cloth_add recognises a make_grid_cloth sheet, chooses how many CTAs hold it (a cloth whose
positions, rest lengths and lambdas overflow one CTA's shared memory is split by rows over a
thread-block cluster), restricts every colour's affine segments to each CTA's rows and verifies
every device item against the reference constraint it replaces. The same planner runs here on the
CPU, so these tests cover the verification for every size of the uneven benchmark batch.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes

SMEM_LIMIT = 232448 - 4352  # sm_100 per-block limit minus the kernel's static shared memory


def sheet(cols, rows, shear=True, params=None):
    w = 0.05 * (cols - 1)
    hgt = 0.05 * (rows - 1)
    return R.HostCloth(cols, rows, w, hgt, shear=shear, params=params or scenes.cloth_params(),
                       jitter=1e-3, seed=cols * 1000 + rows).arrays()


def test_every_uneven_batch_side_plans():
    for side in range(16, 129):
        p = R.plan_cloth(sheet(side, side))
        assert p["n_ranks"] in (1, 2, 4, 8)
        assert 0 < p["smem_bytes"] <= SMEM_LIMIT
        assert p["rows_per_rank"] * p["n_ranks"] >= side
        assert p["rows_per_rank"] >= 2
        assert p["threads"] % 32 == 0 and 64 <= p["threads"] <= 1024
        assert p["layout_slots"] == side * 4 * ((side + 3) // 4)
        assert p["n_colours"] == 16


def test_headline_sheet_stays_in_one_cta():
    p = R.plan_cloth(sheet(64, 64))
    assert p["n_ranks"] == 1 and p["threads"] == 1024


@pytest.mark.parametrize("shape", [(2, 2), (5, 5), (17, 6), (128, 16), (16, 128), (3, 200),
                                   (200, 3), (97, 61), (64, 65), (150, 150)])
@pytest.mark.parametrize("shear", [True, False])
def test_rectangles_and_no_shear_plan(shape, shear):
    p = R.plan_cloth(sheet(*shape, shear=shear))
    assert p["smem_bytes"] <= SMEM_LIMIT
    assert p["n_colours"] == (16 if shear else 12) or min(shape) < 8


def test_aero_off_needs_less_memory():
    on = R.plan_cloth(sheet(64, 64))
    off = R.plan_cloth(sheet(64, 64, params=scenes.cloth_params(air_drag=0.0, air_lift=0.0)))
    assert off["smem_bytes"] <= on["smem_bytes"]


def test_beyond_a_cluster_plans_the_whole_gpu_path():
    for side in (181, 256, 512):
        p = R.plan_cloth(sheet(side, side))
        assert p["n_ranks"] == 0 and p["smem_bytes"] == 0 and p["rows_per_rank"] == side


def test_refusals_match_add_cloth():
    ok = sheet(9, 9)
    odd = ok.copy()
    odd.stretch = odd.stretch[::-1].copy()
    assert R.plan_cloth(odd)["topology"] == 1  # not make_grid_cloth's lists: the general layout
    past = ok.copy()
    past.stretch_batches = past.stretch_batches.copy()
    past.stretch_batches[-1]["end"] = len(past.stretch) + 1
    with pytest.raises(R.PxbError) as e:
        R.plan_cloth(past)
    assert e.value.status == 2
    empty = ok.copy()
    empty.particles = empty.particles[:0]
    with pytest.raises(R.PxbError) as e:
        R.plan_cloth(empty)
    assert e.value.status == 1



def test_self_collision_plans_on_one_cta_only():
    """Self-collision (cloth_solver.h:291-366) runs on cloths one CTA holds: its hash tables go in
    the rest-length region when they fit there, else after the lambdas. Clusters and the
    whole-GPU path report that a step with it enabled would be refused."""
    p = A.ClothParams.defaults()
    p.self_collision = 1
    p.self_distance = 0.1
    for side in (9, 25, 64):
        plan = R.plan_cloth(sheet(side, side, params=p))
        assert plan["n_ranks"] == 1 and plan["self_collision"] == 1
        assert plan["self_smem_bytes"] >= plan["smem_bytes"]
        assert plan["self_smem_bytes"] <= 232448 - 4608
    for side in (100, 512):
        plan = R.plan_cloth(sheet(side, side, params=p))
        assert plan["self_collision"] == 0
    # every constraint list cleared (the reference's own self-collision tests do this): no colour
    free = sheet(9, 9, params=p)
    for f in ("stretch", "bend", "stretch_batches", "bend_batches"):
        setattr(free, f, getattr(free, f)[:0].copy())
    plan = R.plan_cloth(free)
    assert plan["n_colours"] == 0 and plan["self_collision"] == 1
    assert plan["self_smem_bytes"] > plan["smem_bytes"]  # no rest lengths to borrow


def test_swapped_pair_is_caught_by_item_verification():
    """Reversing one bend constraint's endpoints keeps the lists' shape but not the grid
    segments' (a, b) order: the grid layout must not take it (it would solve a different pair
    order); the general layout, which keeps every pair as listed, does."""
    c = sheet(20, 20)
    assert R.plan_cloth(c)["topology"] == 0
    k = len(c.bend) // 2
    a, b = int(c.bend[k]["a"]), int(c.bend[k]["b"])
    c.bend[k]["a"], c.bend[k]["b"] = b, a
    assert R.plan_cloth(c)["topology"] == 1


@pytest.mark.parametrize("shape,shear", [((16, 16), True), ((64, 64), True), ((96, 96), True), ((128, 128), True),
                                         ((33, 20), False), ((150, 130), True)])
def test_disjoint_bend_colours_share_a_phase(shape, shear):
    """On one CTA, consecutive colours that touch disjoint particles run as one phase with no
    barrier between them: the row bends of phases 0 and 1 (columns x = 0, 2 mod 4 against 1, 3),
    of 2 and 3, and the same for the column bends. Every other pair of consecutive colours shares
    particles, so a sheet's 16 colours (12 without shear) take 12 phases (8). Clusters keep a
    barrier after every colour."""
    plan = R.plan_cloth(sheet(*shape, shear=shear))
    n_colours = 16 if shear else 12
    assert plan["n_colours"] == n_colours
    if plan["n_ranks"] == 1:
        assert plan["phases"] == n_colours - 4
    else:
        assert plan["phases"] == n_colours


def expected_phases(c):
    """Phases per iteration restated from the cloth's own batches: the non-empty batches in the
    reference's order (stretch, then bend), a phase growing while the next batch shares no
    particle with any batch already in it."""
    sets = []
    for cons, batches in ((c.stretch, c.stretch_batches), (c.bend, c.bend_batches)):
        for b in batches:
            part = cons[int(b["begin"]):int(b["end"])]
            if len(part):
                sets.append(set(part["a"].tolist()) | set(part["b"].tolist()))
    phases, cur = 0, None
    for s in sets:
        if cur is not None and not (cur & s):
            cur |= s
        else:
            phases += 1
            cur = set(s)
    return phases


@pytest.mark.parametrize("shape", [(2, 2), (3, 3), (2, 7), (5, 3), (4, 9), (7, 7), (9, 4), (17, 5), (30, 31), (44, 44)])
@pytest.mark.parametrize("shear", [True, False])
def test_phases_match_a_restatement_from_the_batches(shape, shear):
    """The host's phase split (colour_sync_mask) against the same rule applied to the reference's
    own batches, on sheets small enough that some colours are empty and others lose their
    neighbours."""
    c = sheet(*shape, shear=shear)
    plan = R.plan_cloth(c)
    assert plan["n_ranks"] == 1 and plan["topology"] == 0
    assert plan["phases"] == expected_phases(c)
