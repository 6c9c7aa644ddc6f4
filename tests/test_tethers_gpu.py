"""cloth::build_tethers on the device (pxb_build_tethers_device) against the library's host
builder, which equals the reference's byte for byte (test_library_cpu.py): geodesic Dijkstra from
every anchor at once, each free particle tethered to the anchor it reached first. Ties between
anchors (a symmetric sheet pinned at both top corners) are where the order matters."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def same_tethers(a, b):
    return len(a) == len(b) and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def grid(side, jitter=0.0, seed=0, tether_scale=1.02):
    p = A.ClothParams.defaults()
    p.tether_scale = tether_scale
    w = 0.05 * (side - 1)
    return R.HostCloth(side, side, w, w, center=(0.0, 0.0, 1.0), params=p, jitter=jitter, seed=seed), w


def compare(ctx, make):
    host, dev = make(), make()
    host.build_tethers()
    dev.build_tethers_device(ctx)
    h, d = host.arrays().tethers, dev.arrays().tethers
    assert same_tethers(h, d), f"{len(h)} host vs {len(d)} device tethers"
    return h


def test_symmetric_sheet_ties_resolve_as_the_reference(ctx):
    def make():
        h, w = grid(32)
        h.pin_static((-w / 2, w / 2, 1.0), 0.01)
        h.pin_static((w / 2, w / 2, 1.0), 0.01)
        return h
    t = compare(ctx, make)
    assert len(t) == 32 * 32 - 2
    assert len(set(t["anchor"].tolist())) == 2  # both corners own particles


@pytest.mark.parametrize("side,seed", [(17, 1), (64, 2), (100, 3)])
def test_jittered_sheets_with_edge_and_corner_pins(ctx, side, seed):
    def make():
        h, w = grid(side, jitter=1e-3, seed=seed, tether_scale=1.1)
        for k in range(0, side, 5):  # every fifth particle of the top edge
            h.pin_static((-w / 2 + 0.05 * k, w / 2, 1.0), 0.015)
        h.pin_static((-w / 2, -w / 2, 1.0), 0.015)
        return h
    compare(ctx, make)


def test_mesh_cloth_and_body_anchors(ctx):
    v, ix = S.disc_mesh(0.5, 14, (0.0, 0.0, 1.0), jitter=0.25, seed=8)

    def make():
        h = R.HostCloth.from_mesh(v, ix)
        h.pin_to_body(0, 0, (0.5, 0.0, 1.0), (0.0, 0.0, 0.0, 1.0), (0.5, 0.0, 1.0), 0.06)
        h.pin_to_body(1, 0, (-0.5, 0.0, 1.0), (0.0, 0.0, 0.0, 1.0), (-0.5, 0.0, 1.0), 0.06)
        h.pin_static((0.0, 0.5, 1.0), 0.05)
        return h
    compare(ctx, make)


def test_unreached_island_and_no_anchors(ctx):
    v1, i1 = S.disc_mesh(0.3, 5, (0.0, 0.0, 1.0), jitter=0.2, seed=1)
    v2, i2 = S.disc_mesh(0.3, 4, (2.0, 0.0, 1.0), jitter=0.2, seed=2)
    v = np.concatenate([v1, v2])
    ix = np.concatenate([i1, i2 + len(v1)])

    def make():
        h = R.HostCloth.from_mesh(v, ix)
        h.pin_static((0.3, 0.0, 1.0), 0.03)
        return h
    t = compare(ctx, make)
    assert len(t) > 0 and t["particle"].max() < len(v1)  # the second disc is not reached
    bare = R.HostCloth.from_mesh(v, ix)
    bare.build_tethers_device(ctx)
    assert len(bare.arrays().tethers) == 0


def test_coincident_particles_are_refused(ctx):
    h, w = grid(12)
    h.pin_static((-w / 2, w / 2, 1.0), 0.01)
    h.build_tethers()
    before = h.arrays().tethers.copy()
    # move particle 40 onto particle 41: a zero-length stretch edge between distinct particles
    parts = h.mutable_particles()
    parts["position"][40] = parts["position"][41]
    with pytest.raises(R.PxbError) as e:
        h.build_tethers_device(ctx)
    assert e.value.status == A.PXB_ERR_UNSUPPORTED
    assert same_tethers(h.arrays().tethers, before)  # unchanged


def test_large_sheet(ctx):
    """A 256 x 256 sheet pinned along its top edge: about 256 relaxation rounds."""
    def make():
        h, w = grid(256, jitter=1e-3, seed=4)
        for k in range(0, 256, 3):
            h.pin_static((-w / 2 + 0.05 * k, w / 2, 1.0), 0.015)
        return h
    compare(ctx, make)
