"""What a cloth's readers take from the device each frame: world_state_hash's cloth part
(pxb_cloths_state_hash, world.h:1334-1359) and a renderer's vertex buffer over Cloth::triangles
(pxb_cloths_read_render_buffer, cloth.h:293-299)."""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes as S

import _checkers as K

pytestmark = pytest.mark.gpu

FNV_BASIS = 1469598103934665603
FNV_PRIME = 1099511628211


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


def fnv1a(h, data: bytes):
    """FNV-1a 64 over `data`, continued from h (world.h:1336-1341)."""
    for b in data:
        h = ((h ^ b) * FNV_PRIME) & 0xFFFFFFFFFFFFFFFF
    return h


def state_bytes(particles):
    rec = np.zeros((len(particles), 6), np.float32)
    rec[:, :3] = particles["position"]
    rec[:, 3:] = particles["velocity"]
    return rec.tobytes()


def test_state_hash_equals_the_reference_mix_of_the_oracle_state(ctx):
    cloths = [S.single_drape(seed=s).cloths[0] for s in (1, 2)]
    cols = [S.single_drape(seed=s).colliders[0] for s in (1, 2)]
    ids = [ctx.add_cloth(c) for c in cloths]
    orc = [c.copy() for c in cloths]
    try:
        h0 = ctx.state_hash(ids)
        assert h0 == fnv1a(fnv1a(FNV_BASIS, state_bytes(orc[0].particles)), state_bytes(orc[1].particles))
        for _ in range(5):
            ctx.step(ids, cols)
            for o, c in zip(orc, cols):
                K.oracle_step_cloth(o, c)
        want = fnv1a(fnv1a(FNV_BASIS, state_bytes(orc[0].particles)), state_bytes(orc[1].particles))
        assert ctx.state_hash(ids) == want != h0
        # continued from a caller's seed (the bodies mixed before the cloths), and in list order
        seed = fnv1a(FNV_BASIS, b"bodies")
        assert ctx.state_hash(ids[::-1], seed) == fnv1a(fnv1a(seed, state_bytes(orc[1].particles)),
                                                        state_bytes(orc[0].particles))
    finally:
        for i in ids:
            ctx.remove_cloth(i)


def render_restated(pos, cols, rows):
    """The vertex normals of pxb_cloths_read_render_buffer in float32, in the same operation
    order: faces (i00, i10, i11) and (i00, i11, i01) of each cell, summed per particle in
    ascending triangle order, cross(b - a, c - a), then v * (1 / sqrt(dot(v, v)))."""
    P = pos.reshape(rows, cols, 3).astype(np.float32)
    out = np.zeros((rows * cols, 6), np.float32)
    f = np.float32

    def face(a, b, c, n):
        u = b - a
        v = c - a
        return np.array([n[0] + (u[1] * v[2] - v[1] * u[2]), n[1] + (u[2] * v[0] - v[2] * u[0]),
                         n[2] + (u[0] * v[1] - v[0] * u[1])], f)

    for y in range(rows):
        for x in range(cols):
            p = P[y, x]
            n = np.zeros(3, f)
            if x >= 1 and y >= 1:
                n = face(P[y - 1, x - 1], P[y - 1, x], p, n)
                n = face(P[y - 1, x - 1], p, P[y, x - 1], n)
            if x + 1 < cols and y >= 1:
                n = face(P[y - 1, x], P[y, x + 1], p, n)
            if x >= 1 and y + 1 < rows:
                n = face(P[y, x - 1], p, P[y + 1, x], n)
            if x + 1 < cols and y + 1 < rows:
                n = face(p, P[y, x + 1], P[y + 1, x + 1], n)
                n = face(p, P[y + 1, x + 1], P[y + 1, x], n)
            l2 = f(f(n[0] * n[0] + n[1] * n[1]) + n[2] * n[2])
            s = f(1.0) / np.sqrt(l2) if l2 > 0 else f(0.0)
            out[y * cols + x, :3] = p
            out[y * cols + x, 3:] = n * s
    return out


def test_render_buffer_positions_and_normals(ctx):
    plain = R.HostCloth(16, 16, 0.75, 0.75, center=(0.0, 0.0, 1.0)).arrays()  # no jitter: flat
    pid = ctx.add_cloth(plain)
    try:
        flat = ctx.read_render_buffer([pid], len(plain.particles))
        assert np.allclose(flat[:, 3:], (0.0, 0.0, 1.0), atol=1e-6)  # a flat sheet in the xy plane faces +z
    finally:
        ctx.remove_cloth(pid)
    sc = S.single_drape(seed=3)
    c = sc.cloths[0]
    cid = ctx.add_cloth(c)
    try:
        assert np.array_equal(ctx.read_render_buffer([cid], len(c.particles)).view(np.uint32),
                              render_restated(c.particles["position"], c.columns, c.rows).view(np.uint32))
        for _ in range(30):
            ctx.step([cid], sc.colliders)
        buf = ctx.read_render_buffer([cid], len(c.particles))
        pos = ctx.read_particles(cid, len(c.particles))["position"]
        assert np.array_equal(buf[:, :3], pos)
        want = render_restated(pos, c.columns, c.rows)
        assert np.array_equal(buf.view(np.uint32), want.view(np.uint32))
        lens = np.linalg.norm(buf[:, 3:].astype(np.float64), axis=1)
        assert np.allclose(lens, 1.0, atol=1e-6)
    finally:
        ctx.remove_cloth(cid)


def test_render_buffer_refusals(ctx):
    c = S.single_drape().cloths[0]
    bare = c.copy()
    bare.triangles = bare.triangles[:0].copy()
    bare.params.air_drag = 0.0
    bare.params.air_lift = 0.0
    cid = ctx.add_cloth(bare)
    try:
        with pytest.raises(R.PxbError) as e:
            ctx.read_render_buffer([cid], len(c.particles))
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
        with pytest.raises(R.PxbError) as e:
            ctx.read_render_buffer([cid], 10)  # output too small
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    finally:
        ctx.remove_cloth(cid)


def test_pipelined_position_reads(ctx):
    """pxb_cloths_read_positions_async: each call snapshots the state after the steps before it
    and lands it in its own buffer while the next step runs; a third call in flight reuses the
    first snapshot buffer once its copy has landed."""
    sc = S.single_drape(seed=4)
    c = sc.cloths[0]
    n = len(c.particles)
    cid = ctx.add_cloth(c)
    orc = c.copy()
    try:
        bufs = [np.zeros(3 * n, np.float32) for _ in range(3)]
        want = []
        for k in range(3):
            ctx.step([cid], sc.colliders)
            K.oracle_step_cloth(orc, sc.colliders[0])
            want.append(orc.particles["position"].copy())
            ctx.read_positions_async([cid], bufs[k])
        ctx.wait_positions()
        for k in range(3):
            assert np.array_equal(bufs[k].reshape(-1, 3), want[k]), k
        with pytest.raises(R.PxbError) as e:
            ctx.read_positions_async([cid], np.zeros(3 * n - 1, np.float32))
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    finally:
        ctx.remove_cloth(cid)


def test_pipelined_results_reads(ctx):
    """pxb_cloths_read_results_async: the last step's per-cloth results in the caller's order,
    equal to the blocking read, landing while the next step runs."""
    cloths = [S.single_drape(seed=s).cloths[0] for s in (5, 6, 7)]
    cols = [S.single_drape(seed=s).colliders[0] for s in (5, 6, 7)]
    ids = [ctx.add_cloth(c) for c in cloths]
    try:
        got = [np.zeros(3, A.FRAME_RESULT) for _ in range(2)]
        want = []
        for k in range(2):
            ctx.step(ids, cols)
            want.append(ctx.read_results(ids[::-1]).copy())
            ctx.read_results_async(ids[::-1], got[k])
        ctx.wait_positions()
        for k in range(2):
            assert np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)), k
        with pytest.raises(R.PxbError) as e:
            ctx.step(ids[:1], cols[:1])
            ctx.read_results_async(ids[1:], got[0][:2])  # not in the last step
        assert e.value.status == A.PXB_ERR_INVALID_ARGUMENT
    finally:
        for i in ids:
            ctx.remove_cloth(i)
