"""pxb_cloths_gather_positions_device, the gather entry point that allocates nothing.

Some callers may not allocate device memory while they run: a renderer or recorder reading
cloth positions every frame inside a fixed device memory budget, or code where cudaMalloc and
cudaFree would synchronise the device. This entry point writes into the caller's device buffer
and keeps its per-call cloth list in a fixed array compiled into the library. Its output must
equal pxb_cloths_read_positions' exactly, call after call (the shared array keeps the previous
call's contents, which must not leak into the next), and it must refuse what does not fit.

This file is named to be collected last, so a run that stops at the first failure has run every
other test before it.
"""
import numpy as np
import pytest

from physxcoopa_b200 import runtime as R
from physxcoopa_b200 import scenes
from physxcoopa_b200.arrays import collider_array, sphere

pytestmark = pytest.mark.gpu


def sheets():
    cloths, cols = [], []
    for k, side in enumerate((7, 33, 64, 80, 130)):  # one CTA, and clusters of 4 and 8
        w = 0.05 * (side - 1)
        h = R.HostCloth(side, side, w, w, center=(0, 0, 1), params=scenes.cloth_params(), jitter=1e-3, seed=40 + k)
        h.pin_static((-w / 2, w / 2, 1), 0.02)
        h.pin_static((w / 2, w / 2, 1), 0.02)
        h.build_tethers()
        cloths.append(h.arrays())
        cols.append(collider_array([sphere(0.3, (0.05 * k, 0, 0.5))]))
    return cloths, cols


def test_device_gather_equals_host_read_on_consecutive_calls():
    import torch
    ctx = R.Context(0)
    try:
        cloths, cols = sheets()
        ids = [ctx.add_cloth(c) for c in cloths]
        total = 3 * sum(len(c.particles) for c in cloths)
        dev = torch.full((total,), float("nan"), dtype=torch.float32, device="cuda")
        for call in range(2):
            ctx.step(ids, cols)
            host = np.zeros(total, np.float32)
            ctx.read_positions(ids, host)
            ctx.gather_positions_device(ids, dev.data_ptr(), total)
            ctx.synchronize()
            got = dev.cpu().numpy()
            assert np.array_equal(got, host), f"call {call}"
        # a shorter list, in another order, after the longer one: no stale entries
        sub = [ids[3], ids[0]]
        n_sub = 3 * (len(cloths[3].particles) + len(cloths[0].particles))
        host = np.zeros(n_sub, np.float32)
        ctx.read_positions(sub, host)
        out = torch.zeros(n_sub, dtype=torch.float32, device="cuda")
        ctx.gather_positions_device(sub, out.data_ptr(), n_sub)
        ctx.synchronize()
        assert np.array_equal(out.cpu().numpy(), host)
    finally:
        ctx.close()


def test_device_gather_allocates_nothing():
    """On a fresh context, after one step and with nothing read back yet (so no buffer of the
    host read path exists), the gather leaves the device's free memory unchanged; its output is
    compared with pxb_cloths_read_positions only afterwards."""
    import torch
    ctx = R.Context(0)
    try:
        cloths, cols = sheets()
        ids = [ctx.add_cloth(c) for c in cloths]
        total = 3 * sum(len(c.particles) for c in cloths)
        out = torch.zeros(total, dtype=torch.float32, device="cuda")
        ctx.step(ids, cols)
        ctx.synchronize()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(2):
            ctx.gather_positions_device(ids, out.data_ptr(), total)
        ctx.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, f"device memory changed by {free0 - free1} bytes across the gathers"
        host = np.zeros(total, np.float32)
        ctx.read_positions(ids, host)
        assert np.array_equal(out.cpu().numpy(), host)
    finally:
        ctx.close()


def test_device_gather_refusals():
    import torch
    ctx = R.Context(0)
    try:
        cloths, cols = sheets()
        ids = [ctx.add_cloth(c) for c in cloths[:2]]
        out = torch.zeros(8, dtype=torch.float32, device="cuda")
        with pytest.raises(R.PxbError) as e:  # registry not on the device yet
            ctx.gather_positions_device(ids, out.data_ptr(), 8)
        assert e.value.status == 1
        ctx.step(ids, cols[:2])
        with pytest.raises(R.PxbError) as e:  # output too small
            ctx.gather_positions_device(ids, out.data_ptr(), 8)
        assert e.value.status == 1
        with pytest.raises(R.PxbError) as e:  # more cloths than the fixed array holds
            ctx.gather_positions_device([ids[0]] * 4097, out.data_ptr(), 8)
        assert e.value.status == 7
    finally:
        ctx.close()
