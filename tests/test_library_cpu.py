"""The C-ABI library on a machine without a GPU: it loads, exports every declared symbol,
refuses to make a context cleanly, and its host builders reproduce the reference's builders
(physxcoopa/cloth/cloth_builder.h) array for array, bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R

import _checkers as K

HEADER = os.path.join(K.ROOT, "include", "physxcoopa_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pxb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = R.library()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"
    assert set(syms) == set(R.SIGNATURES), "runtime.py signature table is out of step with the header"


def test_context_create_fails_cleanly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = R.library()
    h = C.c_void_p()
    st = lib.pxb_context_create(0, C.byref(h))
    assert st == 3  # PXB_ERR_CUDA
    assert not h.value


def test_params_default_match_reference():
    lib = R.library()
    p = A.ClothParams()
    lib.pxb_cloth_params_default(C.byref(p))
    q = A.ClothParams.defaults()
    assert bytes(p) == bytes(q)


def _same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


GRIDS = [dict(res=2), dict(res=3), dict(res=5, jitter=1e-3), dict(res=9, shear=False),
         dict(res=16, jitter=1e-3, seed=11), dict(res=7, center=(1.0, -2.0, 3.0),
                                                  orientation=(0.2, 0.1, 0.3, 0.9273618)),
         dict(res=13, width=3.0, height=1.0)]


@pytest.mark.skipif(not K.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("g", GRIDS, ids=[str(i) for i in range(len(GRIDS))])
def test_builders_match_reference_bitwise(g):
    from test_oracle_ref import grid_desc
    res = g["res"]
    kw = dict(center=g.get("center", (0, 0, 2)), width=g.get("width", 4.0),
              height=g.get("height", 4.0), shear=g.get("shear", True), jitter=g.get("jitter", 0.0),
              seed=g.get("seed", 7), orientation=g.get("orientation", (0, 0, 0, 1)))
    ref = K.RefCloth.make_grid(grid_desc(res, **kw))
    mine = R.HostCloth(res, res, kw["width"], kw["height"], center=kw["center"],
                       orientation=kw["orientation"], shear=kw["shear"], jitter=kw["jitter"],
                       seed=kw["seed"])
    corner = ref.arrays().particles["position"][0]
    assert ref.pin_static(tuple(corner), 0.3) == mine.pin_static(tuple(corner), 0.3)
    ref.build_tethers()
    mine.build_tethers()
    a, b = ref.arrays(), mine.arrays()
    for f in ("particles", "stretch", "stretch_batches", "bend", "bend_batches", "tethers",
              "anchors", "triangles"):
        assert _same(getattr(a, f), getattr(b, f)), f
    assert a.columns == b.columns and a.rows == b.rows
    assert np.float32(a.params.self_distance) == np.float32(b.params.self_distance)


def test_shear_compliance_extension_marks_the_shear_batches():
    p = A.ClothParams.defaults()
    p.has_shear_compliance = 1
    p.shear_compliance = 1e-6
    p.stretch_compliance = 0.0
    c = R.HostCloth(6, 6, 1.0, 1.0, params=p).arrays()
    assert list(c.stretch_batch_compliance) == [0.0] * 4 + [np.float32(1e-6)] * 4
    c2 = R.HostCloth(6, 6, 1.0, 1.0, params=p, shear=False).arrays()
    assert list(c2.stretch_batch_compliance) == [0.0] * 4
