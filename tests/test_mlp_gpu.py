"""The warm-start network on the tensor cores (tcgen05 BF16 MMAs, FP32 accumulation in TMEM)
against a float64 restatement of the same network.

The reference restates the device's roundings: weights, normalised inputs and hidden
activations rounded to bf16 (round to nearest even), so what remains is the accumulation order
and the exponential in SiLU. Where an activation sits next to a bf16 rounding boundary the two
round it to neighbouring values (one bf16 ulp, 2^-8 relative), so the bar is a mean error of
2e-4 and a worst case of 1e-2, relative to the output scale. A plain float32 network without the
bf16 roundings is held to 3e-2.
"""
import numpy as np
import pytest

from physxcoopa_b200 import _abi as A
from physxcoopa_b200 import runtime as R

pytestmark = pytest.mark.gpu


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(x):
    return x / (1.0 + np.exp(-x))


def reference(W, x, round_bf16=True):
    q = bf16 if round_bf16 else (lambda v: np.asarray(v, np.float64))
    xn = q((x - W["in_mean"]) * W["in_scale"])
    h1 = q(silu(xn @ q(W["w1"]).T + W["b1"]))
    h2 = q(silu(h1 @ q(W["w2"]).T + W["b2"]))
    return (h2 @ q(W["w3"]).T + W["b3"]) * W["out_scale"]


def random_weights(rng):
    W = {"w1": rng.normal(0, 1 / np.sqrt(24), (64, 24)), "b1": rng.normal(0, 0.1, 64),
         "w2": rng.normal(0, 1 / np.sqrt(64), (64, 64)), "b2": rng.normal(0, 0.1, 64),
         "w3": rng.normal(0, 1 / np.sqrt(64), (3, 64)), "b3": rng.normal(0, 0.1, 3),
         "in_mean": rng.normal(0, 0.5, 24), "in_scale": rng.uniform(0.5, 2.0, 24),
         "out_scale": np.array([1e-3, 2e-3, 5e-4])}
    return {k: np.asarray(v, np.float32) for k, v in W.items()}


@pytest.fixture(scope="module")
def ctx():
    c = R.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("n", [1, 127, 128, 129, 1000, 70000])
def test_network_matches_reference(ctx, n):
    rng = np.random.default_rng(n)
    W = random_weights(rng)
    ctx.set_mlp(A.MlpWeights.from_numpy(**W))
    x = rng.normal(0, 1, (n, 24)).astype(np.float32)
    y = ctx.mlp_infer(x).astype(np.float64)
    ref = reference(W, x)
    scale = W["out_scale"].astype(np.float64)
    err = np.abs(y - ref) / scale
    assert err.mean() <= 2e-4, err.mean()
    assert err.max() <= 1e-2, err.max()
    loose = np.abs(y - reference(W, x, round_bf16=False)) / scale
    assert loose.max() <= 3e-2, loose.max()


def test_weights_round_trip_and_refusals(ctx):
    rng = np.random.default_rng(7)
    W = random_weights(rng)
    ctx.set_mlp(A.MlpWeights.from_numpy(**W))
    back = ctx.get_mlp().as_numpy()
    for k, v in W.items():
        assert np.array_equal(back[k], v)
    bad = dict(W)
    bad["w2"] = W["w2"].copy()
    bad["w2"][3, 4] = np.nan
    with pytest.raises(R.PxbError) as e:
        ctx.set_mlp(A.MlpWeights.from_numpy(**bad))
    assert e.value.status == 1
    assert np.array_equal(ctx.get_mlp().as_numpy()["w2"], W["w2"])  # the old network stays


def test_deterministic(ctx):
    rng = np.random.default_rng(9)
    ctx.set_mlp(A.MlpWeights.from_numpy(**random_weights(rng)))
    x = rng.normal(0, 1, (5000, 24)).astype(np.float32)
    assert np.array_equal(ctx.mlp_infer(x), ctx.mlp_infer(x))
