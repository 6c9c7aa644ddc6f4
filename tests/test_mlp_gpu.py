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
from oracle import mlp_oracle

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


@pytest.mark.parametrize("n", [1, 300, 40000])
def test_training_gradients_match_the_oracle(ctx, n):
    """Loss and gradients from the tensor-core training kernel (BF16 operands, FP32 accumulation
    in TMEM; 40000 rows = 313 tiles, so CTAs accumulate several tiles) against the oracle's float64
    restatement with the device's bf16 roundings (bar: 2e-3 of each field's largest gradient
    worst case, 2e-4 on average), and against the unrounded float64 gradients (5e-2)."""
    rng = np.random.default_rng(11 + n)
    W = random_weights(rng)
    ctx.set_mlp(A.MlpWeights.from_numpy(**W))
    x = rng.normal(0, 1, (n, 24)).astype(np.float32)
    t = (rng.normal(0, 1, (n, 3)) * W["out_scale"]).astype(np.float32)
    loss, g = ctx.mlp_loss_gradients(x, t)
    ref_loss, ref = mlp_oracle.loss_and_gradients(W, x, t)
    exact_loss, exact = mlp_oracle.loss_and_gradients(W, x, t, round_bf16=False)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    assert abs(loss - exact_loss) <= 2e-2 * exact_loss, (loss, exact_loss)
    for k, v in ref.items():
        scale = np.abs(v).max()
        d = np.abs(np.asarray(g[k], np.float64) - v)
        assert d.max() <= 2e-3 * scale, (k, d.max() / scale)
        assert d.mean() <= 2e-4 * scale, (k, d.mean() / scale)
        assert np.abs(np.asarray(g[k], np.float64) - exact[k]).max() <= 5e-2 * np.abs(exact[k]).max(), k


def test_training_gradients_are_deterministic(ctx):
    rng = np.random.default_rng(5)
    ctx.set_mlp(A.MlpWeights.from_numpy(**random_weights(rng)))
    x = rng.normal(0, 1, (20000, 24)).astype(np.float32)
    t = rng.normal(0, 1e-3, (20000, 3)).astype(np.float32)
    l1, g1 = ctx.mlp_loss_gradients(x, t)
    l2, g2 = ctx.mlp_loss_gradients(x, t)
    assert l1 == l2
    for k in g1:
        assert np.array_equal(g1[k], g2[k]), k


def test_training_fits_a_smooth_map(ctx):
    """Targets from a fixed random network of the same shape: training recovers most of it."""
    rng = np.random.default_rng(12)
    teacher = random_weights(rng)
    x = rng.normal(0, 1, (40000, 24)).astype(np.float32)
    t = reference(teacher, x, round_bf16=False).astype(np.float32)
    loss = ctx.mlp_train(x[:32768], t[:32768], epochs=30, batch=4096, learning_rate=3e-3, seed=1)
    assert loss < 0.05, loss  # normalised units: the targets have unit spread
    pred = ctx.mlp_infer(x[32768:])
    err = np.sqrt(((pred - t[32768:]) ** 2).mean(0)) / t[32768:].std(0)
    assert np.all(err < 0.5), err  # held out, and through the bf16 tensor-core inference
