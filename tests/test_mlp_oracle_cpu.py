"""The network oracle's gradients (oracle/mlp_oracle.py, unrounded float64) against central finite
differences of its own loss: the restatement the tensor-core training kernel is checked against
is itself the gradient of the loss it states."""
import numpy as np

from oracle import mlp_oracle


def weights(rng):
    W = {"w1": rng.normal(0, 1 / np.sqrt(24), (64, 24)), "b1": rng.normal(0, 0.1, 64),
         "w2": rng.normal(0, 1 / np.sqrt(64), (64, 64)), "b2": rng.normal(0, 0.1, 64),
         "w3": rng.normal(0, 1 / np.sqrt(64), (3, 64)), "b3": rng.normal(0, 0.1, 3),
         "in_mean": rng.normal(0, 0.5, 24), "in_scale": rng.uniform(0.5, 2.0, 24),
         "out_scale": np.array([1e-3, 2e-3, 5e-4])}
    return {k: np.asarray(v, np.float64) for k, v in W.items()}


def test_oracle_gradients_are_the_loss_gradient():
    rng = np.random.default_rng(3)
    W = weights(rng)
    x = rng.normal(0, 1, (40, 24))
    t = rng.normal(0, 1, (40, 3)) * W["out_scale"]
    # the float32 casts inside the restatement would swamp a finite difference: work in float64
    # through a copy of the loss that keeps everything in float64
    def loss(Wd):
        f = Wd
        xn = (x - f["in_mean"]) * f["in_scale"]
        h1 = mlp_oracle.silu(xn @ f["w1"].T + f["b1"])
        h2 = mlp_oracle.silu(h1 @ f["w2"].T + f["b2"])
        e = h2 @ f["w3"].T + f["b3"] - t / f["out_scale"]
        return (e * e).sum() / (3 * len(x))

    _, g = mlp_oracle.loss_and_gradients(W, x, t, round_bf16=False)
    for k in ("w1", "b1", "w2", "b2", "w3", "b3"):
        flat = W[k].reshape(-1)
        for i in rng.choice(flat.size, size=min(flat.size, 12), replace=False):
            h = 1e-6
            Wp = {kk: v.copy() for kk, v in W.items()}
            Wm = {kk: v.copy() for kk, v in W.items()}
            Wp[k].reshape(-1)[i] += h
            Wm[k].reshape(-1)[i] -= h
            num = (loss(Wp) - loss(Wm)) / (2 * h)
            ana = g[k].reshape(-1)[i]
            assert abs(num - ana) <= 1e-6 * max(1.0, abs(ana)) + 1e-7, (k, i, num, ana)


def test_oracle_rounding_points():
    """bf16 rounding is nearest-even and the rounded loss stays near the unrounded one."""
    assert mlp_oracle.bf16(np.float32(1.0 + 2.0 ** -8))[()] == 1.0          # tie to even
    assert mlp_oracle.bf16(np.float32(1.0 + 3 * 2.0 ** -8))[()] == 1.0 + 2.0 ** -6
    rng = np.random.default_rng(4)
    W = {k: np.asarray(v, np.float32) for k, v in weights(rng).items()}
    x = rng.normal(0, 1, (500, 24)).astype(np.float32)
    t = (rng.normal(0, 1, (500, 3)) * W["out_scale"]).astype(np.float32)
    l_q, _ = mlp_oracle.loss_and_gradients(W, x, t)
    l_e, _ = mlp_oracle.loss_and_gradients(W, x, t, round_bf16=False)
    assert abs(l_q - l_e) <= 2e-2 * l_e
