"""The learned kernel selector: the CUDA network's gradients against the CPU
reference network, training on the GPU, and what the trained model gains
over the method without it, with its regret against exhaustive tuning."""
import numpy as np
import pytest

import mlp_ref
from lela_b200 import selector as sel


def test_cpu_reference_gradient_is_consistent():
    """The CPU reference network's analytic gradient agrees with central
    finite differences (it is the checker of the CUDA kernels)."""
    g = np.random.default_rng(0)
    F = sel.NFEAT
    P = g.normal(0, 0.2, size=F * 64 + 64 + 64 * 64 + 64 + 64 + 1)
    X = g.random((12, F))
    t = g.normal(size=12)
    _, grad = mlp_ref.loss_and_grad(P, F, X, t)
    for idx in g.choice(len(P), size=40, replace=False):
        e = np.zeros_like(P); e[idx] = 1e-6
        fd = (mlp_ref.loss_and_grad(P + e, F, X, t)[0] - mlp_ref.loss_and_grad(P - e, F, X, t)[0]) / 2e-6
        assert abs(fd - grad[idx]) <= 1e-5 + 1e-4 * abs(fd)


@pytest.mark.gpu
def test_mlp_forward_and_gradient_match_cpu(cuda):
    g = np.random.default_rng(1)
    model = sel.CostModel(cuda, seed=3)
    X = g.random((300, sel.NFEAT)).astype(np.float32)
    t = g.normal(size=300).astype(np.float32)
    params = model.params.cpu().numpy().astype(np.float64)
    pred = model.predict(X)  # mu = 0, sd = 1 before training
    want = mlp_ref.forward(params, sel.NFEAT, X.astype(np.float64))
    assert np.allclose(pred, want, rtol=1e-4, atol=1e-4)
    loss, grad = model.gradient(X, t)
    wl, wg = mlp_ref.loss_and_grad(params, sel.NFEAT, X.astype(np.float64), t.astype(np.float64))
    assert abs(loss - wl) <= 1e-4 * max(1.0, wl)
    # float32 atomics on the GPU vs float64 sums: tolerance relative to the
    # gradient's scale
    scale = np.abs(wg).max()
    assert np.allclose(grad, wg, rtol=1e-3, atol=1e-4 * scale)


@pytest.mark.gpu
def test_mlp_training_reduces_loss(cuda):
    g = np.random.default_rng(2)
    X = g.random((400, sel.NFEAT)).astype(np.float32)
    y = np.sin(3 * X[:, 0]) + X[:, 1] ** 2 - X[:, 2] * X[:, 3]
    model = sel.CostModel(cuda, seed=4)
    curve = model.fit(X, y, epochs=600, lr=3e-3)
    assert curve[-1] < 0.1 * curve[0]


@pytest.mark.gpu
def test_selector_gain_and_regret(cuda):
    """Autotune a family of blocks (every candidate kernel and tile variant
    timed), train the cost model on two thirds of them, and evaluate on the
    held-out third: the model's picks must beat the fixed default choices
    and stay within 15 % of exhaustive tuning (total time of the held-out
    blocks)."""
    tuner = sel.Autotuner(cuda, reps=3)
    rng = np.random.default_rng(5)
    for i in range(48):
        m, n = int(2 ** rng.uniform(6, 12)), int(2 ** rng.uniform(6, 12))
        k = int(2 ** rng.uniform(4, 12)) if i % 2 else int(2 ** rng.uniform(4, 8))
        tuner.tune_gemm(m, n, k, int(rng.choice([251, 65521, 2147483647])), seed=i)
    for i in range(20):
        tuner.tune_gf2_gemm(int(2 ** rng.uniform(6, 12)), int(2 ** rng.uniform(6, 12)),
                            int(2 ** rng.uniform(6, 12)), seed=i)
    for i in range(24):
        s_ = int(2 ** rng.uniform(5, 10))
        tuner.tune_echelon(s_, s_, int(rng.choice([251, 65521, 2147483647])), seed=i)
    blocks = sel.group_blocks(tuner.records)
    keys = sorted(blocks)
    rng.shuffle(keys)
    held = set(keys[::3])
    train = [r for r in tuner.records
             if (r["op"], r["m"], r["n"], r["k"], r["density"], r["pbits"], r["pivots"]) not in held]
    test_blocks = {k: blocks[k] for k in held}
    X, y = sel.records_to_xy(train)
    model = sel.CostModel(cuda, seed=6)
    model.fit(X, y, epochs=1500, lr=3e-3)
    res = sel.evaluate(sel.Selector(model), test_blocks)
    print(res)
    assert res["gain_vs_default"] > 1.0
    assert res["regret"] <= 0.15
