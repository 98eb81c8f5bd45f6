"""The scheduler network's CPU oracle (oracle/mlp_oracle.py) pinned on its
own terms: analytic gradients against central finite differences, BF16
rounding against torch's conversion, Adam against torch.optim.Adam."""
import sys
from pathlib import Path

import numpy as np
import torch

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_gradients_match_finite_differences():
    shapes = mo.layer_shapes(6, 8, 2, 2)
    p = mo.init_params(6, 8, 2, 2, seed=3).astype(np.float64)
    rng = np.random.default_rng(4)
    x, y = rng.normal(size=(5, 6)), rng.normal(size=(5, 2))
    _, g = mo.loss_grad(p, shapes, x, y, exact=True)
    num = np.empty_like(p)
    eps = 1e-6
    for i in range(p.size):
        d = np.zeros_like(p)
        d[i] = eps
        lp, _ = mo.loss_grad(p + d, shapes, x, y, exact=True)
        lm, _ = mo.loss_grad(p - d, shapes, x, y, exact=True)
        num[i] = (lp - lm) / (2 * eps)
    assert np.abs(g - num).max() <= 1e-7 * max(1.0, np.abs(num).max())


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-30, 30, 4000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38]]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(mo.bf16(x), want)


def test_adam_matches_torch():
    rng = np.random.default_rng(6)
    w0 = rng.normal(size=50)
    grads = [rng.normal(size=50) for _ in range(3)]
    t = torch.tensor(w0, requires_grad=True)
    opt = torch.optim.Adam([t], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    w, m, v = w0.copy(), np.zeros(50), np.zeros(50)
    for k, g in enumerate(grads, start=1):
        t.grad = torch.tensor(g)
        opt.step()
        w, m, v = mo.adam(w, g, m, v, k, 1e-2)
    np.testing.assert_allclose(w, t.detach().numpy(), rtol=1e-12, atol=1e-14)
