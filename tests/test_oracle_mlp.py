"""The FP64 MLP oracle against central finite differences, and AdamW against its closed form."""

import numpy as np

from oracle import mlp as om


def _small(seed=0, b=6, n_in=10, h=8, n_out=3):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(b, n_in))
    params = [rng.normal(0, 0.5, (h, n_in)), rng.normal(0, 0.1, h), rng.normal(0, 0.5, (h, h)),
              rng.normal(0, 0.1, h), rng.normal(0, 0.5, (n_out, h)), rng.normal(0, 0.1, n_out)]
    t = rng.normal(size=(b, n_out))
    w = rng.uniform(0.5, 2.0, n_out)
    return x, params, t, w


def _loss(x, params, t, w):
    _, _, y = om.forward(x, *params)
    return om.loss_and_grad_output(y, t, w)[0]


def test_backward_matches_finite_differences():
    x, params, t, w = _small()
    h1, h2, y = om.forward(x, *params)
    _, dy = om.loss_and_grad_output(y, t, w)
    grads = om.backward(x, h1, h2, dy, params[2], params[4])
    eps = 1e-6
    for p, g in zip(params, grads):
        flat = p.reshape(-1)
        num = np.zeros_like(flat)
        for i in range(flat.size):
            old = flat[i]
            flat[i] = old + eps
            lp = _loss(x, params, t, w)
            flat[i] = old - eps
            lm = _loss(x, params, t, w)
            flat[i] = old
            num[i] = (lp - lm) / (2 * eps)
        np.testing.assert_allclose(g.reshape(-1), num, rtol=1e-5, atol=1e-8)


def test_adamw_first_step_and_bf16_rounding():
    w = np.array([1.0, -2.0, 0.5])
    g = np.array([0.1, -0.3, 0.0])
    w1, m, v = om.adamw(w, g, np.zeros(3), np.zeros(3), 1, lr=0.01, weight_decay=0.1)
    # First step: m_hat = g, v_hat = g^2, so the update is lr * (sign(g) + wd * w) where g != 0.
    np.testing.assert_allclose(w1, w - 0.01 * (g / (np.abs(g) + 1e-8) + 0.1 * w), rtol=1e-12)
    assert om.bf16(np.array([1.0 + 2 ** -9]))[0] == 1.0            # tie to even
    assert om.bf16(np.array([1.0 + 3 * 2 ** -9]))[0] == 1.0 + 2 ** -7
    assert om.bf16(np.array([-3.140625]))[0] == -3.140625
