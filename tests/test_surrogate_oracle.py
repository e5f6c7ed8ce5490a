"""Pins of the CPU surrogate oracle (oracle/surrogate.py): its FP64 gradient
against central differences, and its BF16 rounding against torch's."""
import numpy as np
import torch

from oracle import surrogate as S


def _params(D, seed):
    rng = np.random.default_rng(seed)
    n = S.H * D + S.H * S.H + 3 * S.H + 1
    p = rng.uniform(-0.1, 0.1, n)
    return p


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(0, 3, 5000), rng.uniform(-1e-3, 1e-3, 1000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.005859375, 3.0e38]]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(S.bf16(x), want)


def test_fp64_gradient_matches_central_differences():
    D, B = 6, 16
    rng = np.random.default_rng(5)
    p = _params(D, 1)
    X = rng.uniform(-1, 1, (B, D))
    t = rng.normal(0, 1, B)
    _, g, _ = S.loss_and_grad(p, X, t, bf=False)
    idx = np.concatenate([rng.choice(S.H * D, 20, replace=False),          # W1
                          S.H * D + rng.choice(S.H, 5, replace=False),      # b1
                          S.H * D + S.H + rng.choice(S.H * S.H, 20, replace=False),
                          p.size - 1 - rng.choice(2 * S.H + 1, 10, replace=False)])
    for k in idx:
        e = np.zeros_like(p)
        e[k] = 1e-6
        fp = S.loss_and_grad(p + e, X, t, bf=False)[0]
        fm = S.loss_and_grad(p - e, X, t, bf=False)[0]
        fd = (fp - fm) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * (abs(g[k]) + 1e-3), (k, fd, g[k])


def test_adam_step_reference_values():
    # one step from zero moments moves every weight by lr·sign(g) (|g| ≫ eps)
    p = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, -1e-3])
    p1, m, v = S.adam(p, g, np.zeros(4), np.zeros(4), 1)
    np.testing.assert_allclose(p1, -1e-3 * np.sign(g), rtol=1e-4)
