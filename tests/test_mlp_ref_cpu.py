"""The numpy MLP reference (oracle) against central finite differences."""
import numpy as np

from oracle import mlp_ref as M


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(11)
    p = rng.normal(0.0, 0.3, M.NPARAM)
    x = rng.uniform(-1, 1, 17)
    t = rng.uniform(-1, 1, (17, 4))
    loss, g = M.loss_and_grad(p, x, t)
    idx = rng.choice(M.NPARAM, 60, replace=False)
    idx = np.concatenate([idx, [M.OFF["W1"], M.OFF["b1"], M.OFF["b4"] + 3, M.OFF["W4"] + 5]])
    for i in idx:
        e = np.zeros(M.NPARAM)
        e[i] = 1e-6
        fd = (M.loss_and_grad(p + e, x, t)[0] - M.loss_and_grad(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(g[i]), (i, fd, g[i])
    y, _ = M.forward(p, x)
    assert abs(loss - np.mean((y - t) ** 2)) < 1e-15
