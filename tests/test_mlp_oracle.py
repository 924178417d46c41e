"""The NumPy oracle of the rank predictor's training step, checked on the CPU: its
backward pass against central finite differences of its own FP64 forward pass, and
its BF16 rounding against the definition (round to nearest even)."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.standard_normal(mlp.NPARAM) * 0.2
    X = rng.standard_normal((24, mlp.NIN))
    y = rng.random(24)
    loss, g = mlp.loss_and_grad(w, X, y, bf16_round=False)
    idx = rng.choice(mlp.NPARAM, 60, replace=False)
    idx = np.concatenate([idx, [mlp.NPARAM - 1, 0, mlp.NH * mlp.NIN]])
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mlp.loss_and_grad(wp, X, y, False)[0] - mlp.loss_and_grad(wm, X, y, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30], dtype=np.float32)
    r = mlp.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0            # tie to even
    assert r[2] == np.float32(1.0 + 2 ** -7)      # above the tie rounds up
    assert abs(r[3] + 3.140625) < 1e-6
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)
