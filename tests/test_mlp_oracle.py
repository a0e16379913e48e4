"""The CPU restatement of the con2prim-guess network (oracle/mlp.py): its
analytic gradient against central finite differences of its own loss, and
the BF16 rounding helper."""
import numpy as np

from oracle import mlp


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and abs(r[2] - 1.0078125) < 1e-12
    assert abs(r[3] + 3.140625) < 1e-12


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    w = rng.normal(size=mlp.NPARAM + 12) * 0.3
    w[mlp.NPARAM:mlp.NPARAM + 6] = 0.0
    w[mlp.NPARAM + 6:] = 1.0
    x = rng.normal(size=(40, 6))
    t = rng.normal(size=(40, 2))
    # differentiate with the rounding switched off (the derivative of the
    # rounded weights is the derivative at their rounded values)
    orig = mlp.bf16
    mlp.bf16 = lambda v: np.asarray(v, np.float64)
    try:
        L, g = mlp.loss_and_grad(w, x, t)
        for k in rng.choice(mlp.NPARAM, 40, replace=False):
            h = 1e-6
            wp, wm = w.copy(), w.copy()
            wp[k] += h; wm[k] -= h
            lp = ((mlp.forward(wp, x)[3] - t) ** 2).sum() / len(x)
            lm = ((mlp.forward(wm, x)[3] - t) ** 2).sum() / len(x)
            assert abs((lp - lm) / (2 * h) - g[k]) <= 1e-6 * max(1.0, abs(g[k]))
    finally:
        mlp.bf16 = orig
