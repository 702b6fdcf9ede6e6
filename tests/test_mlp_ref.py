"""The CPU restatement of the MLP (oracle/mlp_ref.py) is itself checked
against central finite differences (float64, no bf16 rounding).  CPU only."""
import numpy as np

from oracle import mlp_ref as R


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(R.NPARAM) * 0.2
    p[R.OFF_W1 + R.IN * R.H:R.OFF_B1] = 0.0
    x = rng.standard_normal((12, R.IN))
    t = rng.standard_normal(12)
    g, loss = R.grad(p, x, t, mirror_bf16=False)
    eps = 1e-6
    idx = list(rng.choice(R.IN * R.H, 20, replace=False)) + list(range(R.OFF_B1, R.OFF_B1 + 5)) + \
        list(R.OFF_W2 + rng.choice(R.H * R.H, 20, replace=False)) + list(range(R.OFF_B2, R.NPARAM, 7))
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        lp = 0.5 * np.mean((R.forward(pp, x, False)[0] - t) ** 2)
        lm = 0.5 * np.mean((R.forward(pm, x, False)[0] - t) ** 2)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -3.14159, 0.0], dtype=np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == 1.015625  # ties to even
    assert abs(r[4] + 3.140625) < 1e-9 and r[5] == 0.0
