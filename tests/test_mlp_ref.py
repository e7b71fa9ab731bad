"""The NumPy network reference (the checker of the tensor-core kernels)
against finite differences of its own float64 forward pass."""
import numpy as np

import mlp_ref as R


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = R.init(seed=5).astype(np.float64)
    x = rng.uniform(-1, 1, (16, R.IN))
    t = rng.normal(0, 1, (16, R.OUT))
    w = rng.uniform(0.5, 1.5, R.OUT)
    g, _ = R.gradient(p, x, t, w, emulate=False)

    def loss(q):
        y, _, _ = R.forward(q, x, emulate=False)
        return float((w * (y - t) ** 2).sum() / x.shape[0])

    idx = np.concatenate([rng.integers(0, R.NP, 40), [0, R.H * R.IN, R.NP - 1, R.NP - R.OUT - 5]])
    for i in idx:
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], np.float32)
    r = R.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-7 and r[4] == 0.0
