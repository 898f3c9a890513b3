"""The FP64 reference MLP's analytic backward against finite differences."""
import numpy as np

import mlp_ref


def test_reference_backward_matches_finite_differences():
    rng = np.random.default_rng(4)
    p = rng.normal(0, 0.3, mlp_ref.NP)
    p[:mlp_ref.W1].reshape(64, 16)[:, 12:] = 0.0
    xs = rng.normal(0, 1, (40, 12))
    ys = rng.normal(0, 1, (40, 2))
    g, _ = mlp_ref.gradients(p, xs, ys, quantize=False)
    idx = np.concatenate([rng.choice(mlp_ref.W1, 20), mlp_ref.W1 + rng.choice(mlp_ref.W2, 20),
                          mlp_ref.W1 + mlp_ref.W2 + rng.choice(mlp_ref.W3, 10),
                          mlp_ref.NW + np.arange(0, 130, 7)])
    for i in idx:
        if i < mlp_ref.W1 and (i % 16) >= 12:
            continue
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (mlp_ref.loss(p + e, xs, ys) - mlp_ref.loss(p - e, xs, ys)) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, 3.0e-3, -7.5], dtype=np.float32)
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] - 3.0e-3) / 3.0e-3 < 2 ** -8 and r[4] == -7.5
