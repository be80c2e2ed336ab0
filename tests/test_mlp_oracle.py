"""The CPU oracle of the cost model, pinned by finite differences."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_ref  # noqa: E402


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.3, mlp_ref.N_WEIGHTS)
    x = rng.random((37, mlp_ref.F))
    y = rng.normal(0, 1, (37, mlp_ref.O))
    m = (rng.random((37, mlp_ref.O)) < 0.7).astype(float)
    loss, g = mlp_ref.loss_grad(w, x, y, m)
    idx = rng.choice(mlp_ref.N_WEIGHTS, 60, replace=False)
    eps = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        num = (mlp_ref.loss_grad(wp, x, y, m)[0] - mlp_ref.loss_grad(wm, x, y, m)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])
    assert np.isclose(loss, 0.5 * (m * (mlp_ref.forward(w, x) - y) ** 2).sum() / m.sum())


def test_pack_roundtrip():
    w = np.arange(mlp_ref.N_WEIGHTS, dtype=float)
    assert np.array_equal(mlp_ref.pack(mlp_ref.unpack(w)), w)
    assert mlp_ref.N_WEIGHTS == 16 * 64 + 64 + 64 * 64 + 64 + 64 * 3 + 3
