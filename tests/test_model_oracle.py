"""The CPU restatement of the result-count model (oracle/model_oracle.py):
its analytic gradient against central finite differences (float64)."""
import numpy as np

from oracle import model_oracle as MO


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = rng.standard_normal(MO.NW) * 0.2
    X = rng.uniform(0, 1, size=(40, MO.F))
    y = rng.uniform(0, 4, size=40)
    loss, g = MO.loss_grad(w, X, y)
    assert abs(loss - np.mean((MO.forward(w, X) - y) ** 2)) < 1e-12
    idx = rng.choice(MO.NW, 60, replace=False)
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (MO.loss_grad(wp, X, y)[0] - MO.loss_grad(wm, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd)
