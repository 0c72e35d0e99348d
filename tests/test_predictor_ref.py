"""The NumPy reference MLP used to check the predictor's CUDA training
kernels: its analytic gradient against central finite differences."""

import numpy as np

from mlp_ref import N_HID, N_IN, N_OUT, loss_and_grad


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n_params = N_IN * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * N_OUT + N_OUT
    p = rng.normal(0, 0.3, n_params)
    X = rng.normal(0, 1, (64, N_IN))
    Y = rng.normal(0, 1, (64, N_OUT))
    M = (rng.uniform(size=(64, N_OUT)) > 0.3).astype(np.float64)
    _, g = loss_and_grad(p, X, Y, M)
    h = 1e-6
    for i in rng.choice(n_params, 40, replace=False):
        e = np.zeros(n_params)
        e[i] = h
        num = (loss_and_grad(p + e, X, Y, M)[0] - loss_and_grad(p - e, X, Y, M)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(num), (i, num, g[i])
