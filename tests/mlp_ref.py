"""float64 NumPy reference of the capacity predictor's MLP (test
infrastructure): the flat parameter layout of the CUDA kernels, forward,
masked-MSE loss and its analytic gradient."""

import numpy as np

N_IN, N_HID, N_OUT = 12, 64, 2


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((N_IN, N_HID), (N_HID,), (N_HID, N_HID), (N_HID,), (N_HID, N_OUT), (N_OUT,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == p.size
    return out


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    H1 = np.maximum(X @ W1 + b1, 0.0)
    H2 = np.maximum(H1 @ W2 + b2, 0.0)
    return H2 @ W3 + b3, (H1, H2)


def loss_and_grad(p, X, Y, M):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    O, (H1, H2) = forward(p, X)
    B = X.shape[0]
    D = (O - Y) * M
    loss = float((D * D).sum() / B)
    dO = 2.0 * D / B
    gW3 = H2.T @ dO
    gb3 = dO.sum(0)
    dH2 = (dO @ W3.T) * (H2 > 0)
    gW2 = H1.T @ dH2
    gb2 = dH2.sum(0)
    dH1 = (dH2 @ W2.T) * (H1 > 0)
    gW1 = X.T @ dH1
    gb1 = dH1.sum(0)
    return loss, np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])
