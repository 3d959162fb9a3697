"""NumPy restatement of the cost model's network (TEST INFRASTRUCTURE ONLY).

The same FP32 MLP as pdf-raster_b200/csrc/rrb_mlp.cu — 24 -> 64 -> 64 -> 1 with
ReLU, parameters W1[64][24], b1, W2[64][64], b2, W3[64], b3 — computed in
float64 to check the device forward pass and the device gradients.
"""

import numpy as np

IN, H = 24, 64


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    W1 = w[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    W3 = w[o:o + H]; o += H
    b3 = w[o]
    return W1, b1, W2, b2, W3, b3


def forward(w, X):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def loss_grad(w, X, y):
    """Mean squared error and its gradient w.r.t. the packed parameters."""
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    yhat, (z1, h1, z2, h2) = forward(w, X)
    n = len(y)
    err = yhat - y
    dout = 2 * err / n
    gW3 = h2.T @ dout
    gb3 = dout.sum()
    d2 = np.outer(dout, W3) * (z2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (z1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return float(np.mean(err ** 2)), g
