"""CPU restatement (numpy, FP64) of the far-field surrogate's network, for the
tests only: the same parameter layout, features, forward pass, weighted
squared loss and gradient as the CUDA training kernels.  The network has no
counterpart in the reference; this file is its oracle.

Layout: for each layer l (7->64, 64->64 x3, 64->1): W_l (out x in, row-major)
then b_l; tanh on the hidden layers, linear output.
Loss: sum_s w_s (y_s - t_s)^2 / sum_s w_s.
"""
import numpy as np

SIZES = [7, 64, 64, 64, 64, 1]


def param_count():
    return sum(o * i + o for i, o in zip(SIZES[:-1], SIZES[1:]))


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, k = [], 0
    for i, o in zip(SIZES[:-1], SIZES[1:]):
        W = p[k:k + o * i].reshape(o, i)
        k += o * i
        b = p[k:k + o]
        k += o
        out.append((W, b))
    return out


def features(d):
    """d: n x 3 sorted |displacements| (grid units) -> n x 7 features"""
    d = np.asarray(d, dtype=np.float64)
    r = np.sqrt((d ** 2).sum(1))
    safe = np.where(r > 0, r, 1.0)
    return np.concatenate([d / 16.0, (r / 16.0)[:, None], np.where(r[:, None] > 0, d / safe[:, None], 0.0)], 1)


def forward(p, X):
    hs = [np.asarray(X, dtype=np.float64)]
    layers = unpack(p)
    for l, (W, b) in enumerate(layers):
        z = hs[-1] @ W.T + b
        hs.append(np.tanh(z) if l < len(layers) - 1 else z)
    return hs


def loss_grad(p, X, T, W):
    """weighted mean squared loss and its gradient (flat, same layout)"""
    hs = forward(p, X)
    y = hs[-1][:, 0]
    T = np.asarray(T, dtype=np.float64)
    W = np.asarray(W, dtype=np.float64)
    ws = W.sum()
    loss = float((W * (y - T) ** 2).sum() / ws)
    g = (2.0 * W * (y - T) / ws)[:, None]
    layers = unpack(p)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        Wl, _ = layers[l]
        grads[l] = (g.T @ hs[l], g.sum(0))
        if l > 0:
            g = (g @ Wl) * (1.0 - hs[l] ** 2)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
