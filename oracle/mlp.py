"""FP64 numpy restatement of the cost-model MLP (12 -> 128 -> 128 -> 128 -> 1,
ReLU, MSE) -- TEST INFRASTRUCTURE ONLY: the oracle for the GPU forward /
backward kernels' gradients. Parameter layout matches bbx_mlp_loss_grad:
W1 (12 x 128), b1, W2 (128 x 128), b2, W3 (128 x 128), b3, W4 (128 x 1), b4.
"""
import numpy as np

IN, H = 12, 128
SHAPES = [(IN, H), (H,), (H, H), (H,), (H, H), (H,), (H, 1), (1,)]


def unpack(p):
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(p[o:o + n], np.float64).reshape(s))
        o += n
    return out


def pack(arrs):
    return np.concatenate([a.ravel() for a in arrs])


def loss_grad(p, x, y, mean=None, std=None):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    x = np.asarray(x, np.float64)
    if mean is not None:
        x = (x - mean) / std
    y = np.asarray(y, np.float64)
    n = len(y)
    z1 = x @ W1 + b1; h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2; h2 = np.maximum(z2, 0)
    z3 = h2 @ W3 + b3; h3 = np.maximum(z3, 0)
    out = (h3 @ W4 + b4)[:, 0]
    d = out - y
    loss = np.mean(d * d)
    dout = (2.0 * d / n)[:, None]
    gW4 = h3.T @ dout; gb4 = dout.sum(0)
    d3 = (dout @ W4.T) * (h3 > 0)
    gW3 = h2.T @ d3; gb3 = d3.sum(0)
    d2 = (d3 @ W3.T) * (h2 > 0)
    gW2 = h1.T @ d2; gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    gW1 = x.T @ d1; gb1 = d1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4])


def predict(p, x, mean=None, std=None):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    x = np.asarray(x, np.float64)
    if mean is not None:
        x = (x - mean) / std
    h = np.maximum(x @ W1 + b1, 0)
    h = np.maximum(h @ W2 + b2, 0)
    h = np.maximum(h @ W3 + b3, 0)
    return (h @ W4 + b4)[:, 0]
