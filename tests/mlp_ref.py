"""CPU reference of the cost model's network (numpy, float64): the checker
for the CUDA forward / backward kernels (lela_cuda_mlp_*).  Same parameter
layout: W1[F][64], b1[64], W2[64][64], b2[64], W3[64], b3."""
import numpy as np

H = 64


def unpack(params, F):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    W1 = p[o:o + F * H].reshape(F, H); o += F * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def forward(params, F, X):
    W1, b1, W2, b2, W3, b3 = unpack(params, F)
    h1 = np.maximum(X @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ W3 + b3


def loss_and_grad(params, F, X, t):
    """Mean squared error and its gradient w.r.t. the flat parameters."""
    X = np.asarray(X, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    n = X.shape[0]
    W1, b1, W2, b2, W3, b3 = unpack(params, F)
    z1 = X @ W1 + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ W3 + b3
    err = y - t
    loss = float(np.mean(err ** 2))
    dy = 2.0 * err / n
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = np.outer(dy, W3) * (z2 > 0)
    gW2 = h1.T @ dz2
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2.T) * (z1 > 0)
    gW1 = X.T @ dz1
    gb1 = dz1.sum(axis=0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, grad
