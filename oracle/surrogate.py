"""CPU restatement of the surrogate MLP (test infrastructure only).

D → 256 → 256 → 1 with GELU (erf form), loss (1/B) Σ (y − t)².  The device
kernels round the GEMM operands to BF16 (X, W1, W2, H1, dZ2, dZ1) and keep
everything else in FP32; `bf16=True` reproduces those rounding points with
FP64 arithmetic elsewhere, `bf16=False` is the exact FP64 model (pinned
against central differences by the tests).  Parameter order: W1 [256 × D],
b1 [256], W2 [256 × 256], b2 [256], w3 [256], b3 [1].

The network is this project's own addition (the reference evaluates every
DE trial exactly), so there is no reference file to cite; the layer and
optimiser definitions are the textbook ones (GELU: Hendrycks & Gimpel 2016;
Adam: Kingma & Ba 2015).
"""
import numpy as np
from scipy.special import erf

H = 256


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p, D):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * D].reshape(H, D); o += H * D
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def pack(W1, b1, W2, b2, w3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, w3, [b3]])


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(p, X, bf=True):
    D = X.shape[1]
    W1, b1, W2, b2, w3, b3 = unpack(p, D)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    z1 = r(X) @ r(W1).T + b1
    h1 = gelu(z1)
    z2 = r(h1) @ r(W2).T + b2
    h2 = gelu(z2)
    y = h2 @ w3 + b3
    return y, (z1, h1, z2, h2)


def loss_and_grad(p, X, t, bf=True):
    X = np.asarray(X, np.float64)
    t = np.asarray(t, np.float64)
    B, D = X.shape
    W1, b1, W2, b2, w3, b3 = unpack(p, D)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    y, (z1, h1, z2, h2) = forward(p, X, bf)
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / B
    dz2 = (dy[:, None] * w3[None, :]) * gelu_d(z2)
    dW2 = r(dz2).T @ r(h1)
    dh1 = r(dz2) @ r(W2)
    dz1 = dh1 * gelu_d(z1)
    dW1 = r(dz1).T @ r(X)
    g = pack(dW1, dz1.sum(0), dW2, dz2.sum(0), h2.T @ dy, dy.sum())
    return loss, g, y


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    return p - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
