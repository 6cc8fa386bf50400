"""FP32 CPU reference of the learned estimator's forward and backward passes
(test infrastructure: the checker of the device kernels, never a product path).

It follows the device computation step for step: inputs and weights rounded
to BF16, products accumulated in FP32, activations and their gradients
rounded to BF16 where the device stores them in BF16 (the ReLU outputs H1,
H2 and the gradients dH2, dH1), weight gradients kept in FP32. Parameter
layout as bj_estimator_get_params: W1 (F x 256), b1, W2 (256 x 256), b2,
w3 (256), b3, padding.
"""
import numpy as np

F, H = 1792, 256


def bf16(x):
    """Round FP32 to the nearest BF16 (ties to even), returned as FP32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def split(p):
    o = 0
    W1 = p[o:o + F * H].reshape(F, H); o += F * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o:o + 1]; o += 1
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = [bf16(a) for a in split(p)]
    Xb = bf16(X)
    H1 = bf16(np.maximum(Xb @ W1 + b1, 0))
    H2 = bf16(np.maximum(H1 @ W2 + b2, 0))
    y = H2 @ w3 + b3[0]
    return Xb, H1, H2, y


def loss_and_grads(p, X, t):
    W1, b1, W2, b2, w3, b3 = [bf16(a) for a in split(p)]
    Xb, H1, H2, y = forward(p, X)
    n = len(t)
    d = y - t
    loss = float(np.mean(d * d))
    dy = (2.0 * d / n).astype(np.float32)
    dH2 = bf16(dy[:, None] * w3[None, :] * (H2 > 0))
    g = np.zeros_like(p)
    o = 0
    dH1 = bf16((dH2 @ W2.T) * (H1 > 0))
    g[o:o + F * H] = (Xb.T @ dH1).ravel(); o += F * H
    g[o:o + H] = dH1.sum(0); o += H
    g[o:o + H * H] = (H1.T @ dH2).ravel(); o += H * H
    g[o:o + H] = dH2.sum(0); o += H
    g[o:o + H] = H2.T @ dy; o += H
    g[o] = dy.sum()
    return loss, g
