"""NumPy oracle of the QP-shift network -- TEST INFRASTRUCTURE.

The 4 -> H -> H -> 1 SiLU perceptron with the parameter packing of
libmbpt_b200 ([W1 (H x 4), b1, W2 (H x H), b2, W3 (H), b3]), its loss
0.5/B sum (y - t)^2, the gradient by reverse mode, and one AdamW step.
The network has no counterpart in MBPTcode; this is the checker of the
device kernels' forward, backward and optimiser arithmetic.
"""
import numpy as np


def unpack(p, H):
    o = 0
    W1 = p[o:o + 4 * H].reshape(H, 4); o += 4 * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, H, x):
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, np.float64), H)
    z1 = x @ W1.T + b1
    h1 = silu(z1)
    z2 = h1 @ W2.T + b2
    h2 = silu(z2)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def loss_and_grad(p, H, x, t):
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, np.float64), H)
    y, (z1, h1, z2, h2) = forward(p, H, x)
    B = x.shape[0]
    loss = 0.5 * np.sum((y - t) ** 2) / B
    dy = (y - t) / B
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = np.outer(dy, W3) * dsilu(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * dsilu(z1)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g


def adamw(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=1e-5):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * (mh / (np.sqrt(vh) + eps) + wd * p), m, v
