"""CPU oracle of the per-node predictor MLP -- TEST INFRASTRUCTURE.

numpy restatement of the 12 -> 128 -> 128 -> 3 GELU network and its backward
pass for checking the tensor-core kernels.  With ``bf16=True`` every tensor-core
operand (inputs, weights, H1, H2, dY, dZ2, dZ1) is rounded to bfloat16 (round to
nearest even) exactly where the kernels round them, and sums are taken in
float64; with ``bf16=False`` the network is evaluated in float64 throughout (used
to pin the backward pass against finite differences).

Parameter layout (flat float32, 20752 values): W1 [128][16], b1 [128],
W2 [128][128], b2 [128], W3 [16][128], b3 [16].
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

H, INP, OUTP, NF = 128, 16, 16, 12
NPARAMS = H * INP + H + H * H + H + OUTP * H + OUTP


def split(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * INP].reshape(H, INP); o += H * INP
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + OUTP * H].reshape(OUTP, H); o += OUTP * H
    b3 = p[o:o + OUTP]
    return W1, b1, W2, b2, W3, b3


def join(W1, b1, W2, b2, W3, b3):
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, W3.ravel(), b3])


def bf16(x):
    x = np.ascontiguousarray(np.asarray(x, np.float32))
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b >> 16) & 1) + 0x7FFF
    return ((b + r) & 0xFFFF0000).astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(p, F, bf=True):
    """F: (n, 12) features. Returns Y (n, 3) and the cache for backward."""
    W1, b1, W2, b2, W3, b3 = split(p)
    q = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    X = np.zeros((F.shape[0], INP)); X[:, :NF] = F
    Xb, W1b, W2b, W3b = q(X), q(W1), q(W2), q(W3)
    Z1 = Xb @ W1b.T + b1
    H1b = q(gelu(Z1))
    Z2 = H1b @ W2b.T + b2
    H2b = q(gelu(Z2))
    Y = H2b @ W3b.T + b3
    return Y[:, :3], (Xb, W1b, W2b, W3b, Z1, H1b, Z2, H2b, Y)


def loss_grad(p, F, T, bf=True):
    """Mean squared error over the 3 outputs and its gradient (flat, NPARAMS)."""
    q = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    Yo, (Xb, W1b, W2b, W3b, Z1, H1b, Z2, H2b, Y) = forward(p, F, bf)
    n = F.shape[0]
    E = Yo - T
    loss = float(np.sum(E * E) / (3 * n))
    dY = np.zeros((n, OUTP)); dY[:, :3] = 2.0 * E / (3 * n)
    if bf:  # the kernel's dY is float32 before the bf16 operand rounding
        dY = np.asarray(dY, np.float32).astype(np.float64)
    dYb = q(dY)
    dZ2 = (dYb @ W3b) * gelu_d(Z2)
    dZ2b = q(dZ2)
    dZ1 = (dZ2b @ W2b) * gelu_d(Z1)
    dZ1b = q(dZ1)
    gW3 = dYb.T @ H2b
    gW2 = dZ2b.T @ H1b
    gW1 = dZ1b.T @ Xb
    g = join(gW1, dZ1.sum(0), gW2, dZ2.sum(0), gW3, dY.sum(0))
    return loss, g
