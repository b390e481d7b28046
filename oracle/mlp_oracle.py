"""FP64 numpy restatement of the step-size controller network.

TEST INFRASTRUCTURE ONLY: checks the CUDA forward/backward kernels
(dsgdpp_b200/csrc/kernels_mlp.cu).  Parameter layout: W1[64][16], b1[64],
W2[64][64], b2[64], W3[64], b3; GELU(x) = x Phi(x); output clipped to [-1, 1] when used;
training loss = mean over the batch of (raw output - y)^2 (unclipped).
"""
import math

import numpy as np

IN, HID = 16, 64


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + HID * IN].reshape(HID, IN); o += HID * IN
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + HID]; o += HID
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    z1 = X @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    raw = h2 @ W3 + b3
    return np.clip(raw, -1, 1), (X, z1, h1, z2, h2, raw)


def loss_and_grad(p, X, y):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    out, (X, z1, h1, z2, h2, raw) = forward(p, X)
    y = np.asarray(y, np.float64)
    B = len(y)
    loss = float(np.sum((raw - y) ** 2) / B)
    dout = 2 * (raw - y) / B
    gW3 = h2.T @ dout
    gb3 = dout.sum()
    dz2 = (dout[:, None] * W3[None, :]) * gelu_grad(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    gW1 = dz1.T @ X
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
