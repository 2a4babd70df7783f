"""TEST INFRASTRUCTURE ONLY: CPU oracle of the neural SDF surrogate.

Forward pass, L1-loss gradient and Adam step of the network the library
trains and evaluates (3 -> 128 Fourier features -> 4 x 64 softplus -> 1), in
float64 numpy.  `bf16=True` rounds weights, features and activations to
BF16 (round to nearest even) where the device does, so device results can be
compared with a tolerance; `bf16=False` is the plain real-valued network,
used for finite-difference checks of the backward pass.

The parameter layout and feature order follow include/rayengine_b200.h:
W1 [64][128], b1, W2, b2, W3, b3, W4, b4 ([64][64], 64), w5 [64], b5; features
index chain*48 + octave*6 + 2*axis + {sin, cos} with frequency f0 * 2^octave
(chain 0) or f0 * sqrt(2) * 2^octave (chain 1), then q.xyz, zeros to 128.
"""
from __future__ import annotations

import numpy as np

H, IN = 64, 128
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + H * H
OFF_W5 = OFF_B4 + H
OFF_B5 = OFF_W5 + H
NUM_PARAMS = OFF_B5 + 1

# degree-6 fit of log1p(u) on [0, 1] used by the device softplus
LP = np.array([0.0, 0.9998613, -0.49753284, 0.31643057, -0.19167475, 0.083866805,
               -0.017806457], np.float64)


def bf16(x):
    """Round float values to BF16 (nearest even), returned as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    rounded = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    W = [p[OFF_W1:OFF_B1].reshape(H, IN), p[OFF_W2:OFF_B2].reshape(H, H),
         p[OFF_W3:OFF_B3].reshape(H, H), p[OFF_W4:OFF_B4].reshape(H, H)]
    b = [p[OFF_B1:OFF_W2], p[OFF_B2:OFF_W3], p[OFF_B3:OFF_W4], p[OFF_B4:OFF_W5]]
    return W, b, p[OFF_W5:OFF_B5], p[OFF_B5]


def features(pts, box_min, box_max, f0):
    pts = np.asarray(pts, np.float64)
    lo, hi = np.asarray(box_min, np.float64), np.asarray(box_max, np.float64)
    q = (pts - 0.5 * (lo + hi)) * (2.0 / (hi - lo))
    n = pts.shape[0]
    X = np.zeros((n, IN))
    for chain in range(2):
        base = f0 * (np.sqrt(2.0) if chain else 1.0)
        for o in range(8):
            f = base * 2.0 ** o
            for j in range(3):
                X[:, chain * 48 + o * 6 + 2 * j] = np.sin(2 * np.pi * f * q[:, j])
                X[:, chain * 48 + o * 6 + 2 * j + 1] = np.cos(2 * np.pi * f * q[:, j])
    X[:, 96:99] = q
    return X


def softplus(x):
    u = np.exp(-np.abs(x))
    return np.maximum(x, 0.0) + np.polynomial.polynomial.polyval(u, LP)


def softplus_deriv(x):
    u = np.exp(-np.abs(x))
    g = u * np.polynomial.polynomial.polyval(u, np.polynomial.polynomial.polyder(LP))
    return np.where(x > 0, 1.0 - g, g)


def forward(params, pts, box_min, box_max, f0, bf16_round=True):
    W, b, w5, b5 = unpack(params)
    r = bf16 if bf16_round else (lambda v: np.asarray(v, np.float64))
    X = r(features(pts, box_min, box_max, f0))
    acts, zs = [X], []
    a = X
    for l in range(4):
        z = a @ r(W[l]).T + b[l]
        a = r(softplus(z))
        zs.append(z)
        acts.append(a)
    out = a @ r(w5) + b5
    return out, zs, acts


def loss_grad(params, pts, labels, box_min, box_max, f0, bf16_round=True):
    """Mean L1 loss, its gradient w.r.t. the parameters, and the predictions."""
    W, b, w5, b5 = unpack(params)
    r = bf16 if bf16_round else (lambda v: np.asarray(v, np.float64))
    out, zs, acts = forward(params, pts, box_min, box_max, f0, bf16_round)
    n = out.shape[0]
    diff = out - np.asarray(labels, np.float64)
    loss = np.abs(diff).mean()
    g = np.sign(diff) / n
    grad = np.zeros(NUM_PARAMS)
    grad[OFF_W5:OFF_B5] = acts[4].T @ g
    grad[OFF_B5] = g.sum()
    da = np.outer(g, r(w5))
    offs_w = [OFF_W1, OFF_W2, OFF_W3, OFF_W4]
    offs_b = [OFF_B1, OFF_B2, OFF_B3, OFF_B4]
    for l in range(3, -1, -1):
        dz = da * softplus_deriv(zs[l])
        grad[offs_w[l]:offs_w[l] + W[l].size] = (dz.T @ acts[l]).ravel()
        grad[offs_b[l]:offs_b[l] + H] = dz.sum(0)
        da = dz @ r(W[l])
    return loss, grad, out


def adam(params, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
