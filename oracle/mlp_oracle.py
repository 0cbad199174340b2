"""CPU restatement of the learned warm-start network's forward pass and
gradient (icflow_b200/csrc/icf_mlp.cu), the checker for its kernels.  TEST
INFRASTRUCTURE ONLY.  The network has no counterpart in the reference; this
follows the kernel's own definition: inputs normalised as (x - shift) * scale
and rounded to bf16, weights rounded to bf16, FP32 sums, FP32 biases and
GELU(z) = z Phi(z), hidden activations rounded to bf16 before the next
product, loss = mean squared error over nodes and outputs.  With round=False
everything is float64 and unrounded (for finite-difference checks)."""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NI, NH, NO = 15, 64, 3
SIZES = [(NH, NI), (NH,), (NH, NH), (NH,), (NO, NH), (NO,)]


def unpack(p):
    out, o = [], 0
    for s in SIZES:
        n = int(np.prod(s))
        out.append(np.asarray(p[o:o + n]).reshape(s))
        o += n
    return out


def bf16(x):
    """Round float32 values to bf16 (nearest, ties to even), returned as float32."""
    x = np.ascontiguousarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b >> 16) & 1) + 0x7FFF
    return ((b + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def gelu(z):
    return 0.5 * z * (1 + erf(z / np.sqrt(2)))


def gelu_d(z):
    return 0.5 * (1 + erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def forward(p, norm, x, round=True):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    shift, scale = norm[:NI], norm[NI:2 * NI]
    f = np.float32 if round else np.float64
    r = bf16 if round else (lambda a: np.asarray(a, np.float64))
    xn = r((np.asarray(x, f) - f(shift)) * f(scale))
    W1r, W2r, W3r = r(W1), r(W2), r(W3)
    z1 = (xn.astype(np.float64) @ W1r.T.astype(np.float64)).astype(f) + f(b1)
    h1 = r(gelu(z1.astype(np.float64)).astype(f))
    z2 = (h1.astype(np.float64) @ W2r.T.astype(np.float64)).astype(f) + f(b2)
    h2 = r(gelu(z2.astype(np.float64)).astype(f))
    y = (h2.astype(np.float64) @ W3r.T.astype(np.float64)).astype(f) + f(b3)
    return dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2, y=y, W=(W1r, W2r, W3r))


def loss_and_grad(p, norm, x, t, round=True):
    c = forward(p, norm, x, round)
    n = len(x)
    d = c["y"].astype(np.float64) - np.asarray(t, np.float64)
    loss = float((d * d).sum() / (n * NO))
    dy = 2 * d / (n * NO)
    W1r, W2r, W3r = (w.astype(np.float64) for w in c["W"])
    h1, h2, xn = (c[k].astype(np.float64) for k in ("h1", "h2", "xn"))
    dz2 = (dy @ W3r) * gelu_d(c["z2"].astype(np.float64))
    dz1 = (dz2 @ W2r) * gelu_d(c["z1"].astype(np.float64))
    g = [dz1.T @ xn, dz1.sum(0), dz2.T @ h1, dz2.sum(0), dy.T @ h2, dy.sum(0)]
    return loss, np.concatenate([a.ravel() for a in g])
