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



def _bf16_tie_distance(v):
    """Distance of each float64 value from the nearest bf16 rounding boundary
    (a midpoint between two adjacent bf16 numbers)."""
    v = np.abs(np.asarray(v, np.float64))
    f = v.astype(np.float32)
    b = f.view(np.uint32).astype(np.uint64) & 0xFFFF0000
    lo = b.astype(np.uint32).view(np.float32).astype(np.float64)
    hi = (b + 0x10000).astype(np.uint32).view(np.float32).astype(np.float64)
    prev = (np.maximum(b, 0x10000) - 0x10000).astype(np.uint32).view(np.float32).astype(np.float64)
    return np.minimum(np.abs(v - 0.5 * (lo + hi)), np.abs(v - 0.5 * (prev + lo)))


def check_trace(p, norm, x, tr):
    """Layer-by-layer check of the kernel's forward trace (z1, h1, z2, h2, y
    as returned by icf_mlp_forward_trace), each layer from the kernel's own
    previous layer, so a bf16 rounding that float32 summation order decides
    differently from float64 does not propagate.  Per layer:

      z = bf16(h_prev) W^T + b    float64 from the kernel's h_prev; the
                                  kernel's float32 z must lie within the
                                  summation bound (K + 2) 2^-24 sum|terms| (K
                                  the products per sum);
      h = bf16(GELU(z))           from the kernel's z in float64: equal to the
                                  kernel's h, except where GELU(z) is within
                                  2^-20 (|h| + |z|) of a bf16 rounding boundary
                                  (float32 erff and products), where the two
                                  neighbours are both allowed.

    The first layer's input is the restatement's normalised bf16 input (the
    same float32 subtraction and product).  Returns the worst ratio of error
    to bound per layer (<= 1 passes), the count of near-tie activations and
    the number of activations outside both rules."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    shift, scale = norm[:NI], norm[NI:2 * NI]
    u = 2.0 ** -24
    xn = bf16((np.asarray(x, np.float32) - shift.astype(np.float32)) * scale.astype(np.float32)).astype(np.float64)
    rep = {"near_ties": 0, "mismatched": 0}
    h = xn
    for name, W, b, zk, hk in (("1", W1, b1, tr["z1"], tr["h1"]), ("2", W2, b2, tr["z2"], tr["h2"]),
                               ("3", W3, b3, tr["y"], None)):
        Wr = bf16(W).astype(np.float64)
        z = h @ Wr.T + b.astype(np.float32).astype(np.float64)
        bound = (Wr.shape[1] + 2) * u * (np.abs(h) @ np.abs(Wr).T + np.abs(b)) + 1e-300
        rep["z" + name] = float((np.abs(np.asarray(zk, np.float64) - z) / bound).max())
        if hk is None:
            break
        zk64 = np.asarray(zk, np.float64)
        g = gelu(zk64)
        hr = bf16(g.astype(np.float32)).astype(np.float64)
        hk64 = np.asarray(hk, np.float64)
        tie = _bf16_tie_distance(g) <= 2.0 ** -20 * (np.abs(g) + np.abs(zk64))
        diff = hk64 != hr
        rep["near_ties"] += int((diff & tie).sum())
        rep["mismatched"] += int((diff & ~tie).sum())
        h = hk64
    return rep
