"""CPU oracle of the learned decision network (test infrastructure only).

The network decides, for each decision column of a non-HQ anchor MSA (an
anchor position whose original base differs from the consensus), whether
the consensus base is written. The decision point is the reference's
classifier hook, correctAnchorClf (include/corrector.hpp:1448-1472), which
the reference serves with a random forest (include/forest.hpp:217-226); here
it is a 24 -> 64 -> 64 -> 1 MLP with GELU, trained by binary cross-entropy
with Adam.

Two modes:
- ``emulate=True`` follows the device path's roundings: normalised inputs,
  weights, hidden activations and the backward pass's pre-activation
  gradients are bfloat16 values; products are exact and sums are carried in
  float64 here (the device carries FP32 in tensor-core order), so device and
  oracle differ only by accumulation order.
- ``emulate=False`` is the exact float64 network, used to pin the analytic
  gradient against central finite differences.

Parameter vector (float32): W1[64][24] b1[64] W2[64][64] b2[64] w3[64] b3,
then mean[24] inv_std[24] of the input normalisation.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NFEAT = 24
HIDDEN = 64
W1, B1, W2, B2, W3, B3 = 0, 1536, 1600, 5696, 5760, 5824
NPARAM = 5825
MEAN, ISTD = 5825, 5849
NFLOATS = 5873


def bf16(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 -> float32, round to nearest even."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def unpack(p: np.ndarray):
    p = np.asarray(p)
    return (p[W1:B1].reshape(HIDDEN, NFEAT), p[B1:W2], p[W2:B2].reshape(HIDDEN, HIDDEN), p[B2:W3],
            p[W3:B3], p[B3], p[MEAN:ISTD], p[ISTD:NFLOATS])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def _f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def forward(p: np.ndarray, x: np.ndarray, emulate: bool = True):
    """Logits and the intermediates the backward pass needs."""
    w1, b1, w2, b2, w3, b3, mean, istd = unpack(p)
    if emulate:
        x = np.asarray(x, np.float32)
        xn = bf16((x - mean.astype(np.float32)) * istd.astype(np.float32))
        w1b, w2b, w3b = bf16(w1), bf16(w2), bf16(w3)
        a1 = _f32(xn.astype(np.float64) @ w1b.T.astype(np.float64)) + b1.astype(np.float32)
        h1 = bf16(_f32(gelu(a1.astype(np.float64))))
        a2 = _f32(h1.astype(np.float64) @ w2b.T.astype(np.float64)) + b2.astype(np.float32)
        h2 = bf16(_f32(gelu(a2.astype(np.float64))))
        logit = _f32(h2.astype(np.float64) @ w3b.astype(np.float64)) + np.float32(b3)
    else:
        x = np.asarray(x, np.float64)
        xn = (x - mean) * istd
        w1b, w2b, w3b = w1.astype(np.float64), w2.astype(np.float64), w3.astype(np.float64)
        a1 = xn @ w1b.T + b1
        h1 = gelu(a1)
        a2 = h1 @ w2b.T + b2
        h2 = gelu(a2)
        logit = h2 @ w3b + float(b3)
    return dict(xn=xn, a1=a1, h1=h1, a2=a2, h2=h2, logit=logit, w2b=w2b, w3b=w3b)


def loss_and_grad(p: np.ndarray, x: np.ndarray, y: np.ndarray, emulate: bool = True, w=None):
    """Binary cross-entropy over the rows, each scaled by its weight (1 when
    w is None) and divided by the row count, and its gradient (NPARAM)."""
    f = forward(p, x, emulate)
    B = x.shape[0]
    l = f["logit"].astype(np.float64)
    y = np.asarray(y, np.float64)
    w = np.ones(B) if w is None else np.asarray(w, np.float64)
    loss = float(np.mean(w * (np.maximum(l, 0) - l * y + np.log1p(np.exp(-np.abs(l))))))
    sig = 1.0 / (1.0 + np.exp(-l))
    d = (sig - y) * w / B                                        # dL/dlogit
    g = np.zeros(NPARAM, np.float64)
    h2 = f["h2"].astype(np.float64)
    g[W3:B3] = d @ h2
    g[B3] = d.sum()
    if emulate:
        d32 = _f32(d)
        da2 = bf16((d32[:, None] * f["w3b"][None, :]) * _f32(gelu_grad(f["a2"].astype(np.float64))))
        dh1 = _f32(da2.astype(np.float64) @ f["w2b"].astype(np.float64))
        da1 = bf16(dh1 * _f32(gelu_grad(f["a1"].astype(np.float64))))
    else:
        da2 = d[:, None] * f["w3b"][None, :] * gelu_grad(f["a2"])
        dh1 = da2 @ f["w2b"]
        da1 = dh1 * gelu_grad(f["a1"])
    da2 = da2.astype(np.float64)
    da1 = da1.astype(np.float64)
    g[W2:B2] = (da2.T @ f["h1"].astype(np.float64)).ravel()
    g[B2:W3] = da2.sum(0)
    g[W1:B1] = (da1.T @ f["xn"].astype(np.float64)).ravel()
    g[B1:W2] = da1.sum(0)
    return loss, g


def adam(p: np.ndarray, g: np.ndarray, m: np.ndarray, v: np.ndarray, t: int,
         lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """One Adam update in float32 (bias-corrected moments), in place on the
    first NPARAM entries of p; returns (p, m, v)."""
    f = np.float32
    g = np.asarray(g, f)[:NPARAM]
    bc1 = f(1.0 - b1 ** t)
    bc2 = f(1.0 - b2 ** t)
    m[:] = f(b1) * m + f(1.0 - b1) * g
    v[:] = f(b2) * v + (f(1.0 - b2) * g) * g
    mh = m / bc1
    vh = v / bc2
    p[:NPARAM] = p[:NPARAM] - f(lr) * mh / (np.sqrt(vh) + f(eps))
    return p, m, v


def normalisation(x: np.ndarray):
    """mean and 1/std per feature (std floored at 1e-6)."""
    x = np.asarray(x, np.float64)
    mu = x.mean(0)
    sd = np.maximum(x.std(0), 1e-6)
    return mu.astype(np.float32), (1.0 / sd).astype(np.float32)


def random_params(seed: int, x: np.ndarray | None = None) -> np.ndarray:
    """Uniform fan-in initialisation; normalisation from x if given."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NFLOATS, np.float32)
    p[W1:B1] = rng.uniform(-1, 1, HIDDEN * NFEAT) / np.sqrt(NFEAT)
    p[B1:W2] = rng.uniform(-0.1, 0.1, HIDDEN)
    p[W2:B2] = rng.uniform(-1, 1, HIDDEN * HIDDEN) / np.sqrt(HIDDEN)
    p[B2:W3] = rng.uniform(-0.1, 0.1, HIDDEN)
    p[W3:B3] = rng.uniform(-1, 1, HIDDEN) / np.sqrt(HIDDEN)
    p[B3] = 0.0
    if x is not None:
        p[MEAN:ISTD], p[ISTD:NFLOATS] = normalisation(x)
    else:
        p[ISTD:NFLOATS] = 1.0
    return p
