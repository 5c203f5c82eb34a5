"""CPU oracle of the learned gate's forward and backward passes (test
infrastructure only: tests/, smoke() and bench.py's CPU baseline may use it;
the product path never does).

The gate has no counterpart in the reference: it is a 5 -> 64 -> 64 -> 2 MLP
(ReLU hidden layers, two logits: refine-needed, stop-expanding) that the
batched search consults.  This module restates, in NumPy, the arithmetic the
device kernels perform so their gradients can be checked:

* inputs standardised with (mu, sigma) and rounded to BF16;
* weights rounded to BF16 (round to nearest even), biases FP32;
* hidden activations ReLU'd and rounded to BF16;
* loss per head: masked binary cross-entropy on the logit, positives
  weighted by pos_weight, summed over rows and divided by the row count;
* backward: BF16 roundings treated as identity (straight-through).

Accumulation here is float64, so device results (FP32 accumulation, atomic
order) agree to a relative tolerance, not bit for bit.

Parameter vector layout (FP32, row-major [in][out]):
    w1[5][64] b1[64] w2[64][64] b2[64] w3[64][2] b3[2]
"""
from __future__ import annotations

import numpy as np

IN, HIDDEN, OUT = 5, 64, 2
SIZES = [("w1", (IN, HIDDEN)), ("b1", (HIDDEN,)), ("w2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
         ("w3", (HIDDEN, OUT)), ("b3", (OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    finite = (u & 0x7F800000) != 0x7F800000
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = np.where(finite, r, u & 0xFFFF0000).astype(np.uint32)
    return out.view(np.float32).reshape(a.shape)


def unpack(params: np.ndarray, dtype=np.float32) -> dict:
    p = np.asarray(params, dtype=dtype).ravel()
    assert p.size == N_PARAMS
    out, off = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = p[off:off + n].reshape(shape)
        off += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float32).ravel() for name, _ in SIZES])


def softplus(z):
    return np.where(z > 0, z + np.log1p(np.exp(-np.abs(z))), np.log1p(np.exp(-np.abs(z))))


def forward(params, mu, sigma, x, round_bf16=True):
    """Returns (logits [n][2], cache) for raw inputs x [n][5]."""
    if round_bf16:
        P = unpack(params)
        rnd = lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64)
        xs = rnd((np.asarray(x, np.float32) - np.asarray(mu, np.float32)) / np.asarray(sigma, np.float32))
    else:   # plain float64 network (finite-difference checks of this module)
        P = unpack(params, np.float64)
        rnd = lambda a: np.asarray(a, np.float64)
        xs = (np.asarray(x, np.float64) - np.asarray(mu, np.float64)) / np.asarray(sigma, np.float64)
    w1, w2, w3 = (rnd(P[k]) for k in ("w1", "w2", "w3"))
    a1 = xs @ w1 + P["b1"].astype(np.float64)
    h1 = np.where(a1 > 0, rnd(a1), 0.0)
    a2 = h1 @ w2 + P["b2"].astype(np.float64)
    h2 = np.where(a2 > 0, rnd(a2), 0.0)
    z = h2 @ w3 + P["b3"].astype(np.float64)
    return z, dict(xs=xs, h1=h1, h2=h2, w1=w1, w2=w2, w3=w3)


def loss_and_grad(params, mu, sigma, x, y, m, pos_weight=(1.0, 1.0), round_bf16=True):
    """Mean loss over the n rows and the gradient of every parameter (same
    layout as params), as one device training step computes them."""
    z, c = forward(params, mu, sigma, x, round_bf16)
    y = np.asarray(y, np.float64)
    m = np.asarray(m, np.float64)
    pw = np.asarray(pos_weight, np.float64)[None, :]
    n = z.shape[0]
    loss = float((m * (pw * y * softplus(-z) + (1 - y) * softplus(z))).sum() / n)
    sg = 1.0 / (1.0 + np.exp(-z))
    dz = m * (pw * y * (sg - 1.0) + (1 - y) * sg) / n
    g = {}
    g["w3"] = c["h2"].T @ dz
    g["b3"] = dz.sum(0)
    dh2 = (dz @ c["w3"].T) * (c["h2"] > 0)
    g["w2"] = c["h1"].T @ dh2
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ c["w2"].T) * (c["h1"] > 0)
    g["w1"] = c["xs"].T @ dh1
    g["b1"] = dh1.sum(0)
    return loss, np.concatenate([np.asarray(g[name], np.float64).ravel() for name, _ in SIZES])


def init_params(seed=0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in SIZES:
        if name.startswith("w"):
            lim = np.sqrt(6.0 / shape[0])
            d[name] = rng.uniform(-lim, lim, size=shape).astype(np.float32)
        else:
            d[name] = np.zeros(shape, np.float32)
    return pack(d)
