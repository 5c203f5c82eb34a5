"""The gate's CPU oracle (oracle/gate_oracle.py): its analytic gradients
against central finite differences of its own float64 loss, and its BF16
rounding against known values.  The device kernels are checked against this
oracle in tests/test_gpu_gate.py."""
from __future__ import annotations

import numpy as np

from oracle import gate_oracle as G


def _data(n=64, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, G.IN)).astype(np.float32) * np.array([1, 0.3, 1, 0.2, 2], np.float32) + 1.0
    y = (rng.random((n, G.OUT)) < 0.4).astype(np.float32)
    m = (rng.random((n, G.OUT)) < 0.8).astype(np.float32)
    return x, y, m


def test_bf16_rounding_known_values():
    v = np.array([1.0, 1.00390625, 1.005859375, 3.140625, -2.5, 65504.0, 1e-40], np.float32)
    r = G.bf16(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties to even keep 1.0
    assert r[0] == 1.0 and r[1] == 1.0
    # 1 + 3 * 2^-9 rounds up to 1 + 2^-7
    assert r[2] == np.float32(1.0078125)
    assert r[3] == np.float32(3.140625) and r[4] == -2.5
    assert r[5] == np.float32(65536.0)
    assert G.bf16(np.array([np.inf, -np.inf], np.float32)).tolist() == [np.inf, -np.inf]
    assert np.isnan(G.bf16(np.array([np.nan], np.float32)))[0]


def test_gradients_match_finite_differences():
    x, y, m = _data()
    mu, sigma = x.mean(0), x.std(0) + 1e-3
    params = G.init_params(3).astype(np.float64)
    pw = (2.0, 0.7)
    loss, grad = G.loss_and_grad(params, mu, sigma, x, y, m, pw, round_bf16=False)
    rng = np.random.default_rng(5)
    coords = np.concatenate([rng.choice(G.N_PARAMS, 40, replace=False), [G.N_PARAMS - 1, G.N_PARAMS - 2]])
    eps = 1e-6
    for i in coords:
        pp, pm = params.copy(), params.copy()
        pp[i] += eps
        pm[i] -= eps
        lp, _ = G.loss_and_grad(pp, mu, sigma, x, y, m, pw, round_bf16=False)
        lm, _ = G.loss_and_grad(pm, mu, sigma, x, y, m, pw, round_bf16=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])
    assert np.isfinite(loss) and loss > 0


def test_pack_roundtrip():
    p = G.init_params(1)
    assert p.size == G.N_PARAMS == 4674
    assert np.array_equal(G.pack(G.unpack(p)), p)
