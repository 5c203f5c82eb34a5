"""The seed ranking on the tensor cores (calculator_rover_seed_rank).

The verified seed pool (pq_seed_pool.cuh) ranks every entry seed by
A = |q|^2 + |x|^2 - 2 q.x with TF32 tensor-core dot products and relies on
|A - d| <= eps = 3 * 2^-9 sqrt(|q|^2 |x|^2) + 2^-13 (|q|^2 + |x|^2 + A) for the
exact distance d.  These tests hold the ranks of the tcgen05 kernel (dims 32
to 128 in steps of 32) and of the mma.sync kernel (other dims, or
ROVER_SEED_RANK=mma) to that bound against float64 distances, on shapes whose
query and seed counts are not multiples of the 128 x 128 tiles.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def _case(nq, n, dim, seed, clip=True):
    rng = np.random.default_rng(seed)
    centres = rng.normal(0, 2.0, size=(16, dim))
    q = centres[rng.integers(0, 16, nq)] + rng.normal(0, 0.5, size=(nq, dim))
    x = centres[rng.integers(0, 16, n)] + rng.normal(0, 0.5, size=(n, dim))
    if clip:
        q, x = np.maximum(q, 0), np.maximum(x, 0)
    return q.astype(np.float32), x.astype(np.float32)


def _check(calc, q, x):
    a = calc.seed_rank(q, x).astype(np.float64)
    qd, xd = q.astype(np.float64), x.astype(np.float64)
    qn, xn = (qd * qd).sum(1), (xd * xd).sum(1)
    d = np.maximum(qn[:, None] + xn[None, :] - 2.0 * qd @ xd.T, 0.0)
    eps = 3 * 2.0 ** -9 * np.sqrt(qn[:, None] * xn[None, :]) + 2.0 ** -13 * (qn[:, None] + xn[None, :] + a)
    worst = float(np.max(np.abs(a - d) / eps))
    assert np.all(np.isfinite(a)) and np.all(a >= 0)
    assert worst <= 1.0, f"rank error reaches {worst:.3f} of the verified pool's bound"
    return worst


@pytest.mark.parametrize("dim", [128, 96, 64, 32, 40])
def test_seed_ranks_within_the_verified_pool_bound(calc, dim):
    q, x = _case(300, 1000, dim, dim)
    _check(calc, q, x)


def test_seed_ranks_many_tiles_and_signs(calc):
    q, x = _case(1000, 8192, 128, 3, clip=False)
    _check(calc, q, x)


def test_mma_sync_ranking_meets_the_same_bound():
    """The fallback kernel, selected through the environment in a fresh process."""
    code = (
        "import sys; sys.path.insert(0, %r); sys.path.insert(0, %r)\n"
        "from test_gpu_seed_rank import _case, _check\n"
        "from rover_b200.calculator import Calculator\n"
        "q, x = _case(300, 1000, 128, 7)\n"
        "print('worst', _check(Calculator(), q, x))\n"
    ) % (str(ROOT), str(ROOT / "tests"))
    env = dict(os.environ, ROVER_SEED_RANK="mma")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "worst" in p.stdout
