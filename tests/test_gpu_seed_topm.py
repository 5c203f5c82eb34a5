"""Seed selection of the verified exact seed pool (calculator_rover_seed_topm):
per row of a queries x seeds rank matrix, the m smallest keys
(rank bits << 32 | seed index) in ascending order and the (m+1)-th smallest
rank, bit for bit against a numpy sort of the same row.

Covers rows of 50 to 9,000 seeds with spread, clustered, narrow (a few ulps
apart) and many-exponent values, results the register sort and the
shared-memory sort finish, rows shorter than m, signed zeros, ties across
the cut, a flood of equal ranks and rows with an infinite, huge or NaN rank
(all marked for a scan: NaN next, empty keys).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EMPTY = np.uint64(0xFFFFFFFFFFFFFFFF)
GATHER = 2048


def _expected(rank, m):
    rows, n = rank.shape
    keys = np.full((rows, m), EMPTY, np.uint64)
    nxt = np.zeros(rows, np.float32)
    for i in range(rows):
        x = rank[i]
        if not np.all(x < np.float32(3.0e38)):
            nxt[i] = np.nan
            continue
        bits = (x + np.float32(0.0)).view(np.uint32).astype(np.uint64)
        k = np.sort((bits << np.uint64(32)) | np.arange(n, dtype=np.uint64))
        target = min(m + 1, n)
        t = k[target - 1] >> np.uint64(32)
        if np.count_nonzero(bits <= t) > GATHER:
            nxt[i] = np.nan
            continue
        keys[i, :min(m, n)] = k[:m]
        nxt[i] = (np.uint32(k[m] >> np.uint64(32)).view(np.float32) if n > m else np.float32(np.inf))
    return keys, nxt


def _check(calc, rank, m):
    keys, nxt = calc.seed_topm(rank, m)
    ek, en = _expected(rank, m)
    assert np.array_equal(keys, ek)
    assert np.array_equal(nxt.view(np.uint32)[~np.isnan(en)], en.view(np.uint32)[~np.isnan(en)])
    assert np.array_equal(np.isnan(nxt), np.isnan(en))


def _ranks(rng, rows, n, kind):
    if kind == "gamma":          # squared distances to random points
        return rng.gamma(30.0, 1.0, (rows, n)).astype(np.float32)
    if kind == "uniform":
        return rng.uniform(0, 1e4, (rows, n)).astype(np.float32)
    if kind == "narrow":         # a few ulps apart: every histogram pass needed
        base = np.float32(1.0).view(np.uint32)
        return (base + rng.integers(0, 1 << 20, (rows, n)).astype(np.uint32)).view(np.float32)
    if kind == "wide":           # zero to 1e30: bins over many exponents
        return (10.0 ** rng.uniform(-30, 30, (rows, n))).astype(np.float32)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["gamma", "uniform", "narrow", "wide"])
@pytest.mark.parametrize("n,m", [(4096, 96), (4096, 128), (4096, 1024), (1000, 128), (64, 32), (4096, 1)])
def test_topm_matches_sort(calc, kind, n, m):
    rng = np.random.default_rng(n * 7 + m)
    _check(calc, _ranks(rng, 48, n, kind), m)


def test_wide_rows(calc):
    rng = np.random.default_rng(11)
    _check(calc, _ranks(rng, 16, 5000, "gamma"), 128)
    _check(calc, _ranks(rng, 16, 8192, "gamma"), 96)
    _check(calc, _ranks(rng, 8, 8192, "narrow"), 1024)
    _check(calc, _ranks(rng, 8, 9000, "narrow"), 320)
    _check(calc, _ranks(rng, 8, 9000, "gamma"), 96)


def test_short_rows_signed_zeros_and_ties(calc):
    rng = np.random.default_rng(12)
    short = _ranks(rng, 8, 50, "gamma")
    _check(calc, short, 96)                          # n <= m: all keys, next = +inf
    z = _ranks(rng, 8, 4096, "gamma")
    z[:, ::7] = 0.0
    z[:, 3::11] = -0.0                               # folds to +0 like the kernel's + 0.0f
    _check(calc, z, 128)
    ties = np.round(_ranks(rng, 16, 4096, "gamma"))  # ~60 levels: many equal ranks across the cut
    _check(calc, ties, 128)
    _check(calc, ties, 1024)


def test_flood_and_bad_rows_are_marked(calc):
    rng = np.random.default_rng(13)
    r = _ranks(rng, 6, 4096, "gamma")
    r[0, :3000] = 1.0                                # 3,000 equal smallest ranks
    r[1, :2000] = 1.0                                # 2,000: still sorted in shared memory
    r[2, 17] = np.inf
    r[3, 4095] = 3.5e38
    r[4, :] = 2.0                                    # every rank equal
    keys, nxt = calc.seed_topm(r, 128)
    assert np.isnan(nxt[[0, 2, 3, 4]]).all() and np.all(keys[[0, 2, 3, 4]] == EMPTY)
    _check(calc, r, 128)
    for n in (6000, 9000):
        w = _ranks(rng, 3, n, "gamma")
        w[1, :2500] = 0.5
        w[2, n - 1] = np.nan
        _check(calc, w, 128)
