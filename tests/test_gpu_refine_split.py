"""The final refine's ERROR4 mode and the SQ4 split distance on the GPU,
through the C-ABI, against the oracle (itself pinned against the reference
CLI in tests/test_oracle_refine_split.py) on the golden fixtures' artifacts:
bit-exact ids and distances.

* PQ: calculator_rover_pq_search with third_residual (the fused refine of
  the search kernels, packed and decoded layouts, exact and batched modes)
  and calculator_rover_refine kind 4;
* SQ: calculator_rover_refine kind 3;
* SQ4 split: calculator_rover_sq_search with split_distance (sq_mode 1), and
  the entry points refusing what they cannot serve.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, PQ_FIXTURES, SQ_FIXTURES, load_fixture

pytestmark = pytest.mark.gpu

PACKED, DECODED = 1, 2
AEE_EBADPARM = 14


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _e4(port, name, data):
    from oracle.bindings import read_error4
    qp, blocks, _, _ = read_error4(GOLDEN / name / "error4.refine", data["n"], data["dim"])
    return qp, blocks, port.error4(GOLDEN / name / "error4.refine", data["n"], data["dim"])


@pytest.mark.parametrize("name", PQ_FIXTURES)
@pytest.mark.parametrize("mode,layout", [(0, PACKED), (0, DECODED), (1, DECODED)])
def test_pq_search_error4_refine_matches_oracle(calc, port, name, mode, layout):
    data, graph, b, g, q = load_fixture(name)
    calc.pq_load(graph, data["graph_entry"], b)
    qp, blocks, e4 = _e4(port, name, data)
    calc.error4_load(1, qp, blocks)
    pools = g["pool_sizes"]
    budget, k, ep, exp = 20, 10, 4, min(16, data["graph_degree"])
    kw = dict(entry_points=ep, expand_count=exp, correction=1, layout=layout, mode=mode,
              beam_width=1 if mode else 0)
    r = calc.pq_search(q, pools, top_k=k, pool_stride=int(pools.max()), refine_budget=budget, third_residual=1,
                       **kw)
    ix = port.pq_index(graph, b)
    for i in range(len(q)):
        c = min(int(r["pool_counts"][i]), budget)
        oi, od = port.refine_ex(1, ix, e4, q[i], r["pool_ids"][i, :c], k)
        assert r["counts"][i] == len(oi)
        assert np.array_equal(r["ids"][i, :len(oi)], oi), i
        assert np.array_equal(bits(r["dists"][i, :len(oi)]), bits(od)), i
    # the mode-1 refine of the same pools differs: the term is applied
    r1 = calc.pq_search(q, pools, top_k=k, pool_stride=int(pools.max()), refine_budget=budget, **kw)
    assert np.array_equal(r1["pool_ids"], r["pool_ids"])
    assert not np.array_equal(bits(r1["dists"]), bits(r["dists"]))
    # the refine entry point on explicit lists: kind 4 = kind 1 in mode ERROR4
    cand = r["pool_ids"][:, :budget].copy()
    counts = np.minimum(r["pool_counts"], budget).astype(np.int32)
    ids, dists, cnt = calc.refine(4, q, cand, counts, k)
    assert np.array_equal(ids, r["ids"]) and np.array_equal(bits(dists), bits(r["dists"]))
    calc.error4_unload(1)
    bad = calc.pq_search(q, pools, top_k=k, refine_budget=budget, third_residual=1, check=False, **kw)
    assert bad["rc"] == AEE_EBADPARM


@pytest.mark.parametrize("name", SQ_FIXTURES)
def test_sq_refine_error4_matches_oracle(calc, port, name):
    data, graph, b, g, q = load_fixture(name)
    calc.sq_load(graph, data["graph_entry"], b)
    qp, blocks, e4 = _e4(port, name, data)
    calc.error4_load(0, qp, blocks)
    ix = port.sq_index(graph, b)
    rng = np.random.default_rng(3)
    cand = np.stack([rng.choice(data["n"], 24, replace=False) for _ in range(len(q))]).astype(np.int32)
    counts = np.array([24 - (i % 5) for i in range(len(q))], np.int32)
    ids, dists, cnt = calc.refine(3, q, cand, counts, 10)
    for i in range(len(q)):
        oi, od = port.refine_ex(0, ix, e4, q[i], cand[i, :counts[i]], 10)
        assert cnt[i] == len(oi)
        assert np.array_equal(ids[i, :cnt[i]], oi) and np.array_equal(bits(dists[i, :cnt[i]]), bits(od)), i


def test_sq_split_search_matches_oracle(calc, port):
    from oracle.bindings import read_bias
    name = "sq4_d24"
    data, graph, b, g, q = load_fixture(name)
    calc.sq_load(graph, data["graph_entry"], b)
    bias = read_bias(GOLDEN / name / "correction_bias.f32", data["n"])
    ix = port.sq_index(graph, b)
    pools = g["pool_sizes"]
    kw = dict(entry_points=6, expand_count=8, correction=1, seed=42)
    no_bias = calc.sq_search(q, pools, 30, sq_mode=1, split_distance=1, check=False, **kw)
    assert no_bias["rc"] == AEE_EBADPARM
    calc.sq_split_load(bias)
    r = calc.sq_search(q, pools, 30, sq_mode=1, split_distance=1, **kw)
    for i in range(len(q)):
        oi, od, _ = port.sqmd_search_split(ix, bias, data["graph_entry"], q[i], int(pools[i]), 6, 8, out_cap=30)
        c = r["counts"][i]
        assert c == len(oi), i
        assert np.array_equal(r["ids"][i, :c], oi) and np.array_equal(bits(r["dists"][i, :c]), bits(od)), i
    # DB-pair order and coarse-only searches do not take the split distance
    assert calc.sq_search(q, pools, 30, sq_mode=2, split_distance=1, check=False, **kw)["rc"] == AEE_EBADPARM
    kw["correction"] = 0
    assert calc.sq_search(q, pools, 30, sq_mode=1, split_distance=1, check=False, **kw)["rc"] == AEE_EBADPARM


def test_split_bias_needs_four_bit_codes(calc):
    data, graph, b, g, q = load_fixture("sq8_d32")
    calc.sq_load(graph, data["graph_entry"], b)
    with pytest.raises(Exception, match="4-bit"):
        calc.sq_split_load(np.zeros(data["n"], np.float32))
