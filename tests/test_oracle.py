"""The CPU restatement (oracle/rover_oracle.c) against the golden outputs the
compiled reference produced (tests/golden/make_golden.py), bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import PQ_FIXTURES, SQ_FIXTURES, load_fixture


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.parametrize("name", PQ_FIXTURES)
def test_pq_lut_adc_residual(port, name):
    data, graph, b, g, q = load_fixture(name)
    ix = port.pq_index(graph, b)
    for qi in range(4):
        lut = port.pq_lut(ix, q[qi])
        assert np.array_equal(bits(lut), bits(g["lut"][qi]))
        assert np.array_equal(bits(port.pq_adc(ix, lut, g["sample_ids"])), bits(g["adc"][qi]))
        assert np.array_equal(bits(port.pq_residual_eval(ix, q[qi], g["sample_ids"])), bits(g["residual"][qi]))


@pytest.mark.parametrize("name", PQ_FIXTURES)
def test_pq_known_answer_adc(port, name):
    """build_pure_pq_index.reference_adc (an independent NumPy ADC) agrees
    within 1e-5 relative (its LUT sums may use pairwise order)."""
    data, graph, b, g, q = load_fixture(name)
    ix = port.pq_index(graph, b)
    for qi in range(4):
        ours = port.pq_adc(ix, port.pq_lut(ix, q[qi]), g["known_adc_ids"]).astype(np.float64)
        np.testing.assert_allclose(ours, g["known_adc"][qi], rtol=1e-5)


@pytest.mark.parametrize("name", PQ_FIXTURES)
@pytest.mark.parametrize("tag", ["on", "off", "on_ep8", "on_exp6"])
def test_pq_search(port, name, tag):
    data, graph, b, g, q = load_fixture(name)
    ix = port.pq_index(graph, b)
    corr, ep, exp = (int(x) for x in g[f"search_{tag}_params"])
    r = port.pq_search(ix, data["graph_entry"], q, g["pool_sizes"], ep, exp, correction=corr,
                       refine_budget=20 if corr else 0, top_k=10)
    for k in ("pool_ids", "pool_counts", "ids", "counts", "stats"):
        assert np.array_equal(r[k], g[f"search_{tag}_{k}"]), k
    assert np.array_equal(bits(r["pool_dists"]), bits(g[f"search_{tag}_pool_dists"]))
    assert np.array_equal(bits(r["dists"]), bits(g[f"search_{tag}_dists"]))


@pytest.mark.parametrize("name", SQ_FIXTURES)
def test_sq_codes_and_distances(port, name):
    data, graph, b, g, q = load_fixture(name)
    ix = port.sq_index(graph, b)
    for qi in range(len(q)):
        assert np.array_equal(port.sq_quantize(ix, q[qi]), g["query_codes"][qi])
    for qi in range(4):
        assert np.array_equal(bits(port.sq_coarse(ix, q[qi], g["sample_ids"])), bits(g["coarse"][qi]))
        assert np.array_equal(bits(port.sq_exact(ix, q[qi], g["sample_ids"])), bits(g["exact"][qi]))


def _rerank_candidates(sample, n, seed=0):
    """Candidates as a legacy search hands them to the re-rank: shuffled,
    one id twice, one id outside the index."""
    rng = np.random.default_rng(seed)
    c = list(rng.permutation(np.asarray(sample, np.int32)))
    return np.array(c[:3] + [c[1]] + c[3:] + [n + 5], np.int32)


@pytest.mark.parametrize("name", SQ_FIXTURES)
def test_sq_rerank_restatement(port, name):
    """demo_rerank_candidates restated: its distances are the reference's
    exact residual distances (pinned by the golden vectors), FLT_MAX for an
    id outside the index; the order is stable by distance, ties in id order."""
    data, graph, b, g, q = load_fixture(name)
    ix = port.sq_index(graph, b)
    sample = np.asarray(g["sample_ids"], np.int32)
    for qi in range(4):
        exact = dict(zip(sample.tolist(), bits(g["exact"][qi]).tolist()))
        cand = _rerank_candidates(sample, b.num_vectors, qi)
        ids, d = port.sq_rerank(ix, q[qi], cand, len(cand))
        assert len(ids) == len(cand)
        for i, di in zip(ids.tolist(), bits(d).tolist()):
            assert di == (exact[i] if i in exact else bits(np.float32(3.4028235e38)))
        keys = list(zip(d.tolist(), ids.tolist()))
        assert keys == sorted(keys)          # (distance, id): ties kept in id order
        top, _ = port.sq_rerank(ix, q[qi], cand, 5)
        assert np.array_equal(top, ids[:5])


@pytest.mark.parametrize("name", SQ_FIXTURES)
@pytest.mark.parametrize("tag", ["on", "off", "on_ep8", "off_ep16_exp5"])
def test_sqmd_search(port, name, tag):
    data, graph, b, g, q = load_fixture(name)
    ix = port.sq_index(graph, b)
    corr, ep, exp = (int(x) for x in g[f"sqmd_{tag}_params"])
    stride = int(g["pool_sizes"].max())
    for qi in range(len(q)):
        ids, d, _ = port.sqmd_search(ix, data["graph_entry"], q[qi], int(g["pool_sizes"][qi]), ep, exp,
                                     correction=corr, out_cap=stride)
        c = int(g[f"sqmd_{tag}_counts"][qi])
        assert len(ids) == c
        assert np.array_equal(ids, g[f"sqmd_{tag}_ids"][qi, :c])
        assert np.array_equal(bits(d), bits(g[f"sqmd_{tag}_dists"][qi, :c]))
        if f"sqmd_{tag}_refine_ids" in g:
            ri, rd = port.refine(0, ix, q[qi], ids[:min(c, 20)], 10)
            assert np.array_equal(ri, g[f"sqmd_{tag}_refine_ids"][qi, :len(ri)])
            assert np.array_equal(bits(rd), bits(g[f"sqmd_{tag}_refine_dists"][qi, :len(ri)]))


@pytest.mark.parametrize("name", SQ_FIXTURES)
@pytest.mark.parametrize("tag", ["ep1", "ep8", "ep4_exp4"])
def test_dsp_search(port, name, tag):
    data, graph, b, g, q = load_fixture(name)
    ix = port.sq_index(graph, b)
    ep, exp, num_out = (int(x) for x in g[f"dsp_{tag}_params"])
    for qi in range(len(q)):
        ids, d = port.dsp_search(ix, data["graph_entry"], q[qi], int(g["pool_sizes"][qi]), ep, exp, num_out)
        c = int(g[f"dsp_{tag}_counts"][qi])
        assert np.array_equal(ids, g[f"dsp_{tag}_ids"][qi, :c])
        assert np.array_equal(bits(d), bits(g[f"dsp_{tag}_dists"][qi, :c]))
