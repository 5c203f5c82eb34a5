"""CUDA path (through the C-ABI of libcalculator.so) against the reference's
golden outputs and the oracle restatement: bit-exact ids and distances."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import PQ_FIXTURES, SQ_FIXTURES, load_fixture

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def rows_equal(ids, dists, counts, g_ids, g_dists, g_counts):
    assert np.array_equal(counts, g_counts)
    for i, c in enumerate(counts):
        assert np.array_equal(ids[i, :c], g_ids[i, :c]), f"ids row {i}"
        assert np.array_equal(bits(dists[i, :c]), bits(g_dists[i, :c])), f"dists row {i}"


@pytest.mark.parametrize("name", PQ_FIXTURES)
def test_pq_lut_adc_residual(calc, name):
    data, graph, b, g, q = load_fixture(name)
    calc.pq_load(graph, data["graph_entry"], b)
    luts = calc.pq_lut(q[:4], b.meta.m, b.meta.ks)
    assert np.array_equal(bits(luts), bits(g["lut"]))
    adc = calc.score(0, q[:4], [g["sample_ids"]] * 4)
    res = calc.score(1, q[:4], [g["sample_ids"]] * 4)
    dec = calc.score(4, q[:4], [g["sample_ids"]] * 4)    # the same distances from decoded rows
    for qi in range(4):
        assert np.array_equal(bits(adc[qi]), bits(g["adc"][qi]))
        assert np.array_equal(bits(res[qi]), bits(g["residual"][qi]))
        assert np.array_equal(bits(dec[qi]), bits(g["residual"][qi]))


PACKED, DECODED = 1, 2


@pytest.mark.parametrize("name", PQ_FIXTURES)
@pytest.mark.parametrize("tag", ["on", "off", "on_ep8", "on_exp6"])
@pytest.mark.parametrize("layout", [PACKED, DECODED])
def test_pq_search_matches_reference(calc, name, tag, layout):
    data, graph, b, g, q = load_fixture(name)
    calc.pq_load(graph, data["graph_entry"], b)
    corr, ep, exp = (int(x) for x in g[f"search_{tag}_params"])
    if layout == DECODED and not corr:
        pytest.skip("decoded rows serve the corrected distance only")
    stride = g[f"search_{tag}_pool_ids"].shape[1]
    r = calc.pq_search(q, g["pool_sizes"], top_k=10, pool_stride=stride, entry_points=ep, expand_count=exp,
                       correction=corr, refine_budget=20 if corr else 0, layout=layout)
    rows_equal(r["pool_ids"], r["pool_dists"], r["pool_counts"], g[f"search_{tag}_pool_ids"],
               g[f"search_{tag}_pool_dists"], g[f"search_{tag}_pool_counts"])
    rows_equal(r["ids"], r["dists"], r["counts"], g[f"search_{tag}_ids"], g[f"search_{tag}_dists"],
               g[f"search_{tag}_counts"])
    assert np.array_equal(r["stats"], g[f"search_{tag}_stats"])


@pytest.mark.parametrize("name", SQ_FIXTURES)
def test_sq_rerank_matches_oracle(calc, port, name):
    """Refine kind 2 (demo_rerank_candidates) against the oracle, bit for
    bit: shuffled candidates with a repeated id and one outside the index,
    then the legacy device search's own output lists."""
    data, graph, b, g, q = load_fixture(name)
    calc.sq_load(graph, data["graph_entry"], b)
    ix = port.sq_index(graph, b)
    rng = np.random.default_rng(5)
    sample = np.asarray(g["sample_ids"], np.int32)
    lists = [np.concatenate([rng.permutation(sample), sample[:2], [b.num_vectors + 3]]).astype(np.int32)
             for _ in range(len(q))]
    stride = max(len(x) for x in lists)
    cand = np.full((len(q), stride), -1, np.int32)
    counts = np.array([len(x) for x in lists], np.int32)
    for i, x in enumerate(lists):
        cand[i, :len(x)] = x
    for top_k in (10, stride):
        ids, d, c = calc.refine(2, q, cand, counts, top_k)
        for qi in range(len(q)):
            oi, od = port.sq_rerank(ix, q[qi], lists[qi], top_k)
            assert c[qi] == len(oi)
            assert np.array_equal(ids[qi, :c[qi]], oi)
            assert np.array_equal(bits(d[qi, :c[qi]]), bits(od))


@pytest.mark.parametrize("name", SQ_FIXTURES)
def test_sq_distances(calc, name):
    data, graph, b, g, q = load_fixture(name)
    calc.sq_load(graph, data["graph_entry"], b)
    coarse = calc.score(2, q[:4], [g["sample_ids"]] * 4)
    exact = calc.score(3, q[:4], [g["sample_ids"]] * 4)
    for qi in range(4):
        assert np.array_equal(bits(coarse[qi]), bits(g["coarse"][qi]))
        assert np.array_equal(bits(exact[qi]), bits(g["exact"][qi]))


@pytest.mark.parametrize("name", SQ_FIXTURES)
@pytest.mark.parametrize("tag", ["on", "off", "on_ep8", "off_ep16_exp5"])
def test_sqmd_search_matches_reference(calc, name, tag):
    data, graph, b, g, q = load_fixture(name)
    calc.sq_load(graph, data["graph_entry"], b)
    corr, ep, exp = (int(x) for x in g[f"sqmd_{tag}_params"])
    stride = g[f"sqmd_{tag}_ids"].shape[1]
    r = calc.sq_search(q, g["pool_sizes"], stride, sq_mode=1, entry_points=ep, expand_count=exp, correction=corr)
    rows_equal(r["ids"], r["dists"], r["counts"], g[f"sqmd_{tag}_ids"], g[f"sqmd_{tag}_dists"],
               g[f"sqmd_{tag}_counts"])
    if f"sqmd_{tag}_refine_ids" in g:
        counts = np.minimum(r["counts"], 20)
        oi, od, oc = calc.refine(0, q, r["ids"][:, :20], counts, 10)
        rows_equal(oi, od, oc, g[f"sqmd_{tag}_refine_ids"], g[f"sqmd_{tag}_refine_dists"],
                   g[f"sqmd_{tag}_refine_counts"])


@pytest.mark.parametrize("name", SQ_FIXTURES)
@pytest.mark.parametrize("tag", ["ep1", "ep8", "ep4_exp4"])
def test_dsp_search_matches_reference(calc, name, tag):
    data, graph, b, g, q = load_fixture(name)
    calc.sq_load(graph, data["graph_entry"], b)
    ep, exp, num_out = (int(x) for x in g[f"dsp_{tag}_params"])
    r = calc.sq_search(q, g["pool_sizes"], num_out, sq_mode=0, num_out=num_out, entry_points=ep, expand_count=exp)
    rows_equal(r["ids"], r["dists"], r["counts"], g[f"dsp_{tag}_ids"], g[f"dsp_{tag}_dists"], g[f"dsp_{tag}_counts"])


@pytest.mark.parametrize("name", SQ_FIXTURES)
def test_legacy_retrieval_search(calc, name):
    """calculator_retrieval_load / _search, one query per call, as the
    reference host's RPC worker threads issue them."""
    data, graph, b, g, q = load_fixture(name)
    ep, exp, num_out = (int(x) for x in g["dsp_ep8_params"])
    assert calc.rover_configure(1, b.l1_bits) == 0
    assert calc.retrieval_load(graph, b.l1, b.num_vectors, b.dim, graph.shape[1], data["graph_entry"],
                               b.l1_scale, b.l1_zero) == 0
    for qi in range(len(q)):
        rc, ids, d = calc.retrieval_search(q[qi], ep, exp, int(g["pool_sizes"][qi]), num_out)
        assert rc == 0
        c = int(g["dsp_ep8_counts"][qi])
        assert np.array_equal(ids, g["dsp_ep8_ids"][qi, :c])
        assert np.array_equal(bits(d), bits(g["dsp_ep8_dists"][qi, :c]))
    assert calc.retrieval_unload() == 0


_RANDOM = {}


def _random_pq_index():
    """A 12K x 128 random index (M=16, 8-bit residuals, alpha-pruned
    degree-24 graph) and 200 queries, built once per session."""
    if not _RANDOM:
        from rover_b200 import bundle as B
        from rover_b200 import datasets as D
        n, dim = 12000, 128
        base = D.gmm(n, dim, 32, 5)
        queries = D.gmm(200, dim, 32, 6, centers_seed=5)
        graph = D.pruned_graph(base, 32, 24, 1.2)
        entry = D.medoid(base)
        book, codes, rows, qp = D.pq_prepare(base, 16, 256, 6, 8)
        bundle = B.PqBundle(B.PqMeta(b"\x01" * 16, n, dim, 16, 256, 8, 16), book, codes, 8,
                            B.pack_residual_blocks(rows), qp)
        _RANDOM.update(graph=graph, entry=entry, bundle=bundle, queries=queries)
    return _RANDOM


# (entry points, beam widths): few seeds with uneven beams; many seeds
# (several 64-seed tiles, LCG repeats) with beams wide enough that some
# queries overflow the shared-memory visited table into the global one;
# most of the index as seeds with beams up to 128, where lanes often hold
# more than 8 of the best seeds and the seed selection re-reads its row.
RANDOM_CASES = {"ep4": (4, [16, 32, 64, 100, 128]), "ep700": (700, [32, 64, 512, 1024]),
                "ep4000": (4000, [8, 96, 128])}


@pytest.mark.parametrize("case", sorted(RANDOM_CASES))
@pytest.mark.parametrize("layout", [PACKED, DECODED])
def test_pq_search_random_vs_oracle(calc, port, case, layout):
    """The CUDA search against the oracle restatement on a larger random
    index, both residual layouts."""
    d = _random_pq_index()
    ep, choices = RANDOM_CASES[case]
    queries = d["queries"]
    pools = np.random.default_rng(1).choice(choices, size=len(queries)).astype(np.int32)
    calc.pq_load(d["graph"], d["entry"], d["bundle"])
    stride = int(pools.max())
    r = calc.pq_search(queries, pools, top_k=10, pool_stride=stride, entry_points=ep, expand_count=24,
                       correction=1, refine_budget=20, layout=layout)
    ix = port.pq_index(d["graph"], d["bundle"])
    o = port.pq_search(ix, d["entry"], queries, pools, ep, 24, correction=1, refine_budget=20, top_k=10)
    rows_equal(r["pool_ids"], r["pool_dists"], r["pool_counts"], o["pool_ids"], o["pool_dists"], o["pool_counts"])
    rows_equal(r["ids"], r["dists"], r["counts"], o["ids"], o["dists"], o["counts"])
    assert np.array_equal(r["stats"], o["stats"])


@pytest.mark.parametrize("layout", [PACKED, DECODED])
def test_pq_search_invalid_qparams_fail_like_reference(calc, layout):
    """A vector with scale <= 0 fails every query that scores it
    (retrieval_pq_residual_query_evaluate rejects it); other queries are
    unaffected and the call reports the failure."""
    from rover_b200 import bundle as B
    d = _random_pq_index()
    b0 = d["bundle"]
    qp = b0.qparams.copy()
    bad_id = int(d["entry"])
    qp[bad_id, 0] = 0.0
    bundle = B.PqBundle(b0.meta, b0.codebook, b0.codes, b0.residual_bits, b0.residual_blocks, qp)
    calc.pq_load(d["graph"], d["entry"], bundle)
    queries = d["queries"][:16]
    r = calc.pq_search(queries, 32, top_k=10, entry_points=4, expand_count=24, correction=1, refine_budget=20,
                       layout=layout, check=False)
    assert r["rc"] != 0
    assert np.all(r["status"] == 2)  # the graph entry is every query's first seed
