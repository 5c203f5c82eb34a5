"""The large combined configuration's components at 100K against the
compiled reference (oracle/_ref): the 10M x 128 recipe (workloads.LARGE_
CONFIGS, pq_c5_100k = the same recipe at n = 100,000) with PQ M=32 x 256
trained and encoded by the library's GPU trainer, 8-bit residuals, a
degree-32 clustered graph, and the 4-bit global SQ codec with 8-bit
residuals over the same vectors.

* PQ32: the exact search (both residual layouts) and its refined top-10
  equal retrieval_pure_pq_search_scalar_with_policy + the ONLINE residual
  policy + retrieval_final_refine bit for bit, with uneven beams in
  [32, 256];
* SQ4: the SQMD search with residual correction and the final refine equal
  sqmd_cpu_state_run_fake_dsp + retrieval_final_refine bit for bit.
"""
from __future__ import annotations

import os
import tempfile
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PACKED, DECODED = 1, 2
NQ, EP, TOP_K, REFINE = 300, 2048, 10, 20


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def rows_equal(ids, dists, counts, g_ids, g_dists, g_counts, what):
    assert np.array_equal(counts, g_counts), f"{what}: counts"
    for i, c in enumerate(counts):
        assert np.array_equal(ids[i, :c], g_ids[i, :c]), f"{what}: ids row {i}"
        assert np.array_equal(bits(dists[i, :c]), bits(g_dists[i, :c])), f"{what}: dists row {i}"


@pytest.fixture(scope="module")
def c5(calc):
    from oracle import bindings
    if not bindings.reference_available():
        pytest.skip("oracle/_ref was not built (reference sources absent at build time)")
    from rover_b200 import bundle as B
    from rover_b200 import workloads
    ref = bindings.Reference()
    w = workloads.build_large("pq_c5_100k", calc, verbose=False)
    q = w.queries[:NQ]
    pools = np.random.default_rng(5).integers(32, 257, NQ).astype(np.int32)
    expand = int(w.graph.shape[1])
    with tempfile.TemporaryDirectory() as tmp:
        prefix = Path(tmp) / "index"
        B.write_pq_bundle(prefix, w.pq.codebook, w.pq.codes, w.pq.residual_rows(), w.pq.qparams,
                          w.pq.residual_bits, index_uuid=w.pq.meta.index_uuid)
        h = ref.pq_open(prefix, w.pq.residual_bits)
        pq = ref.pq_search(h, w.graph, w.entry, q, pools, EP, expand, correction=1, refine_budget=REFINE,
                           top_k=TOP_K, threads=os.cpu_count() or 1)
        ref.pq_close(h)
    hs = ref.sq_open(w.sq)
    sq = ref.sqmd_search(hs, w.graph, w.entry, q, 64, EP // 8, 32, correction=1, lanes=4,
                         threads=os.cpu_count() or 1, out_cap=REFINE)
    sq_ref = ref.refine(0, hs, q, sq["ids"], sq["dists"], np.minimum(sq["counts"], REFINE), TOP_K)
    ref.sq_close(hs)
    return dict(w=w, q=q, pools=pools, expand=expand, pq=pq, sq=sq, sq_ref=sq_ref)


def test_the_fixture_searches_the_graph(c5):
    st = c5["pq"]["stats"].astype(np.int64)
    assert st[:, 2].min() > 0 and np.all(c5["pq"]["counts"] == TOP_K)


@pytest.mark.parametrize("layout", [PACKED, DECODED])
def test_pq32_matches_compiled_reference(calc, c5, layout):
    w = c5["w"]
    calc.pq_load(w.graph, w.entry, w.pq)
    r = calc.pq_search(c5["q"], c5["pools"], top_k=TOP_K, pool_stride=256, entry_points=EP,
                       expand_count=c5["expand"], correction=1, refine_budget=REFINE, layout=layout)
    o = c5["pq"]
    rows_equal(r["pool_ids"], r["pool_dists"], r["pool_counts"], o["pool_ids"], o["pool_dists"], o["pool_counts"],
               f"layout {layout} pool")
    rows_equal(r["ids"], r["dists"], r["counts"], o["ids"], o["dists"], o["counts"], f"layout {layout} top-10")
    assert np.array_equal(r["stats"].astype(np.uint64), o["stats"])


def test_sq4_matches_compiled_reference(calc, c5):
    w = c5["w"]
    calc.sq_load(w.graph, w.entry, w.sq)
    r = calc.sq_search(c5["q"], 64, REFINE, sq_mode=1, num_out=REFINE, entry_points=EP // 8, expand_count=32,
                       correction=1)
    s = c5["sq"]
    rows_equal(r["ids"], r["dists"], r["counts"], s["ids"], s["dists"], s["counts"], "SQMD pool")
    ids, dists, counts = calc.refine(0, c5["q"], r["ids"], np.minimum(r["counts"], REFINE), TOP_K)
    oi, od, oc = c5["sq_ref"]
    rows_equal(ids, dists, counts, oi, od, oc, "refined")
    calc.sq_unload()
