"""Parity at the benchmark's own index: the 1M x 128 workload bench.py
searches (pq_1m_d128, 4,096 entry points, expand 48, refine 20, top-10),
in the clustered block order and as built, against the compiled reference
(oracle/_ref: retrieval_pure_pq_search_scalar_with_policy, sqmd_pure_pq.c:793,
with the ONLINE residual policy and retrieval_final_refine) on held-out
queries.  Ids, distance bits and the search statistics must be equal."""
from __future__ import annotations

import os
import tempfile
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QUERIES = 500


@pytest.fixture(scope="module")
def indexes():
    import torch  # noqa: F401
    from oracle import bindings
    from rover_b200 import workloads
    from rover_b200.layout import gorder_workload
    if not bindings.reference_available():
        pytest.skip("oracle/_ref was not built (reference sources absent at build time)")
    w = workloads.build_pq("pq_1m_d128", cache_dir=os.environ.get("ROVER_BENCH_CACHE", "/tmp/rover_bench_cache"),
                           verbose=False)
    wg, _ = gorder_workload(w)
    q, _ = workloads.held_out_set("pq_1m_d128", 2000, 13, cache_dir=os.environ.get("ROVER_BENCH_CACHE",
                                                                                   "/tmp/rover_bench_cache"))
    return dict(original=w, gorder=wg), np.ascontiguousarray(q[:QUERIES])


@pytest.mark.parametrize("layout", ["gorder", "original"])
@pytest.mark.parametrize("L", [40, 48])
def test_benchmark_index_matches_compiled_reference(calc, indexes, layout, L):
    from oracle import bindings
    from rover_b200 import bundle as B
    ws, q = indexes
    w = ws[layout]
    kw = dict(entry_points=4096, expand_count=int(w.graph.shape[1]), correction=1, refine_budget=20)
    calc.pq_load(w.graph, w.entry, w.bundle)
    ours = calc.pq_search(q, L, top_k=10, **kw)
    ref = bindings.Reference()
    with tempfile.TemporaryDirectory() as tmp:
        prefix = Path(tmp) / "index"
        B.write_pq_bundle(prefix, w.bundle.codebook, w.bundle.codes, w.bundle.residual_rows(), w.bundle.qparams,
                          w.bundle.residual_bits, index_uuid=w.bundle.meta.index_uuid)
        h = ref.pq_open(prefix, w.bundle.residual_bits)
        r = ref.pq_search(h, w.graph, w.entry, q, L, kw["entry_points"], kw["expand_count"], correction=1,
                          refine_budget=20, top_k=10, threads=os.cpu_count() or 1)
        ref.pq_close(h)
    assert np.array_equal(ours["counts"], r["counts"])
    assert np.array_equal(ours["ids"], r["ids"])
    assert np.array_equal(ours["dists"].view(np.uint32), r["dists"].view(np.uint32))
    assert np.array_equal(ours["stats"].astype(np.uint64), r["stats"].astype(np.uint64))
