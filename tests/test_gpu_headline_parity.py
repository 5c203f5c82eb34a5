"""Parity at the benchmark's shapes against the compiled reference
(oracle/_ref, the unmodified reference sources built by oracle/Makefile).

* PQ, the 1M x 128 headline shape at 100K vectors: d=128, M=16 x 256, 8-bit
  residuals, a degree-48 graph from the benchmark's own graph builder, 4,096
  entry points, beam widths 32 / 48 / 64 / 128 / 256 mixed in one batch.  The
  reference runs retrieval_pure_pq_search_scalar_with_policy
  (retrieval_sqmd_pure_pq.c:793) with the ONLINE residual policy
  (retrieval_pq_residual.c:983) and retrieval_final_refine
  (retrieval_final_refine.c:294); the library's exact mode must return the
  same pools, statistics, ids and distances bit for bit, on both residual
  layouts, through the host-buffer and the device-buffer entry points, and
  its batched kernel at beam width 1 must too.
* SQ, the 20K x 128 SQ8 shape (exact 32-NN graph, L=64, expand 32, exact
  residual correction, top-20 refined to 10): the SQMD search
  (sqmd_cpu_state_run_fake_dsp, retrieval_sqmd_common.c:2052) plus the final
  refine, against calculator_rover_sq_search + calculator_rover_refine.
"""
from __future__ import annotations

import os
import tempfile
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PACKED, DECODED = 1, 2
L_SET = (32, 48, 64, 128, 256)
PQ_QUERIES = 400
ENTRY_POINTS = 4096
TOP_K, REFINE = 10, 20


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def rows_equal(ids, dists, counts, g_ids, g_dists, g_counts, what):
    assert np.array_equal(counts, g_counts), f"{what}: counts"
    for i, c in enumerate(counts):
        assert np.array_equal(ids[i, :c], g_ids[i, :c]), f"{what}: ids row {i}"
        assert np.array_equal(bits(dists[i, :c]), bits(g_dists[i, :c])), f"{what}: dists row {i}"


def _reference():
    from oracle import bindings
    if not bindings.reference_available():
        pytest.skip("oracle/_ref was not built (reference sources absent at build time)")
    return bindings.Reference()


@pytest.fixture(scope="module")
def c2():
    """The 100K x 128 workload (pq_100k_d128: 256-component mixture clipped
    to >= 0, 64-NN alpha=1.2 pruned to degree 48 plus long-range edges) and
    the reference's own results for it."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200 import bundle as B
    from rover_b200 import workloads
    ref = _reference()
    w = workloads.build_pq("pq_100k_d128", nq=PQ_QUERIES, verbose=False)
    pools = np.random.default_rng(11).choice(L_SET, size=PQ_QUERIES).astype(np.int32)
    expand = int(w.graph.shape[1])
    with tempfile.TemporaryDirectory() as tmp:
        prefix = Path(tmp) / "index"
        B.write_pq_bundle(prefix, w.bundle.codebook, w.bundle.codes, w.bundle.residual_rows(), w.bundle.qparams,
                          w.bundle.residual_bits, index_uuid=w.bundle.meta.index_uuid)
        h = ref.pq_open(prefix, w.bundle.residual_bits)
        o = ref.pq_search(h, w.graph, w.entry, w.queries, pools, ENTRY_POINTS, expand, correction=1,
                          refine_budget=REFINE, top_k=TOP_K, threads=os.cpu_count() or 1)
        ref.pq_close(h)
    return dict(w=w, pools=pools, expand=expand, ref=o)


def _check_against_reference(r, c2, what):
    o = c2["ref"]
    rows_equal(r["pool_ids"], r["pool_dists"], r["pool_counts"], o["pool_ids"], o["pool_dists"],
               o["pool_counts"], what + " pool")
    rows_equal(r["ids"], r["dists"], r["counts"], o["ids"], o["dists"], o["counts"], what + " top-10")
    assert np.array_equal(r["stats"].astype(np.uint64), o["stats"]), what + ": statistics"


def test_headline_workload_reaches_the_graph(c2):
    """The fixture is a real graph search: every beam width expands nodes
    beyond the entry seeds, and the widest pools expand the most."""
    st = c2["ref"]["stats"].astype(np.int64)
    pools = c2["pools"]
    assert st[:, 2].min() > 0
    assert st[pools == 256, 2].mean() > st[pools == 32, 2].mean()


@pytest.mark.parametrize("layout", [PACKED, DECODED])
def test_pq_headline_shape_matches_compiled_reference(calc, c2, layout):
    w = c2["w"]
    calc.pq_load(w.graph, w.entry, w.bundle)
    r = calc.pq_search(w.queries, c2["pools"], top_k=TOP_K, pool_stride=max(L_SET), entry_points=ENTRY_POINTS,
                       expand_count=c2["expand"], correction=1, refine_budget=REFINE, layout=layout)
    _check_against_reference(r, c2, f"layout {layout}")


def test_pq_headline_shape_device_entry_matches_compiled_reference(calc, c2):
    import torch
    w = c2["w"]
    calc.pq_load(w.graph, w.entry, w.bundle)
    dev = torch.device("cuda", 0)
    nq, stride = PQ_QUERIES, max(L_SET)
    q = torch.from_numpy(np.ascontiguousarray(w.queries)).to(dev)
    pools = torch.from_numpy(c2["pools"]).to(dev)
    out = dict(ids=torch.empty((nq, TOP_K), dtype=torch.int32, device=dev),
               dists=torch.empty((nq, TOP_K), dtype=torch.float32, device=dev),
               counts=torch.empty(nq, dtype=torch.int32, device=dev),
               pool_ids=torch.empty((nq, stride), dtype=torch.int32, device=dev),
               pool_dists=torch.empty((nq, stride), dtype=torch.float32, device=dev),
               pool_counts=torch.empty(nq, dtype=torch.int32, device=dev),
               stats=torch.empty((nq, 4), dtype=torch.int64, device=dev),
               status=torch.empty(nq, dtype=torch.int32, device=dev))
    ptrs = {k: v.data_ptr() for k, v in out.items()}
    ptrs["stride"] = TOP_K
    calc.pq_search_device(q.data_ptr(), nq, pools.data_ptr(), ptrs, top_k=TOP_K, pool_stride=stride,
                          entry_points=ENTRY_POINTS, expand_count=c2["expand"], correction=1, refine_budget=REFINE)
    torch.cuda.synchronize()
    r = {k: v.cpu().numpy() for k, v in out.items()}
    assert np.all(r["status"] == 0)
    _check_against_reference(r, c2, "device entry")


def test_pq_headline_shape_batched_width_one_is_the_reference_order(calc, c2):
    """ROVER_MODE_BATCHED with one entry expanded per step is the
    reference's expansion order: the same results bit for bit."""
    w = c2["w"]
    calc.pq_load(w.graph, w.entry, w.bundle)
    r = calc.pq_search(w.queries, c2["pools"], top_k=TOP_K, pool_stride=max(L_SET), entry_points=ENTRY_POINTS,
                       expand_count=c2["expand"], correction=1, refine_budget=REFINE, mode=1, beam_width=1)
    _check_against_reference(r, c2, "batched W=1")


SQ_L, SQ_EXPAND, SQ_EPS = 64, 32, (1, 256)


@pytest.fixture(scope="module")
def c1():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200 import workloads
    ref = _reference()
    w = workloads.build_sq("sq_20k_d128")
    hs = ref.sq_open(w.bundle)
    out = {}
    for ep in SQ_EPS:
        rr = ref.sqmd_search(hs, w.graph, w.entry, w.queries, SQ_L, ep, SQ_EXPAND, correction=1, lanes=4,
                             threads=os.cpu_count() or 1, out_cap=REFINE)
        oi, od, oc = ref.refine(0, hs, w.queries, rr["ids"], rr["dists"], np.minimum(rr["counts"], REFINE), TOP_K)
        out[ep] = dict(search=rr, ids=oi, dists=od, counts=oc)
    ref.sq_close(hs)
    return dict(w=w, ref=out)


@pytest.mark.parametrize("ep", SQ_EPS)
def test_sq_small_shape_matches_compiled_reference(calc, c1, ep):
    """20K x 128 SQ8: the SQMD pool (first 20 entries) and the refined top-10."""
    w, o = c1["w"], c1["ref"][ep]
    calc.sq_load(w.graph, w.entry, w.bundle)
    r = calc.sq_search(w.queries, SQ_L, REFINE, sq_mode=1, num_out=REFINE, entry_points=ep,
                       expand_count=SQ_EXPAND, correction=1)
    s = o["search"]
    rows_equal(r["ids"], r["dists"], r["counts"], s["ids"], s["dists"], s["counts"], f"ep {ep} SQMD pool")
    ids, dists, counts = calc.refine(0, w.queries, r["ids"], np.minimum(r["counts"], REFINE), TOP_K)
    rows_equal(ids, dists, counts, o["ids"], o["dists"], o["counts"], f"ep {ep} refined")
    calc.sq_unload()
