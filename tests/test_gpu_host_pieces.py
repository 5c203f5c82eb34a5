"""Host-buffer searches of large batches upload their queries in pieces on a
copy stream and rank each piece's seeds as soon as it has arrived; their
results are fetched with the status into page-locked staging.  The results
must be those of the device-buffer entry point on the same queries, bit for
bit, in every form that reaches the seed ranking (exact on decoded rows,
batched) and on packed rows (which wait for the whole upload)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOP_K = 10


@pytest.fixture(scope="module")
def big():
    import torch  # noqa: F401
    from rover_b200 import workloads
    w = workloads.build_pq("pq_100k_d128", verbose=False)
    rng = np.random.default_rng(5)
    base = np.tile(w.queries, (int(np.ceil(3000 / len(w.queries))), 1))[:3000]
    q = (base + rng.normal(0, 0.05, size=base.shape)).astype(np.float32)
    return w, np.ascontiguousarray(q)


def _device(calc, q, pool, kw):
    import torch
    dev = torch.device("cuda", 0)
    nq = len(q)
    qd = torch.from_numpy(q).to(dev)
    pd = torch.full((nq,), pool, dtype=torch.int32, device=dev)
    out = dict(ids=torch.empty((nq, TOP_K), dtype=torch.int32, device=dev),
               dists=torch.empty((nq, TOP_K), dtype=torch.float32, device=dev),
               counts=torch.empty(nq, dtype=torch.int32, device=dev),
               stats=torch.empty((nq, 4), dtype=torch.int64, device=dev),
               status=torch.empty(nq, dtype=torch.int32, device=dev))
    ptrs = {k: v.data_ptr() for k, v in out.items()}
    ptrs["stride"] = TOP_K
    calc.pq_search_device(qd.data_ptr(), nq, pd.data_ptr(), ptrs, top_k=TOP_K, **kw)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("form", ["decoded", "packed", "batched"])
def test_piecewise_upload_matches_device_entry(calc, big, form):
    from rover_b200.calculator import MODE_BATCHED
    w, q = big
    calc.pq_load(w.graph, w.entry, w.bundle)
    kw = dict(entry_points=2048, expand_count=int(w.graph.shape[1]), correction=1, refine_budget=20)
    if form == "decoded":
        kw.update(layout=2)
    elif form == "packed":
        kw.update(layout=1)
    else:
        kw.update(mode=MODE_BATCHED, beam_width=3)
    pool = 32
    h = calc.pq_search(q, pool, top_k=TOP_K, **kw)
    d = _device(calc, q, pool, kw)
    assert np.array_equal(h["status"], d["status"]) and not h["status"].any()
    assert np.array_equal(h["counts"], d["counts"])
    assert np.array_equal(h["ids"], d["ids"])
    assert np.array_equal(h["dists"].view(np.uint32), d["dists"].view(np.uint32))
    assert np.array_equal(h["stats"].astype(np.int64), d["stats"])


def test_results_into_page_locked_buffers(calc, big):
    """Page-locked result arrays passed back in (out=) receive the copies
    directly; the results equal those of a call with fresh pageable arrays,
    on two calls in a row."""
    import torch
    w, q = big
    calc.pq_load(w.graph, w.entry, w.bundle)
    kw = dict(entry_points=2048, expand_count=int(w.graph.shape[1]), correction=1, refine_budget=20)
    nq = len(q)
    want = calc.pq_search(q, 32, top_k=TOP_K, stats=False, **kw)
    out = {k: torch.empty(shape, dtype=dt).pin_memory().numpy() for k, shape, dt in
           (("ids", (nq, TOP_K), torch.int32), ("dists", (nq, TOP_K), torch.float32),
            ("counts", (nq,), torch.int32), ("status", (nq,), torch.int32))}
    out["ids"][:] = -1                      # as a fresh result's rows past its count
    out["dists"][:] = 0.0
    for _ in range(2):
        got = calc.pq_search(q, np.full(nq, 32, np.int32), top_k=TOP_K, stats=False, out=out, **kw)
        assert got["ids"] is out["ids"]
        for k in ("counts", "ids", "status"):
            assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(got["dists"].view(np.uint32), want["dists"].view(np.uint32))
