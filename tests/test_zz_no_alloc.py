"""calculator_rover_pq_search_noalloc: the batched PQ search for callers that
cannot allocate device memory while searching (a server whose memory pool
already owns the GPU, or a loop that must not synchronize on cudaMalloc).
Its scratch lives in a fixed device array inside the library.  This test
calls it through the C-ABI twice in a row and checks each result against the
allocating entry point, calculator_rover_pq_search_device, bit for bit.

The file is named so that pytest collects it last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def _device_outputs(torch, nq, k, pool_stride):
    dev = torch.device("cuda", 0)
    return dict(
        ids=torch.full((nq, k), -1, dtype=torch.int32, device=dev),
        dists=torch.zeros((nq, k), dtype=torch.float32, device=dev),
        counts=torch.zeros(nq, dtype=torch.int32, device=dev),
        pool_ids=torch.full((nq, pool_stride), -1, dtype=torch.int32, device=dev),
        pool_dists=torch.zeros((nq, pool_stride), dtype=torch.float32, device=dev),
        pool_counts=torch.zeros(nq, dtype=torch.int32, device=dev),
        stats=torch.zeros((nq, 4), dtype=torch.int64, device=dev),
        status=torch.full((nq,), 99, dtype=torch.int32, device=dev),
    )


def _ptrs(calc_mod, o, k):
    P = lambda t, ty: C.cast(C.c_void_p(t.data_ptr()), ty)
    return calc_mod.SearchOutputs(P(o["ids"], calc_mod._i32p), P(o["dists"], calc_mod._f32p),
                                  P(o["counts"], calc_mod._i32p), k, P(o["pool_ids"], calc_mod._i32p),
                                  P(o["pool_dists"], calc_mod._f32p), P(o["pool_counts"], calc_mod._i32p),
                                  P(o["stats"], calc_mod._u64p), P(o["status"], calc_mod._i32p))


def test_noalloc_matches_allocating_search_twice():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200 import calculator as cm

    calc = cm.Calculator()
    lib = calc.lib
    lib.calculator_rover_pq_search_noalloc.argtypes = [C.c_uint64, C.POINTER(cm.SearchParams), cm._f32p,
                                                       C.c_int32, cm._i32p, C.c_int32, cm._i32p,
                                                       C.POINTER(cm.SearchOutputs), C.c_void_p]
    data, graph, bundle, golden, queries = load_fixture("pq8_d64")
    calc.pq_load(graph, data["graph_entry"], bundle)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    nq, k, stride = len(queries), 10, 64
    q = torch.from_numpy(np.ascontiguousarray(queries)).to(dev)
    # two calls in a row with different beam widths: the second reuses the
    # array the first one left behind
    for call, pools_np in enumerate((golden["pool_sizes"], np.full(nq, 48, np.int32))):
        pools = torch.from_numpy(np.ascontiguousarray(pools_np, dtype=np.int32)).to(dev)
        params = calc.params(entry_points=4, expand_count=16, correction=1, refine_budget=20, top_k=k,
                             pool_stride=stride)
        ref_out = _device_outputs(torch, nq, k, stride)
        rc = lib.calculator_rover_pq_search_device(calc.handle, C.byref(params),
                                                   C.cast(C.c_void_p(q.data_ptr()), cm._f32p), nq,
                                                   C.cast(C.c_void_p(pools.data_ptr()), cm._i32p), None,
                                                   C.byref(_ptrs(cm, ref_out, k)), C.c_void_p(stream.cuda_stream))
        assert rc == 0, calc.last_error()
        new_out = _device_outputs(torch, nq, k, stride)
        rc = lib.calculator_rover_pq_search_noalloc(calc.handle, C.byref(params),
                                                    C.cast(C.c_void_p(q.data_ptr()), cm._f32p), nq,
                                                    C.cast(C.c_void_p(pools.data_ptr()), cm._i32p),
                                                    int(pools_np.max()), None, C.byref(_ptrs(cm, new_out, k)),
                                                    C.c_void_p(stream.cuda_stream))
        assert rc == 0, calc.last_error()
        torch.cuda.synchronize()
        assert torch.equal(new_out["status"], torch.zeros_like(new_out["status"])), f"call {call}"
        for key in ("counts", "pool_counts", "stats"):
            assert torch.equal(new_out[key], ref_out[key]), f"call {call}: {key}"
        for key in ("ids", "pool_ids"):
            assert torch.equal(new_out[key], ref_out[key]), f"call {call}: {key}"
        for key in ("dists", "pool_dists"):
            assert torch.equal(new_out[key].view(torch.int32), ref_out[key].view(torch.int32)), f"call {call}: {key}"


def test_noalloc_rejects_requests_beyond_its_scratch():
    """A request whose visited tables cannot fit the fixed array is refused
    before anything is launched."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200 import bundle as B
    from rover_b200 import calculator as cm

    calc = cm.Calculator()
    lib = calc.lib
    lib.calculator_rover_pq_search_noalloc.argtypes = [C.c_uint64, C.POINTER(cm.SearchParams), cm._f32p,
                                                       C.c_int32, cm._i32p, C.c_int32, cm._i32p,
                                                       C.POINTER(cm.SearchOutputs), C.c_void_p]
    # a tiny index whose rows are 128 wide (one edge each, -1 padded)
    n, dim, m = 300, 8, 2
    rng = np.random.default_rng(0)
    graph = np.full((n, 128), -1, np.int32)
    graph[:, 0] = (np.arange(n) + 1) % n
    book = rng.normal(size=(m, 16, dim // m)).astype(np.float32)
    codes = rng.integers(0, 256, size=(n, 1)).astype(np.uint8)
    rows = rng.integers(0, 256, size=(n, dim)).astype(np.uint8)
    qp = np.tile(np.array([[0.01, -1.0]], np.float32), (n, 1))
    bundle = B.PqBundle(B.PqMeta(b"\x03" * 16, n, dim, m, 16, dim // m, 1), book, codes, 8,
                        B.pack_residual_blocks(rows), qp)
    calc.pq_load(graph, 0, bundle)
    dev = torch.device("cuda", 0)
    q = torch.zeros((4, dim), dtype=torch.float32, device=dev)
    pools = torch.full((4,), 4096, dtype=torch.int32, device=dev)
    out = _device_outputs(torch, 4, 10, 64)
    # beam 4096 x 128 neighbours per expansion needs a 32 MiB table per warp
    params = calc.params(entry_points=n, expand_count=128, correction=1, refine_budget=0, top_k=10,
                         pool_stride=64)
    rc = lib.calculator_rover_pq_search_noalloc(calc.handle, C.byref(params),
                                                C.cast(C.c_void_p(q.data_ptr()), cm._f32p), 4,
                                                C.cast(C.c_void_p(pools.data_ptr()), cm._i32p), 4096, None,
                                                C.byref(_ptrs(cm, out, 10)), None)
    assert rc == 14  # AEE_EBADPARM
    assert "no-alloc scratch" in calc.last_error()


def _noalloc(lib, cm):
    lib.calculator_rover_pq_search_noalloc.argtypes = [C.c_uint64, C.POINTER(cm.SearchParams), cm._f32p,
                                                       C.c_int32, cm._i32p, C.c_int32, cm._i32p,
                                                       C.POINTER(cm.SearchOutputs), C.c_void_p]
    return lib.calculator_rover_pq_search_noalloc


def _chain_index(n=5000):
    """A path graph 0 -> 1 -> ... -> n-1 whose ADC distances to the zero
    query fall strictly along the path: a search with a one-entry pool walks
    the whole chain, claiming one new id per expansion."""
    from rover_b200 import bundle as B
    m, ks, sub = 2, 256, 4
    graph = np.full((n, 1), -1, np.int32)
    graph[:-1, 0] = np.arange(1, n, dtype=np.int32)
    book = np.zeros((m, ks, sub), np.float32)
    book[0] = np.sqrt(250.0 * np.arange(ks, dtype=np.float64))[:, None].astype(np.float32)   # LUT0 ~ 1000 k
    book[1] = np.sqrt(np.arange(ks, dtype=np.float64) / 4.0)[:, None].astype(np.float32)     # LUT1 ~ k
    v = (n - 1 - np.arange(n)).astype(np.int64)
    codes = np.stack([v // 256, v % 256], axis=1).astype(np.uint8)
    rows = np.zeros((n, m * sub), np.uint8)
    qp = np.tile(np.array([[0.01, 0.0]], np.float32), (n, 1))
    return graph, B.PqBundle(B.PqMeta(b"\x05" * 16, n, m * sub, m, ks, sub, m), book, codes, 8,
                             B.pack_residual_blocks(rows), qp)


def test_noalloc_table_overflow_fails_the_call():
    """A query that claims more ids than its visited table's load limit
    (half of 4,096 entries here) fails the call with AEE_EFAILED and the
    overflow message; the query's status says which one, and the scratch is
    fit for the next call."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200 import calculator as cm

    calc = cm.Calculator()
    fn = _noalloc(calc.lib, cm)
    graph, bundle = _chain_index()
    calc.pq_load(graph, 0, bundle)
    dev = torch.device("cuda", 0)
    nq = 2
    q = torch.zeros((nq, 8), dtype=torch.float32, device=dev)
    pools = torch.ones(nq, dtype=torch.int32, device=dev)
    out = _device_outputs(torch, nq, 1, 1)
    params = calc.params(entry_points=1, expand_count=1, correction=0, refine_budget=0, top_k=1, pool_stride=1)
    rc = fn(calc.handle, C.byref(params), C.cast(C.c_void_p(q.data_ptr()), cm._f32p), nq,
            C.cast(C.c_void_p(pools.data_ptr()), cm._i32p), 1, None, C.byref(_ptrs(cm, out, 1)), None)
    torch.cuda.synchronize()
    assert rc == 1, calc.last_error()   # AEE_EFAILED
    assert "exceeded its visited table" in calc.last_error()
    assert torch.equal(out["status"].cpu(), torch.full((nq,), 3, dtype=torch.int32))   # ROVER_QUERY_TABLE_FULL
    # the allocating entry retries with a larger table and walks the chain to its end
    r = calc.pq_search(np.zeros((1, 8), np.float32), 1, top_k=1, entry_points=1, expand_count=1, correction=0,
                       refine_budget=0)
    assert int(r["ids"][0, 0]) == graph.shape[0] - 1
    # a request the table holds succeeds on the same scratch afterwards
    pools_ok = torch.ones(nq, dtype=torch.int32, device=dev)
    out2 = _device_outputs(torch, nq, 1, 1)
    short = np.full((graph.shape[0], 1), -1, np.int32)
    short[:100, 0] = np.arange(1, 101)
    calc.pq_load(short, 0, bundle)
    rc = fn(calc.handle, C.byref(params), C.cast(C.c_void_p(q.data_ptr()), cm._f32p), nq,
            C.cast(C.c_void_p(pools_ok.data_ptr()), cm._i32p), 1, None, C.byref(_ptrs(cm, out2, 1)), None)
    torch.cuda.synchronize()
    assert rc == 0, calc.last_error()
    assert torch.equal(out2["ids"][:, 0].cpu(), torch.full((nq,), 100, dtype=torch.int32))


def test_noalloc_refuses_modes_it_does_not_run():
    """The no-alloc entry runs the exact search over packed rows: a batched,
    gated or decoded-layout request is refused, not silently run otherwise."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rover_b200 import calculator as cm

    calc = cm.Calculator()
    fn = _noalloc(calc.lib, cm)
    data, graph, bundle, golden, queries = load_fixture("pq8_d64")
    calc.pq_load(graph, data["graph_entry"], bundle)
    dev = torch.device("cuda", 0)
    nq = 4
    q = torch.from_numpy(np.ascontiguousarray(queries[:nq])).to(dev)
    pools = torch.full((nq,), 32, dtype=torch.int32, device=dev)
    for kw in (dict(mode=1), dict(mode=2), dict(layout=2)):
        out = _device_outputs(torch, nq, 10, 32)
        params = calc.params(entry_points=4, expand_count=16, correction=1, refine_budget=20, top_k=10,
                             pool_stride=32, **kw)
        rc = fn(calc.handle, C.byref(params), C.cast(C.c_void_p(q.data_ptr()), cm._f32p), nq,
                C.cast(C.c_void_p(pools.data_ptr()), cm._i32p), 32, None, C.byref(_ptrs(cm, out, 10)), None)
        assert rc == 14, kw   # AEE_EBADPARM
        assert "ROVER_MODE_EXACT" in calc.last_error()
