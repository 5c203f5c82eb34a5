"""The neighbourhood-aware layout (rover_b200/host/layout.cpp,
rover_layout_order) against the reference's own rover-layout tool
(src/graph/layout_opt_kmeans.cpp, compiled from the reference sources into
oracle/_ref/rover_layout by oracle/Makefile): the same order, id for id, on
the golden fixtures' graphs and on a mixture graph, across block sizes,
reverse-edge limits and the two affinity rankings, with graphs that carry
self loops, duplicate edges and short rows.  Also the permutation of a
workload: the same search in the new ids."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import PQ_FIXTURES, SQ_FIXTURES, load_fixture

ROOT = Path(__file__).resolve().parents[1]
TOOL = ROOT / "oracle" / "_ref" / "rover_layout"


def _reference(graph, labels, clusters, per_block, tmp, rrf_c=60.0, max_rev=1024, use_cn=1, use_mnn=1):
    if not TOOL.exists():
        pytest.skip("oracle/_ref/rover_layout was not built (reference sources absent at build time)")
    g, lab, out = tmp / "g.nsg", tmp / "labels.txt", tmp / "order.txt"
    with open(g, "wb") as f:       # NSG graph file: width, entry, then (k, ids) per row
        np.array([graph.shape[1], 0], np.uint32).tofile(f)
        for row in graph:
            r = row[:np.argmax(row < 0)] if np.any(row < 0) else row     # the valid prefix
            np.array([len(r)], np.uint32).tofile(f)
            r.astype(np.uint32).tofile(f)
    lab.write_text(" ".join(str(int(x)) for x in labels))
    p = subprocess.run([str(TOOL), str(g), str(lab), str(out), str(clusters), str(per_block), repr(rrf_c),
                        str(max_rev), "1", str(use_cn), str(use_mnn)], capture_output=True, timeout=600)
    assert p.returncode == 0, p.stderr.decode()[-2000:]
    return np.array(out.read_text().split(), dtype=np.int32)


def _labels(base, clusters, seed=0):
    rng = np.random.default_rng(seed)
    cent = base[rng.choice(len(base), clusters, replace=False)]
    d = ((base[:, None, :] - cent[None, :, :]) ** 2).sum(2)
    return np.argmin(d, axis=1).astype(np.int32)


@pytest.mark.parametrize("name", PQ_FIXTURES + SQ_FIXTURES)
@pytest.mark.parametrize("per_block,clusters", [(32, 8), (21, 16), (128, 4)])
def test_layout_matches_the_reference_tool(name, per_block, clusters, tmp_path):
    from rover_b200 import datasets as D
    from rover_b200.layout import gorder
    data, graph, b, _, _ = load_fixture(name)
    # labels: nearest of `clusters` centres over vectors of the fixture's shape
    labels = _labels(D.gmm(data["n"], data["dim"], 16, 11), clusters)
    ours = gorder(graph, labels, clusters, per_block, threads=4)
    want = _reference(graph, labels, clusters, per_block, tmp_path)
    assert np.array_equal(ours, want)
    assert np.array_equal(np.sort(ours), np.arange(len(graph)))


@pytest.mark.parametrize("max_rev,use_cn,use_mnn,rrf_c", [(3, 1, 1, 60.0), (0, 1, 0, 10.0), (1024, 0, 1, 1.0)])
def test_layout_options_match_the_reference_tool(max_rev, use_cn, use_mnn, rrf_c, tmp_path):
    from rover_b200.layout import gorder
    data, graph, _, _, _ = load_fixture("pq8_d64")
    labels = (np.arange(len(graph)) * 7 % 5).astype(np.int32)
    ours = gorder(graph, labels, 5, 24, rrf_c=rrf_c, max_reverse=max_rev, use_cn=bool(use_cn), use_mnn=bool(use_mnn))
    want = _reference(graph, labels, 5, 24, tmp_path, rrf_c=rrf_c, max_rev=max_rev, use_cn=use_cn, use_mnn=use_mnn)
    assert np.array_equal(ours, want)


def test_layout_of_irregular_rows_matches_the_reference_tool(tmp_path):
    """Self loops, duplicate edges and short (-1 padded) rows."""
    from rover_b200.layout import gorder
    rng = np.random.default_rng(4)
    n, deg = 600, 12
    graph = rng.integers(0, n, size=(n, deg)).astype(np.int32)
    graph[::7, 3] = np.arange(0, n, 7)          # self loops
    graph[::5, 6] = graph[::5, 5]               # duplicates
    short = rng.integers(1, deg, size=n)
    for i in range(0, n, 3):
        graph[i, short[i]:] = -1
    labels = rng.integers(0, 6, size=n).astype(np.int32)
    ours = gorder(graph, labels, 6, 16)
    want = _reference(graph, labels, 6, 16, tmp_path)
    assert np.array_equal(ours, want)


def test_permuted_workload_is_the_same_index(tmp_path):
    """Renumbering ids keeps every vector's codes, residuals and edges."""
    from rover_b200.layout import gorder, permute_pq
    from rover_b200.workloads import PqWorkload
    data, graph, b, _, _ = load_fixture("pq8_d64")
    w = PqWorkload("pq8_d64", (data["n"], data["dim"]), np.zeros((1, data["dim"]), np.float32),
                   np.zeros((1, 10), np.int32), graph, data["graph_entry"], b)
    labels = (np.arange(len(graph)) % 9).astype(np.int32)
    n2o = gorder(graph, labels, 9, 32)
    p, _ = permute_pq(w, n2o)
    assert np.array_equal(p.bundle.codes, b.codes[n2o])
    assert np.array_equal(p.bundle.residual_rows(), b.residual_rows()[n2o])
    assert np.array_equal(p.bundle.qparams, b.qparams[n2o])
    o2n = np.argsort(n2o)
    assert p.entry == o2n[data["graph_entry"]]
    back = np.where(p.graph >= 0, n2o[np.maximum(p.graph, 0)], -1)
    assert np.array_equal(back, graph[n2o])


def test_permuted_large_workload_moves_both_bundles():
    """The large combined workload renumbered: the PQ and SQ rows, the
    graph, the ground truth and the entry move together."""
    from rover_b200 import bundle as B
    from rover_b200 import datasets as D
    from rover_b200.layout import gorder_large
    from rover_b200.workloads import LargeWorkload
    data, graph, pq, _, _ = load_fixture("pq8_d64")
    n, dim = data["n"], data["dim"]
    base = D.gmm(n, dim, 8, 3)
    scale, zero, l1, res, qp = D.sq_encode(base, 4, 8)
    sq = B.SqBundle(n, dim, 4, scale, zero, l1, 8, res, qp)
    labels = (np.arange(n) * 5 % 7).astype(np.int32)
    gt = np.random.default_rng(1).integers(-1, n, size=(6, 100)).astype(np.int32)
    w = LargeWorkload("t", np.zeros((6, dim), np.float32), gt, graph, data["graph_entry"], pq, sq, 0.0, labels)
    p, n2o = gorder_large(w, per_block=16, threads=2)
    assert np.array_equal(np.sort(n2o), np.arange(n))
    assert p.labels is None
    assert np.array_equal(p.pq.codes, pq.codes[n2o])
    assert np.array_equal(p.pq.residual_rows(), pq.residual_rows()[n2o])
    assert np.array_equal(p.sq.l1, sq.l1[n2o])
    assert np.array_equal(p.sq.residual_rows, sq.residual_rows[n2o])
    assert np.array_equal(p.sq.qparams, sq.qparams[n2o])
    o2n = np.argsort(n2o)
    assert p.entry == o2n[data["graph_entry"]]
    assert np.array_equal(np.where(p.gt >= 0, n2o[np.maximum(p.gt, 0)], -1), gt)
    back = np.where(p.graph >= 0, n2o[np.maximum(p.graph, 0)], -1)
    assert np.array_equal(back, graph[n2o])
