"""The oracle's restatement of the final refine's ERROR4 mode and of the SQ4
split distance, pinned against the reference CLI's own outputs.

tests/golden/make_refine_artifacts.py wrote each fixture's ERROR4 artifact
(error4.refine) and the 4-bit SQ fixture's split-distance bias
(correction_bias.f32) with the reference's own tools, and
tests/golden/make_cli_golden.py recorded the reference CLI (oracle/_ref/
rover_ref, the unmodified reference host) with `--third-residual on` and
`--split-distance on`.  Here the oracle (oracle/rover_oracle.c) runs the same
pipeline -- the search, then retrieval_final_refine (retrieval_final_refine.c:
256-292) with decode_vector's ERROR4 term (:221-246), or the SQMD search with
sqmd_split_distance_for_id / the split pipeline's coarse + delta
(retrieval_rpc_demo_pipeline.c:909-995, retrieval_sqmd_common.c:1533-1556) --
and must print the reference's results.jsonl lines byte for byte.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, PQ_FIXTURES, SQ_FIXTURES, load_fixture


def _opt(args, name, default):
    return type(default)(args[args.index(name) + 1]) if name in args else default


def _lines(ids, dists):
    out = []
    for q, (i, d) in enumerate(zip(ids, dists)):
        out.append('{"query":%d,"ids":[%s],"distances":[%s]}' % (
            q, ",".join(str(int(x)) for x in i), ",".join(format(float(np.float32(x)), ".9g") for x in d)))
    return ("\n".join(out) + "\n").encode()


def _cases(names, tags):
    out = []
    for name in names:
        cases = json.loads((GOLDEN / name / "cli_cases.json").read_text())
        out += [(name, t) for t in tags if t in cases]
    return out


@pytest.mark.parametrize("name,tag", _cases(PQ_FIXTURES, ["third_residual"]))
def test_pq_error4_refine_matches_reference_cli(port, name, tag):
    data, graph, b, _, queries = load_fixture(name)
    args = json.loads((GOLDEN / name / "cli_cases.json").read_text())[tag]
    pool, ep, exp = _opt(args, "--pool", 0), _opt(args, "--entry-points", 0), _opt(args, "--expand-count", 0)
    k, factor, seed = _opt(args, "--top-k", 10), _opt(args, "--refine-factor", 2), _opt(args, "--seed", 42)
    entry = _opt(args, "--graph-entry", -1)
    ix = port.pq_index(graph, b)
    e4 = port.error4(GOLDEN / name / "error4.refine", data["n"], data["dim"])
    r = port.pq_search(ix, entry, queries, pool, ep, exp, correction=1, refine_budget=0, top_k=k, seed=seed)
    ids, dists = [], []
    for q in range(len(queries)):
        c = min(int(r["pool_counts"][q]), k * factor)
        i, d = port.refine_ex(1, ix, e4, queries[q], r["pool_ids"][q, :c], k)
        ids.append(i)
        dists.append(d)
    assert _lines(ids, dists) == (GOLDEN / name / f"cli_{tag}.jsonl").read_bytes()


@pytest.mark.parametrize("name,tag", _cases(SQ_FIXTURES, ["third_residual", "split_refine", "split_first_stage",
                                                          "split_third_residual"]))
def test_sq_error4_and_split_match_reference_cli(port, name, tag):
    from oracle.bindings import read_bias
    data, graph, b, _, queries = load_fixture(name)
    args = json.loads((GOLDEN / name / "cli_cases.json").read_text())[tag]
    pool, ep, exp = _opt(args, "--pool", 0), _opt(args, "--entry-points", 0), _opt(args, "--expand-count", 0)
    k, factor, seed = _opt(args, "--top-k", 10), _opt(args, "--refine-factor", 2), _opt(args, "--seed", 42)
    first = _opt(args, "--first-stage-factor", 3)
    entry = _opt(args, "--graph-entry", -1)
    refine = args[args.index("--refine") + 1] == "on"
    ix = port.sq_index(graph, b)
    e4 = port.error4(GOLDEN / name / "error4.refine", data["n"], data["dim"]) if "--third-residual" in args else None
    bias = read_bias(GOLDEN / name / "correction_bias.f32", data["n"]) if "--split-distance" in args else None
    cap = k * factor if refine else k * first
    ids, dists = [], []
    for q in range(len(queries)):
        if bias is not None:
            i, d, _ = port.sqmd_search_split(ix, bias, entry, queries[q], pool, ep, exp, seed=seed, out_cap=cap)
        else:
            i, d, _ = port.sqmd_search(ix, entry, queries[q], pool, ep, exp, correction=1, seed=seed, out_cap=cap)
        if refine:
            i, d = port.refine_ex(0, ix, e4, queries[q], i, k)
        elif bias is not None:
            # split first stage: demo_rerank_candidates over the candidates
            # (retrieval_rpc_demo_pipeline.c:3310-3320)
            i, d = port.sq_rerank(ix, queries[q], i, k)
        ids.append(i[:k])
        dists.append(d[:k])
    assert _lines(ids, dists) == (GOLDEN / name / f"cli_{tag}.jsonl").read_bytes()


def test_split_distance_parts_match_their_definition(port):
    """The split distance is the L2 distance to the L1 + residual
    reconstruction when the query sits on the 17-fold grid: check the
    restatement's parts against that identity in float64."""
    from oracle.bindings import read_bias
    name = "sq4_d24"
    data, graph, b, _, queries = load_fixture(name)
    ix = port.sq_index(graph, b)
    bias = read_bias(GOLDEN / name / "correction_bias.f32", data["n"])
    ids = np.arange(0, data["n"], 97)
    for q in queries[:4]:
        sq = port.split_query(ix, q)
        qs = np.float64(np.float32(b.l1_scale)) / 17.0
        qg = np.frombuffer(bytes(sq.q), dtype=np.uint8)[:data["dim"]].astype(np.float64) * qs + np.float64(
            np.float32(b.l1_zero))
        parts = port.split_parts(ix, bias, q, ids)
        for row, i in enumerate(ids):
            codes = np.array([(b.l1[i][d // 2] >> (4 * (d & 1))) & 15 for d in range(data["dim"])], np.float64)
            a = codes * np.float64(np.float32(b.l1_scale)) + np.float64(np.float32(b.l1_zero))
            rr = b.residual_rows[i]
            rc = np.array([(rr[d // 2] >> (4 * (d & 1))) & 15 for d in range(data["dim"])], np.float64) \
                if b.residual_bits == 4 else rr.astype(np.float64)
            r = rc * np.float64(b.qparams[i][0]) + np.float64(b.qparams[i][1])
            want = np.sum((qg - (a + r)) ** 2)
            assert abs(float(parts[row][2]) - want) <= 1e-3 * max(1.0, want), (i, parts[row], want)
