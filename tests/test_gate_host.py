"""Host-side gate analysis on the CPU: rover_b200.gate.stop_savings on a
hand-made trace whose savings and losses are known."""
from __future__ import annotations

import numpy as np

from rover_b200 import gate as G
from rover_b200.calculator import TRACE_DTYPE


def _trace():
    rows = []

    def add(q, hop, id_, flags):
        r = np.zeros(1, TRACE_DTYPE)
        r["query"], r["hop"], r["id"], r["flags"] = q, hop, id_, flags
        rows.append(r)
    # query 0: results 100 (an entry seed), 5 (scored at hop 0), 7 (hop 2); four expansions
    add(0, 0, 100, G.SEED | G.ENTERED)
    add(0, 0, 101, G.SEED)
    for h in range(4):
        add(0, h, 50 + h, G.SOURCE)
    add(0, 0, 5, G.ENTERED)
    add(0, 2, 7, G.ENTERED)
    add(0, 1, 9, 0)
    # query 1: every result is an entry seed; two expansions
    for i in (200, 201, 202):
        add(1, 0, i, G.SEED | G.ENTERED)
    for h in range(2):
        add(1, h, 60 + h, G.SOURCE)
    rows = np.concatenate(rows)
    rows = rows[np.random.default_rng(0).permutation(len(rows))]     # trace order is arbitrary
    ids = np.array([[100, 5, 7], [200, 201, 202]], np.int32)
    counts = np.array([3, 3], np.int32)
    return rows, ids, counts


def test_stop_savings_by_hand():
    rows, ids, counts = _trace()
    src = rows[(rows["flags"] & G.SOURCE) != 0]
    scores = {"hop": src["hop"].astype(np.float64), "never": np.zeros(len(src))}
    res = G.stop_savings(rows, ids, counts, scores, top_k=3, budgets=(0.0, 0.2, 0.5))
    # lossless: only query 0's last expansion (hop 3) can go -> 1 of 6
    assert abs(res["hop"]["0.0"]["saved"] - 1 / 6) < 1e-12
    assert 2 <= res["hop"]["0.0"]["threshold"] < 3
    # losing result 7 of query 0 (1 of 6 results) allows stopping both
    # queries before hop 1 -> 4 of 6
    assert abs(res["hop"]["0.2"]["saved"] - 4 / 6) < 1e-12
    assert 0 <= res["hop"]["0.2"]["threshold"] < 1
    assert abs(res["hop"]["0.5"]["saved"] - 4 / 6) < 1e-12      # a threshold never fires at hop 0 (s > t)
    assert all(v["saved"] == 0.0 for v in res["never"].values())


def test_labels_agree_with_savings():
    """A source labelled stop-safe (labels) is exactly one whose stop loses nothing."""
    rows, ids, counts = _trace()
    y, m = G.labels(rows, ids, counts, 3)
    src = (rows["flags"] & G.SOURCE) != 0
    safe = {(int(r["query"]), int(r["hop"])) for r, yy in zip(rows[src], y[src, 1]) if yy}
    assert safe == {(0, 3), (1, 0), (1, 1)}
