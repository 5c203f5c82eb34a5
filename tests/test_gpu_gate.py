"""Batched / gated PQ search and the learned gate, through the C-ABI.

* beam width 1 of the batched search is the reference's expansion order:
  bit-identical to the exact mode;
* wider beams keep recall@10 within 0.002 of the exact mode (or above it);
* trace rows agree with the search statistics;
* the gate's device gradients agree with the CPU oracle
  (oracle/gate_oracle.py) and device training learns a separable rule;
* the gate's limits: refine-all corrects the whole seed shortlist,
  refine-none none of it, a stop threshold every step passes stops at once.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import gate_oracle as G

pytestmark = pytest.mark.gpu

_IDX = {}


def _index():
    if not _IDX:
        from rover_b200 import bundle as B
        from rover_b200 import datasets as D
        n, dim = 20000, 128
        base = D.gmm(n, dim, 16, 11)
        queries = D.gmm(300, dim, 16, 12, centers_seed=11)
        graph = D.navigable_graph(base, 32, 24, 1.2, long_edges=4, clusters=16)
        entry = D.medoid(base)
        book, codes, rows, qp = D.pq_prepare(base, 16, 256, 6, 8)
        bundle = B.PqBundle(B.PqMeta(b"\x02" * 16, n, dim, 16, 256, 8, 16), book, codes, 8,
                            B.pack_residual_blocks(rows), qp)
        gt = D.exact_knn(queries, base, 10)
        _IDX.update(graph=graph, entry=entry, bundle=bundle, queries=queries, gt=gt)
    return _IDX


def _load(calc):
    d = _index()
    calc.pq_load(d["graph"], d["entry"], d["bundle"])
    return d


def _recall(r, gt):
    from rover_b200.workloads import recall_at_k
    return recall_at_k(r["ids"], r["counts"], gt, 10)


KW = dict(top_k=10, entry_points=64, expand_count=24, correction=1, refine_budget=20)


def test_beam_width_one_is_the_exact_search(calc):
    d = _load(calc)
    pools = np.random.default_rng(3).choice([16, 32, 64], size=len(d["queries"])).astype(np.int32)
    ex = calc.pq_search(d["queries"], pools, pool_stride=64, layout=2, **KW)
    bt = calc.pq_search(d["queries"], pools, pool_stride=64, mode=1, beam_width=1, **KW)
    for k in ("ids", "counts", "pool_ids", "pool_counts", "stats"):
        assert np.array_equal(ex[k], bt[k]), k
    for k in ("dists", "pool_dists"):
        assert np.array_equal(ex[k].view(np.uint32), bt[k].view(np.uint32)), k


@pytest.mark.parametrize("width", [2, 4])
def test_wider_beams_keep_recall(calc, width):
    d = _load(calc)
    ex = calc.pq_search(d["queries"], 48, layout=2, **KW)
    bt = calc.pq_search(d["queries"], 48, mode=1, beam_width=width, **KW)
    r_ex, r_bt = _recall(ex, d["gt"]), _recall(bt, d["gt"])
    assert r_bt >= r_ex - 0.002, (r_ex, r_bt)
    # fewer serial steps: expansions grow by less than the width
    assert bt["stats"][:, 2].mean() < width * ex["stats"][:, 2].mean()


def test_trace_rows_agree_with_statistics(calc):
    d = _load(calc)
    q = d["queries"][:64]
    tr = calc.pq_trace(q, 32, capacity=200000, **KW)
    ex = calc.pq_search(q, 32, layout=2, **KW)
    assert np.array_equal(tr["ids"], ex["ids"]) and np.array_equal(tr["stats"], ex["stats"])
    rows = tr["rows"]
    assert tr["row_count"] == len(rows)
    src = (rows["flags"] & 2) != 0
    seed = (rows["flags"] & 4) != 0
    cand = ~src & ~seed
    per_q = lambda mask: np.bincount(rows["query"][mask], minlength=len(q))
    stats = tr["stats"].astype(np.int64)
    assert np.array_equal(per_q(src), stats[:, 2])                       # one row per expansion
    n_seeds = stats[:, 0] - per_q(cand)                                   # scored = seeds + candidates
    assert np.all(n_seeds == n_seeds[0]) and n_seeds[0] > 0
    # seed rows: the ADC shortlist (twice the pool); entered = in the seed pool
    assert np.all(per_q(seed) == min(2 * 32, n_seeds[0]))
    for i in range(len(q)):
        rq = rows[rows["query"] == i]
        cand_ids = rq[cand[rows["query"] == i]]["id"]
        seed_ids = rq[seed[rows["query"] == i]]["id"]
        assert len(np.unique(cand_ids)) == len(cand_ids)            # each candidate scored once
        assert not np.intersect1d(cand_ids, seed_ids).size           # seeds are never re-scored
        entered = set(rq[(~src[rows["query"] == i]) & ((rq["flags"] & 1) != 0)]["id"].tolist())
        for rid in ex["ids"][i, :ex["counts"][i]]:
            if rid in set(cand_ids.tolist()):
                assert rid in entered


def _gate_data(n=300, seed=0):
    rng = np.random.default_rng(seed)
    x = np.stack([rng.normal(3, 1, n), rng.random(n), rng.normal(3, 0.5, n), rng.random(n),
                  rng.normal(10, 2, n)], 1).astype(np.float32)
    y = np.stack([(x[:, 0] < x[:, 2]), (x[:, 3] > 0.6)], 1).astype(np.float32)
    m = (rng.random((n, 2)) < 0.9).astype(np.float32)
    return x, y, m


def test_gate_gradients_match_the_oracle(calc):
    x, y, m = _gate_data()
    mu, sigma = x.mean(0), x.std(0)
    params = G.init_params(7)
    pw = (1.7, 0.6)
    loss_d, grad_d = calc.gate_grad(x, y, m, params, mu, sigma, pw)
    loss_o, grad_o = G.loss_and_grad(params, mu, sigma, x, y, m, pw)
    assert abs(loss_d - loss_o) <= 1e-4 * abs(loss_o) + 1e-6
    off = 0
    for name, shape in G.SIZES:
        k = int(np.prod(shape))
        gd, go = grad_d[off:off + k], grad_o[off:off + k]
        rel = np.linalg.norm(gd - go) / max(np.linalg.norm(go), 1e-12)
        assert rel < 1e-3, (name, rel)
        off += k


def test_gate_training_learns_a_separable_rule(calc):
    x, y, m = _gate_data(40000, seed=1)
    m[:] = 1.0
    out = calc.gate_train(x, y, m, epochs=6, batch=1024, lr=3e-3, seed=2)
    losses = out["losses"]
    assert losses[-1] < 0.5 * losses[0], losses
    z, _ = G.forward(out["params"], out["mu"], out["sigma"], x)
    acc = ((z > 0) == (y > 0.5)).mean(0)
    assert acc[0] > 0.97 and acc[1] > 0.97, acc


def _seed_count(n, entry, entry_points, seed=42):
    """Distinct entry seeds (graph entry, then the LCG draws)."""
    ids, lcg = [], seed
    for i in range(min(entry_points, n)):
        if i == 0 and 0 <= entry < n:
            ids.append(entry)
        else:
            lcg = (lcg * 1103515245 + 12345) & 0xFFFFFFFF
            ids.append((lcg * n) >> 32)
    return len(set(ids))


def test_gate_limits(calc):
    d = _load(calc)
    q = d["queries"][:128]
    params = G.init_params(0)
    mu, sigma = np.zeros(5, np.float32), np.ones(5, np.float32)
    calc.gate_unload()
    batched = calc.pq_search(q, 32, mode=1, beam_width=2, **KW)
    no_gate = calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    assert np.array_equal(batched["ids"], no_gate["ids"]) and np.array_equal(batched["stats"], no_gate["stats"])
    n_seeds = _seed_count(len(d["graph"]), d["entry"], KW["entry_points"])
    short = min(2 * 32, n_seeds)
    # every ratio inside the "correct" side: the seed shortlist and every
    # expansion candidate corrected, the other seeds ranked by ADC only
    calc.gate_load(params, mu, sigma, band_lo=np.inf, band_hi=np.inf, refine_logit=0.0, stop_logit=np.inf)
    all_ = calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    st = all_["stats"].astype(np.int64)
    assert np.all(st[:, 0] - st[:, 1] == n_seeds - short)
    # every ratio on the "keep" side: no seed corrected (expansion
    # candidates always are)
    calc.gate_load(params, mu, sigma, band_lo=-1.0, band_hi=0.0, refine_logit=0.0, stop_logit=np.inf)
    none = calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    sn = none["stats"].astype(np.int64)
    assert np.all(sn[:, 1] == sn[:, 0] - n_seeds)
    assert _recall(all_, d["gt"][:128]) >= _recall(none, d["gt"][:128])
    # a stop threshold every query passes: no expansion at all
    calc.gate_load(params, mu, sigma, band_lo=np.inf, band_hi=np.inf, refine_logit=0.0, stop_logit=-np.inf)
    stop = calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    assert np.all(stop["stats"][:, 2] == 0)
    calc.gate_unload()


def test_gate_rows_count_the_network_evaluations(calc):
    """calculator_rover_gate_rows counts the MLP rows the searches ran: none
    when the thresholds keep the network out, the stop head's sources (one
    row per expansion source) when it is on, and every shortlisted seed when
    the refine band covers all ratios."""
    d = _load(calc)
    q = d["queries"][:64]
    params = G.init_params(0)
    mu, sigma = np.zeros(5, np.float32), np.ones(5, np.float32)
    calc.gate_load(params, mu, sigma, band_lo=np.inf, band_hi=np.inf, refine_logit=-np.inf, stop_logit=np.inf)
    calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    assert calc.gate_rows() == 0
    # stop head on but never firing: one row per expansion source
    calc.gate_load(params, mu, sigma, band_lo=np.inf, band_hi=np.inf, refine_logit=-np.inf, stop_logit=3e38)
    r = calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    assert calc.gate_rows() == int(r["stats"][:, 2].sum())
    # refine band open over every ratio: every shortlisted seed is a row
    n_seeds = _seed_count(len(d["graph"]), d["entry"], KW["entry_points"])
    calc.gate_load(params, mu, sigma, band_lo=-1.0, band_hi=np.inf, refine_logit=0.0, stop_logit=np.inf)
    calc.pq_search(q, 32, mode=2, beam_width=2, **KW)
    assert calc.gate_rows() == len(q) * min(2 * 32, n_seeds)
    calc.gate_unload()


RULES = ("hop", "rank", "ratio")


def test_trained_stop_head_beats_the_method_without_it(calc):
    """What the trained network gains over the method without it.  On the
    100K x 128 workload (256 entry seeds, L = 48), the gate is trained on the
    traces of 4,000 held-out queries; on the traces of the workload's 2,000
    queries its stop head saves more expansions than a threshold on any one
    of its inputs (hop count, source rank, source / worst distance) at every
    loss budget of final top-10 results, and at least twice as many at the
    tight budgets.  In the gated search kernel, the network's threshold for
    a 0.5 % budget cuts expansions while the top-10 stay within that budget
    of the same search without stopping."""
    from rover_b200 import gate as gate_mod
    from rover_b200 import workloads
    w = workloads.build_pq("pq_100k_d128", verbose=False)
    calc.pq_load(w.graph, w.entry, w.bundle)
    kw = dict(entry_points=256, expand_count=48, correction=1, refine_budget=20)
    L = 48
    train_q = workloads.training_queries("pq_100k_d128", 4000, offset=8)
    rows, ids, counts = gate_mod.collect(calc, train_q, L, top_k=10, **kw)
    model = gate_mod.train(calc, rows, ids, counts, L, top_k=10, epochs=6, seed=1)
    er, eids, ecounts = gate_mod.collect(calc, w.queries, L, top_k=10, **kw)
    _, scores = gate_mod.stop_scores(calc, model, er, L)
    budgets = ("0.002", "0.005", "0.01", "0.02")
    res = gate_mod.stop_savings(er, eids, ecounts, scores, top_k=10, budgets=tuple(float(b) for b in budgets))
    table = {k: [round(v[b]["saved"], 3) for b in budgets] for k, v in res.items()}
    for b in budgets:
        best_rule = max(res[r][b]["saved"] for r in RULES)
        assert res["network"][b]["saved"] >= best_rule, table
    for b in ("0.002", "0.005"):
        assert res["network"][b]["saved"] >= 2 * max(res[r][b]["saved"] for r in RULES), table
    # the same threshold inside the gated kernel (beam width 1, every
    # shortlisted seed corrected)
    thr = res["network"]["0.005"]["threshold"]
    model.load(calc, band_lo=np.inf, band_hi=np.inf, refine_logit=-np.inf, stop_logit=np.inf)
    full = calc.pq_search(w.queries, L, top_k=10, mode=2, beam_width=1, **kw)
    model.load(calc, band_lo=np.inf, band_hi=np.inf, refine_logit=-np.inf, stop_logit=thr)
    stop = calc.pq_search(w.queries, L, top_k=10, mode=2, beam_width=1, **kw)
    calc.gate_unload()
    exp_full = full["stats"][:, 2].astype(np.int64).sum()
    exp_stop = stop["stats"][:, 2].astype(np.int64).sum()
    kept = np.mean([len(np.intersect1d(stop["ids"][i, :10], full["ids"][i, :10])) / 10 for i in range(len(w.queries))])
    assert exp_stop <= 0.85 * exp_full, (exp_stop, exp_full)
    assert kept >= 1.0 - 0.005 - 0.01, kept
